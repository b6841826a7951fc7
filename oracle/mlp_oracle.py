"""NumPy restatement of the radius-surrogate network (FP64).

TEST INFRASTRUCTURE ONLY: the checker for the GPU training kernels
(smoldyn_b200/csrc/surrogate.cu k_mlp_grad / k_mlp_forward).  Same parameter
layout and input normalisation as the device code:
  W1[64][3] b1[64] W2[64][64] b2[64] W3[2][64] b3[2]
  xn = (x - XO) * XS, h1 = tanh(W1 xn + b1), h2 = tanh(W2 h1 + b2), y = W3 h2 + b3
  loss = mean over samples of sum over the two outputs of LOSS_W[o] (y - t)^2
"""
import numpy as np

NIN, NHID, NOUT = 3, 64, 2
LOSS_W = np.array([1.0, 0.1])
LK_LO, LK_HI, RHO_HI = -5.5, 3.1, 2.0
XO = np.array([0.5 * (LK_LO + LK_HI), 0.5 * RHO_HI, 0.5])
XS = np.array([2.0 / (LK_HI - LK_LO), 2.0 / RHO_HI, 2.0])


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + NHID * NIN].reshape(NHID, NIN); o += NHID * NIN
    b1 = p[o:o + NHID]; o += NHID
    W2 = p[o:o + NHID * NHID].reshape(NHID, NHID); o += NHID * NHID
    b2 = p[o:o + NHID]; o += NHID
    W3 = p[o:o + NOUT * NHID].reshape(NOUT, NHID); o += NOUT * NHID
    b3 = p[o:o + NOUT]; o += NOUT
    return W1, b1, W2, b2, W3, b3


def forward(p, x, ym=(0.0, 0.0), ys=(1.0, 1.0)):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    xn = (np.asarray(x, dtype=np.float64) - XO) * XS
    h1 = np.tanh(xn @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    yn = h2 @ W3.T + b3
    return yn * np.asarray(ys) + np.asarray(ym)


def loss_grad(p, x, t):
    """Loss and gradient with the device's normalisation before training
    (targets used as given)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    n = len(x)
    xn = (np.asarray(x, dtype=np.float64) - XO) * XS
    z1 = xn @ W1.T + b1
    h1 = np.tanh(z1)
    z2 = h1 @ W2.T + b2
    h2 = np.tanh(z2)
    y = h2 @ W3.T + b3
    e = y - np.asarray(t, dtype=np.float64)
    loss = (LOSS_W * e * e).sum() / n
    d3 = 2.0 * LOSS_W * e / n
    gW3 = d3.T @ h2
    gb3 = d3.sum(0)
    dz2 = (d3 @ W3) * (1 - h2 * h2)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * (1 - h1 * h1)
    gW1 = dz1.T @ xn
    gb1 = dz1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g

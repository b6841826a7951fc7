"""Product placement at the unbinding radius against a step recorded from the
reference (tests/golden/onestep_unbind.npz, made by tests/golden/make_golden.py
with oracle/_ref/ref_harness).

The recorded step splits 3000 immobile C molecules (C -> A + B, first-order
probability 1 - e^-10) with product_placement unbindrad 0.6: each pair of
products lies on one random direction through the reaction site, A at
0.6 * D_A / (D_A + D_B) on one side and B at 0.6 * D_B / (D_A + D_B) on the
other (rxnsetproduct, smolreact.c:1545-1548; one random rotation per event,
doreact smolreact.c:2840-2850).

CPU: the recording itself has that geometry and an isotropic orientation
(pins what the engine is compared with).
GPU: the engine runs the same configuration from the same start state; its
products have the same geometry (distances to 1e-5 of the box-local
precision), and the orientation of the product axis has the reference's
distribution: two-sample KS tests of each component of the unit axis and of
its azimuth against the recording, and one-sample tests against the
isotropic law (each component uniform on [-1, 1]).
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest
from scipy import stats

import smoldyn_b200 as sb

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "onestep_unbind.npz")
DA, DB = 1.0, 0.5


def min_image(v, L):
    return v - L * np.rint(v / L)


def product_axes(site, pa, pb, ub, L):
    """Pair every A with the B of the same event and return (unit axes A->B,
    |B-A| - ub, reconstructed site error), matching each C site to the
    D-weighted point between its products."""
    fa, fb = DA / (DA + DB), DB / (DA + DB)
    out_u, dist_err, site_err = [], [], []
    for c in site:
        da = np.linalg.norm(min_image(pa - c, L), axis=1)
        db = np.linalg.norm(min_image(pb - c, L), axis=1)
        ia, ib = int(np.argmin(np.abs(da - ub * fa))), int(np.argmin(np.abs(db - ub * fb)))
        va, vb = min_image(pa[ia] - c, L), min_image(pb[ib] - c, L)
        v = vb - va
        out_u.append(v / np.linalg.norm(v))
        dist_err.append(np.linalg.norm(v) - ub)
        site_err.append(np.linalg.norm(fb * va + fa * vb))  # D-weighted site: fb*(A-c) + fa*(B-c) = 0
    return np.array(out_u), np.array(dist_err), np.array(site_err)


def recorded():
    g = np.load(FIX)
    L, ub = float(g["L"]), float(g["ub"])
    site = g["pos0"]
    pa = g["pos1"][g["sp1"] == 1]
    pb = g["pos1"][g["sp1"] == 2]
    return g, L, ub, site, pa, pb


def test_recording_geometry_and_isotropy():
    g, L, ub, site, pa, pb = recorded()
    assert len(pa) == len(pb) == len(site) == 3000
    u, de, se = product_axes(site, pa, pb, ub, L)
    assert np.abs(de).max() < 1e-9 and se.max() < 1e-9
    for k in range(3):
        assert stats.kstest(u[:, k], "uniform", args=(-1, 2)).pvalue > 1e-3


@pytest.mark.gpu
def test_engine_placement_matches_recording():
    g, L, ub, site, pa_ref, pb_ref = recorded()
    lib = sb.load()
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(str(g["config"]))
        simp = C.c_void_p()
        assert lib.smolLoadSimFromFile((d + "/").encode(), b"c.txt", C.byref(simp), b"") == 0, sb.last_error()
    s = sb.Sim(ptr=simp.value)
    s.set_molecules(site, g["sp0"], g["serno0"])
    s.update()
    s.run_steps(1)
    pos, sp, _ = s.molecules()
    s.close()
    pa, pb = pos[sp == 1], pos[sp == 2]
    assert len(pa) == len(pb) and len(pa) >= 2990  # a C survives with probability e^-10
    u_ref, _, _ = product_axes(site, pa_ref, pb_ref, ub, L)
    u, de, se = product_axes(site, pa, pb, ub, L)
    ok = np.abs(de) < 0.5 * ub  # events only (a surviving C has no products)
    u, de, se = u[ok], de[ok], se[ok]
    assert len(u) == len(pa)
    # box-local FP32 coordinates: 1e-5 of the box side bounds the rounding
    assert np.abs(de).max() < 1e-5 * L and se.max() < 1e-5 * L, (np.abs(de).max(), se.max())
    for k in range(3):
        p2 = stats.ks_2samp(u[:, k], u_ref[:, k]).pvalue
        p1 = stats.kstest(u[:, k], "uniform", args=(-1, 2)).pvalue
        assert p2 > 1e-3 and p1 > 1e-3, (k, p2, p1)
    az, az_ref = np.arctan2(u[:, 1], u[:, 0]), np.arctan2(u_ref[:, 1], u_ref[:, 0])
    assert stats.ks_2samp(az, az_ref).pvalue > 1e-3

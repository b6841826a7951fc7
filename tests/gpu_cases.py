"""Shared builders for the GPU parity tests (deterministic single steps)."""
import numpy as np

import smoldyn_b200 as sb
from tests import oracle_lib


def make_sim(L=20.0, wall="r", kf=20.0, kr=1.0, difc=(1.0, 1.0, 0.5), dt=0.01, seed=5, rev_placement=None,
             molperbox=None):
    s = sb.Sim(3, (0, 0, 0), (L, L, L))
    for nm, d in zip(("A", "B", "C"), difc):
        s.add_species(nm, d)
    for d in range(3):
        s.boundary(d, -1, wall)
    s.set_times(0, 1000, dt)
    s.seed(seed)
    s.add_reaction("fwd", "A", "B", ["C"], kf)
    s.add_reaction("rev", "C", None, ["A", "B"], kr)
    if rev_placement is not None:
        s.set_products("rev", *rev_placement)
    if molperbox is not None:
        s.lib.smolSetPartitions(s.ptr, b"molperbox", float(molperbox))
    return s


def random_state(n, L, rng, frac=(0.4, 0.4, 0.2)):
    pos = rng.uniform(0, L, size=(n, 3))
    sp = rng.choice([1, 2, 3], size=n, p=list(frac)).astype(np.int32)
    serno = np.arange(1, n + 1, dtype=np.uint64)
    return pos, sp, serno


def oracle_net(sim, L, wall, difc, bind2, rev_prdpos=(0.0, 0.0)):
    net = oracle_lib.OraNet()
    net.dim = 3
    for d in range(3):
        net.lo[d] = 0.0
        net.hi[d] = L
        net.wall[d][0] = wall.encode()
        net.wall[d][1] = wall.encode()
    net.nsp = 4
    for i, dc in enumerate(difc):
        net.difc[i + 1] = dc
    net.nr1 = 1
    net.r1_rct[0] = 3
    net.r1_nprod[0] = 2
    net.r1_prd[0][0] = 1
    net.r1_prd[0][1] = 2
    net.r1_prdpos[0][0][0] = rev_prdpos[0]
    net.r1_prdpos[0][1][0] = rev_prdpos[1]
    net.nr2 = 1
    net.r2_rct[0][0] = 1
    net.r2_rct[0][1] = 2
    net.r2_bind2[0] = bind2
    net.r2_nprod[0] = 1
    net.r2_prd[0][0] = 3
    return net


def min_image(v, L, periodic):
    if periodic:
        v = v - L * np.round(v / L)
    return v


def near_threshold(pos, sp, bind2, L, periodic, rel=2e-4):
    """Molecules with an A-B partner whose squared distance is within `rel` of
    the binding radius squared (FP32 and FP64 may disagree on those)."""
    ia = np.where(sp == 1)[0]
    ib = np.where(sp == 2)[0]
    out = set()
    if len(ia) == 0 or len(ib) == 0:
        return out
    for i in ia:
        v = min_image(pos[ib] - pos[i], L, periodic)
        d2 = (v * v).sum(1)
        close = np.abs(d2 - bind2) < rel * bind2
        if close.any():
            out.add(int(i))
            out.update(int(j) for j in ib[close])
    return out


def apply_walls_np(p, L, wall):
    p = p.copy()
    if wall == "p":
        return np.mod(p, L)
    if wall == "r":
        p = np.where(p < 0, -p, p)
        p = np.where(p > L, 2 * L - p, p)
    return p


def ambiguous_set(moved, sp, bind2, L, periodic, alive=None):
    """Molecules in connected groups of in-radius A-B pairs that contain a
    molecule with two or more partners: first-come-first-served (reference)
    and mutual-closest (engine) resolution may pick different pairs there."""
    ia = np.where(sp == 1)[0]
    ib = np.where(sp == 2)[0]
    if alive is not None:
        ia = ia[alive[ia]]
        ib = ib[alive[ib]]
    adj = {}
    for i in ia:
        v = min_image(moved[ib] - moved[i], L, periodic)
        d2 = (v * v).sum(1)
        for j in ib[d2 <= bind2 * (1 + 2e-4)]:
            adj.setdefault(int(i), set()).add(int(j))
            adj.setdefault(int(j), set()).add(int(i))
    out = set()
    seen = set()
    for s0 in adj:
        if s0 in seen:
            continue
        comp, stack = set(), [s0]
        while stack:
            x = stack.pop()
            if x in comp:
                continue
            comp.add(x)
            stack.extend(adj[x] - comp)
        seen |= comp
        if any(len(adj[x]) > 1 for x in comp):
            out |= comp
    return out

"""One-step golden fixtures recorded from the reference engine (see
tests/golden/make_golden.py) and the comparison used by the CPU oracle test
and the GPU test.

A final state is a dict with pos (n,3), sp (n,), serno (n,) and orig (n,) —
True for molecules that existed at the start of the step.  Two states agree
when, away from binding-radius ties and ambiguous multi-candidate groups
(where the reference's list order decides which pair reacts):
  - the same original molecules survive, at the same positions (within tol·L);
  - every product of one state has a product of the same species at the same
    position (within tol·L) in the other, unless it sits within one binding
    radius of a tied molecule.
"""
import os

import numpy as np

from tests import gpu_cases as gc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("onestep_reflect", "onestep_periodic", "onestep_sparse")
DIFC = (1.0, 1.0, 0.5)
DT = 0.01


def load(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    g = {k: d[k] for k in d.files}
    g["L"] = float(g["L"])
    g["wall"] = str(g["wall"])
    g["bind2"] = float(g["bind2"])
    g["kf"], g["kr"] = float(g["kf"]), float(g["kr"])
    return g


def reference_state(g):
    start = set(g["serno0"].tolist())
    return dict(pos=g["pos1"], sp=g["sp1"], serno=g["serno1"],
                orig=np.array([int(s) in start for s in g["serno1"].tolist()], dtype=bool))


def tie_set(g):
    """Indices (into the start state) of molecules near a binding-radius tie or
    in an ambiguous group, and their moved positions."""
    periodic = g["wall"] == "p"
    moved = gc.apply_walls_np(g["pos0"] + g["disp"], g["L"], g["wall"])
    ties = gc.near_threshold(moved, g["sp0"], g["bind2"], g["L"], periodic)
    alive = g["uni"] == 0
    amb = gc.ambiguous_set(moved, g["sp0"], g["bind2"], g["L"], periodic, alive)
    return ties | amb, moved


def compare(g, exp, act, tol):
    L, periodic = g["L"], g["wall"] == "p"
    idx, moved = tie_set(g)
    tie_sn = {int(g["serno0"][i]) for i in idx}
    tie_pos = moved[sorted(idx)] if idx else np.zeros((0, 3))
    e_sn = {int(s): i for i, s in enumerate(exp["serno"].tolist()) if exp["orig"][i]}
    a_sn = {int(s): i for i, s in enumerate(act["serno"].tolist()) if act["orig"][i]}
    diff = (set(e_sn) ^ set(a_sn)) - tie_sn
    assert not diff, ("survivor sets differ", len(diff), sorted(diff)[:10])
    common = sorted(set(e_sn) & set(a_sn))
    d = gc.min_image(exp["pos"][[e_sn[k] for k in common]] - act["pos"][[a_sn[k] for k in common]], L, periodic)
    assert np.abs(d).max() <= tol * L, np.abs(d).max()
    bind = np.sqrt(g["bind2"])

    def unmatched(P, Q):
        out = 0
        for sp in (1, 2, 3):
            A = P["pos"][(~P["orig"]) & (P["sp"] == sp)]
            B = Q["pos"][(~Q["orig"]) & (Q["sp"] == sp)]
            for x in A:
                if len(B) and np.abs(gc.min_image(B - x, L, periodic)).max(1).min() <= tol * L:
                    continue
                near = len(tie_pos) and np.sqrt((gc.min_image(tie_pos - x, L, periodic) ** 2).sum(1)).min() <= bind
                assert near, ("product without a counterpart", sp, x)
                out += 1
        return out

    nprod = int((~exp["orig"]).sum())
    unmatched(exp, act)
    unmatched(act, exp)
    return len(common), nprod, len(tie_sn)

"""The bucketed molecule layout against the sorted one.

Both layouts run the same per-molecule code with the same random streams
(Philox keyed by serial number and step), so the same simulation must give
the same molecules (serial numbers, species, positions) in both, up to the
ranking of exactly equidistant reaction candidates.  Checked on:
  - the scale-up network at reduced size (periodic cube, A + B <-> C, births);
  - a dense start (every molecule in a cube of side 3 inside a box of side
    30), so that boxes overflow their 32 slots and the spill list carries
    molecules through the move, the pair search (spill pass) and the conflict
    rounds, with a fast A + B -> C reaction;
  - leaving the layout for injected displacements and coming back;
  - single steps (smolRunTimeStep) in the bucketed layout.
"""
import numpy as np
import pytest

import smoldyn_b200 as sb

pytestmark = pytest.mark.gpu


def scaleup_sim(layout, n=20000, seed=11):
    L = 1000.0 * (n / 1e7) ** (1 / 3)
    s = sb.Sim(3, (0, 0, 0), (L, L, L))
    for nm, d in (("A", 1.0), ("B", 1.0), ("C", 0.5)):
        s.add_species(nm, d)
    for d in range(3):
        s.boundary(d, -1, "p")
    s.set_times(0, 1e9, 0.01)
    s.seed(seed)
    s.add_reaction("fwd", "A", "B", ["C"], 0.05)
    s.add_reaction("rev", "C", None, ["A", "B"], 0.1)
    s.add_reaction("birth", None, None, ["A"], 1e-4)
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, L, size=(n, 3))
    sp = rng.choice([1, 2, 3], size=n, p=[0.45, 0.45, 0.10]).astype(np.int32)
    s.set_molecules(pos, sp, np.arange(1, n + 1, dtype=np.uint64))
    s.bucket_layout(layout)
    s.update()
    return s


def dense_sim(layout, n=6000, seed=12):
    s = sb.Sim(3, (0, 0, 0), (30, 30, 30))
    for nm, d in (("A", 1.0), ("B", 1.0), ("C", 0.5)):
        s.add_species(nm, d)
    for d in range(3):
        s.boundary(d, -1, "r")
    s.set_times(0, 1e9, 0.01)
    s.seed(seed)
    s.add_reaction("fwd", "A", "B", ["C"], 2.0)
    rng = np.random.default_rng(seed)
    pos = rng.uniform(13.5, 16.5, size=(n, 3))
    sp = rng.choice([1, 2], size=n).astype(np.int32)
    s.set_molecules(pos, sp, np.arange(1, n + 1, dtype=np.uint64))
    s.bucket_layout(layout)
    s.update()
    return s


def compare(a, b, tol):
    pa, spa, sna = a.molecules()
    pb, spb, snb = b.molecules()
    ka, kb = np.argsort(sna), np.argsort(snb)
    common = np.intersect1d(sna, snb)
    only = len(sna) + len(snb) - 2 * len(common)
    ia = ka[np.searchsorted(sna[ka], common)]
    ib = kb[np.searchsorted(snb[kb], common)]
    assert np.array_equal(spa[ia], spb[ib])
    err = np.abs(pa[ia] - pb[ib]).max() if len(common) else 0.0
    return only, len(common), err


def test_scaleup_same_in_both_layouts():
    a, b = scaleup_sim(1), scaleup_sim(0)
    assert a.bucket_layout() == 1 and b.bucket_layout() == 0
    a.run_steps(100)
    b.run_steps(100)
    assert a.bucket_layout() == 1
    only, common, err = compare(a, b, 1e-4)
    print("scale-up: %d molecules in both, %d in one only, max position difference %.2e" % (common, only, err))
    assert only <= 2 and err < 1e-4
    assert [a.count(x) for x in "ABC"] == [b.count(x) for x in "ABC"] or only > 0
    a.close()
    b.close()


def test_dense_start_uses_spill_and_matches():
    a, b = dense_sim(1), dense_sim(0)
    assert a.bucket_layout() == 1
    for _ in range(4):
        a.run_steps(5)
        b.run_steps(5)
        only, common, err = compare(a, b, 1e-4)
        assert only <= 4 and err < 1e-4, (only, err)
    ea, eb = a.events(), b.events()
    print("dense: second-order events %d / %d, status %d / %d" % (ea[3], eb[3], ea[6], eb[6]))
    assert ea[3] > 500 and ea[6] == 0 and eb[6] == 0
    assert abs(ea[3] - eb[3]) <= 2
    a.close()
    b.close()


def test_leave_for_injection_and_return():
    s = scaleup_sim(1, n=5000, seed=13)
    assert s.bucket_layout() == 1
    s.run_steps(3)
    pos, sp, sn = s.molecules()
    disp = np.zeros((len(sn), 4))
    disp[:, 3] = -1
    s.inject(sn, disp)           # deterministic mode: the sorted layout
    s.run_steps(1)
    assert s.bucket_layout() == 0
    pos1, sp1, sn1 = s.molecules()
    k0, k1 = np.argsort(sn), np.argsort(sn1)
    same = np.intersect1d(sn, sn1)
    assert len(same) >= len(sn) - 50
    s.run_steps(3)               # back in buckets
    assert s.bucket_layout() == 1
    assert s.total() > 0
    s.close()


def test_single_steps_in_buckets():
    a, b = scaleup_sim(1, n=8000, seed=14), scaleup_sim(0, n=8000, seed=14)
    for _ in range(12):
        a.run_step()
        b.run_step()
        ca, cb = [a.count(x) for x in "ABC"], [b.count(x) for x in "ABC"]
        assert sum(abs(x - y) for x, y in zip(ca, cb)) <= 2, (ca, cb)
    assert a.bucket_layout() == 1
    a.close()
    b.close()

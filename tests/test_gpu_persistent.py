"""The persistent ensemble kernel against the step pipeline.

Both engines step the same ensemble (same seed, boxes, rates and molecules)
with the same per-molecule code and random streams (Philox keyed by serial
number and step), so they must give the same trajectory replicate by
replicate; they differ only in the order of molecules inside a box, which
ranks exactly equidistant reaction candidates differently.  Checked on:
  - an A + B <-> C ensemble with per-replicate rates and uneven sizes
    (reflective cubes, unbinding ratio 1.5 for the reverse products), over
    100 steps in blocks of 7 and 93 steps (odd blocks exercise the buffer
    parity and a launch boundary mid-run);
  - births, first-order decay and absorbing walls (periodic on one axis);
  - the molecules themselves after the run (positions, species, serial
    numbers), read back through the step pipeline's layout;
  - stepping on after the read-back, and switching engines mid-run.
The engine choice is reported by smolgpuEnsembleGetEngine; the default
(mode 0) is the step pipeline.
"""
import numpy as np
import pytest

import smoldyn_b200 as sb

pytestmark = pytest.mark.gpu


def reversible(R, seed=5):
    rng = np.random.default_rng(seed)
    n = np.rint(10 ** rng.uniform(2, 3.7, R)).astype(np.int64)
    side = (n / 0.01) ** (1.0 / 3.0)
    kf = 10 ** rng.uniform(-2, 0.5, R)
    kr = 10 ** rng.uniform(-2, 0, R)
    s = sb.Sim(3, (0, 0, 0), (1, 1, 1))
    for nm, d in (("A", 1.0), ("B", 1.0), ("C", 0.5)):
        s.add_species(nm, d)
    for d in range(3):
        s.boundary(d, -1, "r")
    s.set_times(0, 1e9, 0.01)
    s.seed(99)
    s.add_reaction("fwd", "A", "B", ["C"], 0.05)
    s.add_reaction("rev", "C", None, ["A", "B"], 0.1)
    s.set_products("rev", sb.RPratio, 1.5)
    e = sb.Ensemble(s, R)
    e.set_boxes(np.zeros((R, 3)), np.repeat(side[:, None], 3, 1))
    e.set_rates("fwd", kf)
    e.set_rates("rev", kr)
    e.add_molecules("A", n // 2 + n % 2)
    e.add_molecules("B", n // 2)
    return e


def births_decay(R):
    s = sb.Sim(3, (0, 0, 0), (25, 25, 25))
    for nm, d in (("A", 1.0), ("B", 0.5), ("C", 0.3)):
        s.add_species(nm, d)
    s.boundary(0, -1, "a")
    s.boundary(1, -1, "p")
    s.boundary(2, -1, "r")
    s.set_times(0, 1e9, 0.01)
    s.seed(17)
    s.add_reaction("birth", None, None, ["A"], 0.05)
    s.add_reaction("decay", "A", None, ["B"], 0.3)
    s.add_reaction("bind", "A", "B", ["C"], 2.0)
    e = sb.Ensemble(s, R)
    e.add_molecules("A", np.full(R, 300))
    return e


def run_both(make, blocks):
    out = []
    for mode in (1, 2):
        e = make()
        e.engine(mode)
        e.update()
        assert e.engine() == mode
        for b in blocks:
            e.run_steps(b)
        counts = e.counts(4)
        mols = e.molecules()
        e.close()
        out.append((counts, mols))
    return out


def compare(a, b, what):
    ca, cb = a[0], b[0]
    diff = np.nonzero(np.any(ca != cb, axis=1))[0]
    print("%s: %d of %d replicates differ; totals %s vs %s" % (what, len(diff), len(ca), ca.sum(0), cb.sum(0)))
    assert len(diff) <= max(1, len(ca) // 200), (what, diff[:10], ca[diff[:5]], cb[diff[:5]])
    return diff


def test_reversible_ensemble_same_trajectory():
    a, b = run_both(lambda: reversible(256), [7, 93])
    diff = compare(a, b, "reversible")
    # molecules of the replicates that agree: same serials, species and positions
    (pa, spa, ra, sna), (pb, spb, rb, snb) = a[1], b[1]
    keep_a = ~np.isin(ra, diff)
    keep_b = ~np.isin(rb, diff)
    ka = np.lexsort((sna[keep_a], ra[keep_a]))
    kb = np.lexsort((snb[keep_b], rb[keep_b]))
    assert np.array_equal(sna[keep_a][ka], snb[keep_b][kb])
    assert np.array_equal(spa[keep_a][ka], spb[keep_b][kb])
    err = np.abs(pa[keep_a][ka] - pb[keep_b][kb]).max()
    assert err < 1e-3, err


def test_births_decay_absorbing_same_trajectory():
    a, b = run_both(lambda: births_decay(128), [50, 51])
    compare(a, b, "births/decay/absorbing")
    assert a[0][:, 2].sum() > 0 and a[0][:, 3].sum() > 0


def test_default_engine_is_pipeline():
    e = reversible(8)
    e.update()
    assert e.engine() == 1
    e.engine(2)
    assert e.engine() == 2
    e.close()


def test_switch_engines_mid_run():
    ref = reversible(64, seed=8)
    ref.engine(1)
    ref.update()
    ref.run_steps(60)
    c_ref = ref.counts(4)
    ref.close()
    e = reversible(64, seed=8)
    e.engine(2)
    e.update()
    e.run_steps(20)
    e.molecules()                # read-back through the pipeline layout, then on
    e.run_steps(20)
    e.engine(1)                  # pipeline for the last 20 steps
    e.run_steps(20)
    c = e.counts(4)
    e.close()
    diff = np.nonzero(np.any(c != c_ref, axis=1))[0]
    assert len(diff) <= 1, diff

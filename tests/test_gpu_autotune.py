"""Autotuner (smolgpuAutotune / smolgpuEnsembleAutotune).

- After tuning, the simulation is back at its start state: the same molecules
  (serial numbers, species) at the same positions (to FP32 rounding of the
  box-local coordinates, 1e-5 of the side).
- A tuned and an untuned copy of the same simulation (same seed) stay together
  over 100 steps: species counts differ by at most 0.1% of all molecules (box
  width changes only the rounding of box-local coordinates, which can flip a
  pair at the binding-radius threshold; each flip changes that pair's later
  history, so a rare species can differ by several molecules).
- The tuner refuses to run after the first step; an ensemble can be tuned.
"""
import numpy as np
import pytest

import smoldyn_b200 as sb
from tests import gpu_cases as gc

pytestmark = pytest.mark.gpu


def _sim(seed=3):
    s = gc.make_sim(L=100.0, wall="r", kf=0.05, kr=0.1, seed=seed)
    s.add_molecules("A", 10000)
    s.add_molecules("B", 10000)
    s.update()
    return s


def test_autotune_restores_state_and_keeps_trajectory():
    s = _sim()
    pos0, sp0, sn0 = s.molecules()
    ms = s.autotune(10)
    t = s.tuning()
    assert ms > 0
    assert t["pair_tile"] in (128, 256) and t["molperbox"] in (1, 2, 4, 8)
    pos1, sp1, sn1 = s.molecules()
    o0, o1 = np.argsort(sn0), np.argsort(sn1)
    assert np.array_equal(sn0[o0], sn1[o1]) and np.array_equal(sp0[o0], sp1[o1])
    assert np.abs(pos0[o0] - pos1[o1]).max() <= 1e-5 * 100.0
    ref = _sim()
    s.run_steps(100)
    ref.run_steps(100)
    total = sum(ref.count(nm) for nm in ("A", "B", "C"))
    for nm in ("A", "B", "C"):
        assert abs(s.count(nm) - ref.count(nm)) <= max(3, 0.001 * total), (nm, s.count(nm), ref.count(nm), t)


def test_autotune_only_before_first_step():
    s = _sim()
    s.run_steps(2)
    with pytest.raises(RuntimeError, match="before the first time step"):
        s.autotune(4)


def test_ensemble_autotune():
    t = gc.make_sim(L=30.0, wall="r", kf=0.05, kr=0.1)
    e = sb.Ensemble(t, 64)
    rng = np.random.default_rng(4)
    n = rng.integers(100, 3000, 64)
    e.add_molecules("A", n)
    e.add_molecules("B", n)
    e.update()
    before = e.counts(4).copy()
    ms = e.autotune(6)
    assert ms > 0
    assert np.array_equal(e.counts(4), before)
    e.run_steps(20)
    c = e.counts(4)
    # A + C and B + C are conserved per replicate (A + B <-> C only)
    assert np.array_equal(c[:, 1] + c[:, 3], n) and np.array_equal(c[:, 2] + c[:, 3], n)

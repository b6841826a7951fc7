"""Single steps through smolRunTimeStep with a count read after each: the
counts come from the copies that the single-step graph makes of its own step
(and the status check reads the previous step's copy).  They must equal the
counts of the molecules actually present after that step, taken here by
downloading the molecules and tallying species on the host, and a bulk run
from the same start must land on counts of the same size."""
import ctypes as C

import numpy as np
import pytest

import smoldyn_b200 as sb

pytestmark = pytest.mark.gpu


def make_sim(seed):
    s = sb.Sim(3, (0, 0, 0), (60, 60, 60))
    for nm, d in (("A", 1.0), ("B", 1.0), ("C", 0.5)):
        s.add_species(nm, d)
    for d in range(3):
        s.boundary(d, -1, "p")
    s.set_times(0, 1e6, 0.01)
    s.seed(seed)
    s.add_reaction("fwd", "A", "B", ["C"], 20.0)
    s.add_reaction("rev", "C", None, ["A", "B"], 1.0)
    s.add_molecules("A", 20000)
    s.add_molecules("B", 20000)
    s.add_molecules("C", 5000)
    s.update()
    return s


def host_counts(s):
    _, sp, _ = s.molecules()
    return [int(np.count_nonzero(sp == k)) for k in (1, 2, 3)]


def test_counts_after_each_single_step_are_that_steps():
    s = make_sim(3)
    lib = s.lib
    changed = 0
    prev = None
    for step in range(40):
        assert lib.smolRunTimeStep(s.ptr) == sb.ECok, sb.last_error()
        got = [lib.smolGetMoleculeCount(s.ptr, nm, 0) for nm in (b"A", b"B", b"C")]
        if step % 5 == 4:
            assert got == host_counts(s), (step, got)
        if prev is not None and got != prev:
            changed += 1
        prev = got
    assert changed > 20  # reactions run, so the counts move from step to step
    s.close()


def test_single_steps_and_bulk_agree_in_size():
    a, b = make_sim(5), make_sim(5)
    for _ in range(60):
        assert a.lib.smolRunTimeStep(a.ptr) == sb.ECok
    b.run_steps(60)
    ca = [a.count(nm) for nm in ("A", "B", "C")]
    cb = [b.count(nm) for nm in ("A", "B", "C")]
    for x, y in zip(ca, cb):
        assert abs(x - y) <= 5 * np.sqrt(max(x, y)) + 5, (ca, cb)
    a.close()
    b.close()

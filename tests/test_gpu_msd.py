"""The meansqrdisp runtime command (cmdmeansqrdisp, smolcmd.c:2505-2606) on
the device, against the reference binary and against diffusion theory.

The same configuration runs through the reference (oracle/_ref/smoldyn, 8
seeds of 4000 molecules, its meansqrdisp output file) and through this
library's config reader (smolLoadSimFromFile, smolRunSim, smolGetOutputData)
with 32000 molecules.  Each output row is (time, <r^2>, <r^4>) over the molecules
recorded on the first call.  Checks:
- periodic cube of side 10: <r^2> keeps growing as 6 D t far beyond L^2/4
  (periodic wraps undone, as the reference does with posoffset), and agrees
  with the reference;
- reflective cube: <r^2> bends below 6 D t towards L^2/2 along the
  reference's curve;
- drift along x in a periodic cube, x axis only: 2 D t + v^2 t^2;
- an engine rebuild in the middle of a run (molecules added) keeps the
  recorded molecules and their unwrapped positions.
Tolerances: 4% for <r^2> and 8% for <r^4> (standard errors of a mean over
32000 molecules: about 0.7% and 1%; the difference of two such means, 1% and
1.4%).
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import smoldyn_b200 as sb
from tests import oracle_lib

pytestmark = pytest.mark.gpu

REF_EXE = os.path.join(oracle_lib.REF_DIR, "smoldyn")
SEEDS = 8

BASE = """dim 3
species A
difc A 1
time_start 0
time_stop {tstop}
time_step 0.01
random_seed {seed}
boundaries 0 0 10 {b}
boundaries 1 0 10 {b}
boundaries 2 0 10 {b}
{extra}
mol {nmol} A u u u
output_files msd.txt
cmd N 100 meansqrdisp A {dim} msd.txt
end_file
"""

CASES = {
    "periodic": dict(b="p", dim="all", extra="", tstop=15.0),
    "reflective": dict(b="r", dim="all", extra="", tstop=15.0),
    "drift_x": dict(b="p", dim="x", extra="drift A 2 0 0", tstop=10.0),
}


def config(case, seed, nmol):
    c = CASES[case]
    return BASE.format(tstop=c["tstop"], seed=seed, b=c["b"], extra=c["extra"], nmol=nmol, dim=c["dim"])


def parse(path):
    rows = []
    for ln in open(path):
        t = ln.replace(",", " ").split()
        if len(t) >= 3:
            try:
                rows.append([float(x) for x in t[:3]])
            except ValueError:
                pass
    return np.array(rows)


def reference_msd(case):
    env = dict(os.environ, SMOLDYN_NO_PROMPT="1")
    out = []
    with tempfile.TemporaryDirectory() as d:
        procs = []
        for seed in range(1, SEEDS + 1):
            sd = os.path.join(d, str(seed))
            os.mkdir(sd)
            with open(os.path.join(sd, "c.txt"), "w") as f:
                f.write(config(case, seed, 4000))
            procs.append(subprocess.Popen([REF_EXE, "c.txt", "-qt"], cwd=sd, stdout=subprocess.DEVNULL,
                                          stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, env=env))
        for p in procs:
            assert p.wait(timeout=900) == 0
        for seed in range(1, SEEDS + 1):
            out.append(parse(os.path.join(d, str(seed), "msd.txt")))
    n = min(len(a) for a in out)
    return np.mean([a[:n] for a in out], axis=0)


def engine_msd(case, rebuild_at=None):
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(config(case, 7, 4000 * SEEDS))
        s = sb.Sim.from_file(os.path.join(d, "c.txt"))
    if rebuild_at is None:
        s.run()
    else:
        s.run_until(rebuild_at)
        s.add_molecules("A", 100)  # pulls the molecules, rebuilds the engine
        s.run()
    return s.output_data("msd.txt")


def rows_close(got, want):
    n = min(len(got), len(want))
    assert n >= 10
    assert np.allclose(got[:n, 0], want[:n, 0], atol=1e-6)
    for k, rel in ((1, 0.04), (2, 0.08)):
        g, w = got[1:n, k], want[1:n, k]
        assert np.all(np.abs(g - w) <= rel * np.abs(w)), (k, np.max(np.abs(g / w - 1)))


def needs_reference():
    if not os.path.exists(REF_EXE):
        pytest.skip("reference binary not built")


def test_periodic_unwraps_and_matches_reference():
    needs_reference()
    eng = engine_msd("periodic")
    t = eng[:, 0]
    assert eng[0, 1] == 0 and eng[0, 2] == 0
    assert np.all(np.abs(eng[1:, 1] / (6 * t[1:]) - 1) < 0.04), eng[:, 1] / np.maximum(6 * t, 1e-9)
    # <r^4> of a 3-D Gaussian displacement: 15 (2 D t)^2
    assert np.all(np.abs(eng[1:, 2] / (15 * (2 * t[1:]) ** 2) - 1) < 0.08)
    assert eng[-1, 1] > 3 * 25.0   # far past the saturation a wrapped measure would show
    rows_close(eng, reference_msd("periodic"))


def test_reflective_saturates_like_reference():
    needs_reference()
    eng = engine_msd("reflective")
    # the walls bend the curve below free diffusion (6 D t = 90 at t = 15) on
    # its way to L^2/2 = 50, the value for independent uniform start and end
    assert 0.3 * 90 < eng[-1, 1] < 0.5 * 90 and eng[-1, 1] < 50
    rows_close(eng, reference_msd("reflective"))


def test_drift_single_axis():
    needs_reference()
    eng = engine_msd("drift_x")
    t = eng[1:, 0]
    assert np.all(np.abs(eng[1:, 1] / (2 * t + 4 * t * t) - 1) < 0.04)
    rows_close(eng, reference_msd("drift_x"))


def test_rebuild_keeps_tracking():
    eng = engine_msd("periodic", rebuild_at=5.0)
    t = eng[:, 0]
    assert len(eng) >= 15
    assert np.all(np.abs(eng[1:, 1] / (6 * t[1:]) - 1) < 0.04), eng[:, 1] / np.maximum(6 * t, 1e-9)

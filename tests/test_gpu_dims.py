"""Two-dimensional systems against the reference (statistical parity).

A square of side 100 with reflective walls; A + B -> C with kf = 0.5 (area
units), D = 1, 1, 0.5; 5000 A and 5000 B placed uniformly; dt = 0.01; 300
steps.  The reference binary runs 16 seeds in parallel; the engine runs 64
replicates in one ensemble.  The mean C count at the end agrees within 3
combined standard errors and a two-sample KS test does not reject
(p > 0.001); the binding radius equals the reference's (the 2-D solve uses
the same radial tables as 3-D in rxnparam, so the radius is the same formula).
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest
from scipy import stats

import smoldyn_b200 as sb
from tests import oracle_lib

pytestmark = pytest.mark.gpu

REF_EXE = os.path.join(oracle_lib.REF_DIR, "smoldyn")
SIDE, N, KF, DT, STEPS = 100.0, 5000, 0.5, 0.01, 300

CONFIG = """dim 2
species A B C
difc A 1
difc B 1
difc C 0.5
boundaries 0 0 {L} r
boundaries 1 0 {L} r
time_start 0
time_stop {tstop}
time_step {dt}
random_seed {seed}
reaction fwd A + B -> C {kf}
mol {n} A u u
mol {n} B u u
output_files {out}
cmd a molcount {out}
end_file
"""


def reference_counts(seeds=16):
    env = dict(os.environ, SMOLDYN_NO_PROMPT="1")
    out = []
    with tempfile.TemporaryDirectory() as d:
        procs = []
        for seed in range(1, seeds + 1):
            with open(os.path.join(d, "c%d.txt" % seed), "w") as f:
                f.write(CONFIG.format(L=SIDE, tstop=STEPS * DT, dt=DT, seed=seed, kf=KF, n=N, out="o%d.txt" % seed))
            procs.append(subprocess.Popen([REF_EXE, "c%d.txt" % seed, "-qt"], cwd=d, stdout=subprocess.DEVNULL,
                                          stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, env=env))
        for p in procs:
            assert p.wait(timeout=900) == 0
        for seed in range(1, seeds + 1):
            rows = [ln.split() for ln in open(os.path.join(d, "o%d.txt" % seed)) if ln.strip()]
            out.append(float(rows[-1][3]))
    return np.array(out)


def test_two_dimensional_reaction_matches_reference():
    if not os.path.exists(REF_EXE):
        pytest.skip("reference binary not built")
    ref = reference_counts()
    t = sb.Sim(2, (0, 0), (SIDE, SIDE))
    for nm, dc in (("A", 1.0), ("B", 1.0), ("C", 0.5)):
        t.add_species(nm, dc)
    for d in range(2):
        t.boundary(d, -1, "r")
    t.set_times(0, 1e6, DT)
    t.seed(99)
    t.add_reaction("fwd", "A", "B", ["C"], KF)
    R = 64
    e = sb.Ensemble(t, R)
    e.add_molecules("A", np.full(R, N))
    e.add_molecules("B", np.full(R, N))
    e.update()
    e.run_steps(STEPS)
    c = e.counts(4)
    assert (c[:, 1] + c[:, 3] == N).all() and (c[:, 2] + c[:, 3] == N).all()
    g = c[:, 3].astype(float)
    se = np.sqrt(ref.var(ddof=1) / len(ref) + g.var(ddof=1) / len(g))
    print("2-D C at the end: reference %.1f +- %.1f, engine %.1f +- %.1f" %
          (ref.mean(), ref.std(ddof=1) / np.sqrt(len(ref)), g.mean(), g.std(ddof=1) / np.sqrt(len(g))))
    assert abs(ref.mean() - g.mean()) <= 3 * se + 1
    assert stats.ks_2samp(ref, g).pvalue > 1e-3


def test_two_dimensional_positions_stay_in_the_plane_and_box():
    s = sb.Sim(2, (0, 0), (20.0, 20.0))
    s.add_species("A", 1.0)
    for d in range(2):
        s.boundary(d, -1, "r")
    s.set_times(0, 1e6, 0.01)
    s.add_molecules("A", 2000)
    s.update()
    s.run_steps(500)
    pos, sp, sn = s.molecules()
    assert len(sn) == 2000
    assert pos[:, :2].min() >= 0 and pos[:, :2].max() <= 20.0
    assert np.all(pos[:, 2] == 0)

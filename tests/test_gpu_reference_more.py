"""More behaviour against reference ensembles: absorbing walls, zeroth-order
births with first-order decay, branching first-order reactions, drift, and
reversible A + B <-> C in one and two dimensions (the products' unbinding
offsets take a random sign in 1-D and a random in-plane angle in 2-D).

Each case runs the same text configuration through the reference binary
(oracle/_ref/smoldyn, 32 seeds in parallel, molcount at the end) and through
the engine as an ensemble of 48 replicates built from the same configuration
(config reader → template simulation → smolgpuNewEnsemble).  The mean end
count of each species agrees within 3 combined standard errors (+1 molecule
for the discreteness of counts).
"""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

import smoldyn_b200 as sb
from tests import oracle_lib

pytestmark = pytest.mark.gpu

REF_EXE = os.path.join(oracle_lib.REF_DIR, "smoldyn")
SEEDS, NREP = 32, 48

HEAD = """dim {dim}
species A B C
difc A 1
difc B 0.5
difc C 0.3
time_start 0
time_stop {tstop}
time_step 0.01
random_seed {seed}
"""

CASES = {
    # x walls absorb (including the reference's second coin for molecules that
    # stay inside, smolwall.c:417-420); y and z reflect
    "absorbing_walls": dict(steps=300, body="""boundaries 0 0 20 a
boundaries 1 0 20 r
boundaries 2 0 20 r
mol 2000 A u u u
"""),
    # births 0 -> A at 0.02 per unit volume per unit time, A -> 0 at 0.5
    "births_and_decay": dict(steps=400, body="""boundaries 0 0 30 r
boundaries 1 0 30 r
boundaries 2 0 30 r
reaction birth 0 -> A 0.02
reaction decay A -> 0 0.5
"""),
    # C -> A (0.2) and C -> B (0.1) compete: branching 2:1
    "branching": dict(steps=200, body="""boundaries 0 0 20 r
boundaries 1 0 20 r
boundaries 2 0 20 r
reaction toA C -> A 0.2
reaction toB C -> B 0.1
mol 5000 C u u u
"""),
    # reversible binding in the plane and on a line (default pgemmaxw placement)
    "reversible_2d": dict(steps=300, dim=2, init=[("A", 1500), ("B", 1500)], body="""boundaries 0 0 40 r
boundaries 1 0 40 r
reaction fwd A + B <-> C 5 0.5
mol 1500 A u u
mol 1500 B u u
"""),
    "reversible_1d": dict(steps=300, dim=1, init=[("A", 400), ("B", 400)], body="""boundaries 0 0 200 r
reaction fwd A + B <-> C 2 0.5
mol 400 A u
mol 400 B u
"""),
}


def config(case, seed, out):
    c = CASES[case]
    return (HEAD.format(dim=c.get("dim", 3), tstop=c["steps"] * 0.01, seed=seed) + c["body"] +
            "output_files %s\ncmd a molcount %s\nend_file\n" % (out, out))


def reference_counts(case):
    env = dict(os.environ, SMOLDYN_NO_PROMPT="1")
    rows = []
    with tempfile.TemporaryDirectory() as d:
        procs = []
        for seed in range(1, SEEDS + 1):
            with open(os.path.join(d, "c%d.txt" % seed), "w") as f:
                f.write(config(case, seed, "o%d.txt" % seed))
            procs.append(subprocess.Popen([REF_EXE, "c%d.txt" % seed, "-qt"], cwd=d, stdout=subprocess.DEVNULL,
                                          stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, env=env))
        for p in procs:
            assert p.wait(timeout=600) == 0
        for seed in range(1, SEEDS + 1):
            last = [ln.split() for ln in open(os.path.join(d, "o%d.txt" % seed)) if ln.strip()][-1]
            rows.append([float(x) for x in last[1:4]])
    return np.array(rows)  # [seed, species A B C]


def engine_counts(case):
    lib = sb.load()
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(config(case, 1, "o.txt"))
        simp = C.c_void_p()
        assert lib.smolLoadSimFromFile((d + "/").encode(), b"c.txt", C.byref(simp), b"") == 0, sb.last_error()
    t = sb.Sim(ptr=simp.value)
    e = sb.Ensemble(t, NREP)
    init = {"absorbing_walls": [("A", 2000)], "branching": [("C", 5000)]}.get(case, CASES[case].get("init", []))
    for sp, n in init:
        e.add_molecules(sp, np.full(NREP, n))
    e.update()
    e.run_steps(CASES[case]["steps"])
    return e.counts(4)[:, 1:4].astype(float)


@pytest.mark.parametrize("case", sorted(CASES))
def test_end_counts_match_reference(case):
    if not os.path.exists(REF_EXE):
        pytest.skip("reference binary not built")
    ref = reference_counts(case)
    eng = engine_counts(case)
    for k, nm in enumerate("ABC"):
        r, g = ref[:, k], eng[:, k]
        if r.max() == 0 and g.max() == 0:
            continue
        se = np.sqrt(r.var(ddof=1) / len(r) + g.var(ddof=1) / len(g))
        print("%s %s: reference %.1f +- %.1f, engine %.1f +- %.1f" %
              (case, nm, r.mean(), r.std(ddof=1) / np.sqrt(len(r)), g.mean(), g.std(ddof=1) / np.sqrt(len(g))))
        assert abs(r.mean() - g.mean()) <= 3 * se + 1, (case, nm, r.mean(), g.mean(), se)


def test_drift_moves_the_mean():
    """drift (smolmolec.c:3149): the mean displacement after time t is v t,
    the spread stays 2 D t per axis."""
    L, n, dt, steps = 1000.0, 20000, 0.01, 200
    s = sb.Sim(3, (0, 0, 0), (L, L, L))
    s.add_species("A", 1.0)
    for d in range(3):
        s.boundary(d, -1, "r")
    s.set_times(0, 1e6, dt)
    v = np.array([3.0, -1.0, 0.5])
    assert s.lib.smolSetSpeciesMobility(s.ptr, b"A", sb.MSsoln, 1.0, sb.dptr(v), None) == 0
    rng = np.random.default_rng(9)
    pos0 = rng.uniform(400, 600, size=(n, 3))
    s.set_molecules(pos0, np.ones(n, dtype=np.int32), np.arange(1, n + 1, dtype=np.uint64))
    s.run_steps(steps)
    pos1, _, sn = s.molecules()
    disp = pos1[np.argsort(sn)] - pos0
    t = steps * dt
    mean_se = np.sqrt(2 * 1.0 * t / n)
    assert np.all(np.abs(disp.mean(0) - v * t) <= 4 * mean_se), (disp.mean(0), v * t)
    assert np.all(np.abs(disp.var(0) / (2 * t) - 1.0) < 0.05), disp.var(0) / (2 * t)

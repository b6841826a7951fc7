"""Plain small workload against reference ensembles (statistical parity).

Workload: cube of side 100 with reflective walls; A, B, C with D = 1, 1, 0.5;
A + B <-> C with kf = 0.05, kr = 0.1 and the reference's default product
placement for the reverse reaction; 10^4 A and 10^4 B placed uniformly;
dt = 0.01; 1000 steps.

The reference binary (oracle/_ref/smoldyn, built from the reference sources)
runs 32 seeds in parallel and records molcount every 50 steps; the engine runs
128 replicates of the same workload in one ensemble.  Checks:
  - the mean C count agrees at every recorded time within 3 combined standard
    errors (+1 molecule for the discreteness of counts);
  - two-sample KS tests on the C counts at t = 5 and t = 10 do not reject
    (p > 0.001);
  - the effective forward rate constant measured from the first 2 time units,
    k = <C(2)> / (2 * A * B / V), agrees within 3 combined standard errors;
  - the steady-state forward rate constant, from the rate balance
    dC/dt = kf A B / V - kr C over t in [0.5, 10] (after the initial
    transient of the pair distribution, whose relaxation time is of order
    binding radius^2 / D, a fraction of a step):
        kf = (C(10) - C(0.5) + kr * integral C dt) / integral A B / V dt,
    per seed and per replicate, agrees within 3 combined standard errors.
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
SIDE, N, KF, KR, DT, STEPS, EVERY = 100.0, 10000, 0.05, 0.1, 0.01, 1000, 50
SEEDS = 32
NREP = 128

CONFIG = """dim 3
species A B C
difc A 1
difc B 1
difc C 0.5
boundaries 0 0 {L} r
boundaries 1 0 {L} r
boundaries 2 0 {L} r
time_start 0
time_stop {tstop}
time_step {dt}
random_seed {seed}
reaction fwd A + B -> C {kf}
reaction rev C -> A + B {kr}
mol {n} A u u u
mol {n} B u u u
output_files {out}
cmd N {every} molcount {out}
end_file
"""


def reference_runs():
    env = dict(os.environ, SMOLDYN_NO_PROMPT="1")
    out = []
    with tempfile.TemporaryDirectory() as d:
        procs = []
        for seed in range(1, SEEDS + 1):
            cfg = os.path.join(d, "c%d.txt" % seed)
            with open(cfg, "w") as f:
                f.write(CONFIG.format(L=SIDE, tstop=STEPS * DT, dt=DT, seed=seed, kf=KF, kr=KR, n=N,
                                      out="o%d.txt" % seed, every=EVERY))
            procs.append(subprocess.Popen([REF_EXE, "c%d.txt" % seed, "-qt"], cwd=d, stdout=subprocess.DEVNULL,
                                          stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, env=env))
        for p in procs:
            assert p.wait(timeout=900) == 0
        for seed in range(1, SEEDS + 1):
            rows = np.array([[float(x) for x in ln.split()] for ln in open(os.path.join(d, "o%d.txt" % seed))
                             if ln.strip()])
            out.append(rows)
    return out


def engine_runs():
    t = sb.Sim(3, (0, 0, 0), (SIDE, SIDE, SIDE))
    for nm, dc in (("A", 1.0), ("B", 1.0), ("C", 0.5)):
        t.add_species(nm, dc)
    for d in range(3):
        t.boundary(d, -1, "r")
    t.set_times(0, 1e6, DT)
    t.seed(2024)
    t.add_reaction("fwd", "A", "B", ["C"], KF)
    t.add_reaction("rev", "C", None, ["A", "B"], KR)
    e = sb.Ensemble(t, NREP)
    e.add_molecules("A", np.full(NREP, N))
    e.add_molecules("B", np.full(NREP, N))
    e.update()
    times, cs = [0.0], [e.counts(4)[:, 1:4].copy()]
    for k in range(STEPS // EVERY):
        e.run_steps(EVERY)
        times.append((k + 1) * EVERY * DT)
        cs.append(e.counts(4)[:, 1:4].copy())
    return np.array(times), np.array(cs).transpose(1, 0, 2)  # [rep, time, species A B C]


@pytest.fixture(scope="module")
def runs():
    if not os.path.exists(REF_EXE):
        pytest.skip("reference binary not built")
    ref = reference_runs()
    times, full = engine_runs()
    return ref, times, full[:, :, 2], full


def _steady_kf(t, a, b, c, t1=0.5, t2=10.0):
    """Forward rate constant from the rate balance over [t1, t2] (trapezoid
    rule over the recorded times)."""
    sel = (t >= t1 - 1e-9) & (t <= t2 + 1e-9)
    t, a, b, c = t[sel], a[sel].astype(float), b[sel].astype(float), c[sel].astype(float)
    expo = np.trapezoid(a * b / SIDE ** 3, t)
    return (c[-1] - c[0] + KR * np.trapezoid(c, t)) / expo


def _ref_at(ref, t):
    vals = []
    for rows in ref:
        k = np.argmin(np.abs(rows[:, 0] - t))
        assert abs(rows[k, 0] - t) < 1e-6
        vals.append(rows[k, 3])
    return np.array(vals)


def test_mean_trajectory_within_3_sigma(runs):
    ref, times, gpu, _ = runs
    worst = 0.0
    for k, t in enumerate(times):
        r = _ref_at(ref, t)
        g = gpu[:, k].astype(float)
        se = np.sqrt(r.var(ddof=1) / len(r) + g.var(ddof=1) / len(g))
        dev = abs(r.mean() - g.mean())
        assert dev <= 3 * se + 1, (t, r.mean(), g.mean(), se)
        worst = max(worst, dev / (se + 1e-12))
    print("worst deviation of the mean C trajectory: %.2f standard errors" % worst)


@pytest.mark.parametrize("t", [5.0, 10.0])
def test_ks_on_counts(runs, t):
    ref, times, gpu, _ = runs
    k = int(np.argmin(np.abs(times - t)))
    p = stats.ks_2samp(_ref_at(ref, t), gpu[:, k]).pvalue
    print("KS p-value of C counts at t=%g: %.3f" % (t, p))
    assert p > 1e-3


def test_effective_forward_rate(runs):
    ref, times, gpu, _ = runs
    t = 2.0
    k = int(np.argmin(np.abs(times - t)))
    scale = t * N * N / SIDE ** 3
    kr_ = _ref_at(ref, t) / scale
    kg = gpu[:, k] / scale
    se = np.sqrt(kr_.var(ddof=1) / len(kr_) + kg.var(ddof=1) / len(kg))
    print("effective kf: reference %.4f +- %.4f, engine %.4f +- %.4f" %
          (kr_.mean(), kr_.std(ddof=1) / np.sqrt(len(kr_)), kg.mean(), kg.std(ddof=1) / np.sqrt(len(kg))))
    assert abs(kr_.mean() - kg.mean()) <= 3 * se


def test_steady_state_forward_rate(runs):
    ref, times, _, full = runs
    kr_ = np.array([_steady_kf(rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3]) for rows in ref])
    kg = np.array([_steady_kf(times, full[k, :, 0], full[k, :, 1], full[k, :, 2]) for k in range(len(full))])
    se = np.sqrt(kr_.var(ddof=1) / len(kr_) + kg.var(ddof=1) / len(kg))
    print("steady-state kf: reference %.5f +- %.5f, engine %.5f +- %.5f (requested %.3f)" %
          (kr_.mean(), kr_.std(ddof=1) / np.sqrt(len(kr_)), kg.mean(), kg.std(ddof=1) / np.sqrt(len(kg)), KF))
    assert abs(kr_.mean() - kg.mean()) <= 3 * se

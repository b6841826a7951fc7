"""Batched ensembles: per-replicate parameters and dynamics.

- Per-replicate binding/unbinding radii from the device FP64 path equal the
  host path and the single-simulation derivation (1e-9 relative).
- Replicates sharing one parameter set reproduce the reference's ensemble
  mean of the remaining reactant count (reference binary, 16 seeds) within
  3 combined standard errors; replicates with other parameters in the same
  engine do not disturb them.
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


def template(side, kf, kr, wall="r", dt=0.01, seed=7):
    s = sb.Sim(3, (0, 0, 0), (side, side, side))
    for nm, d in (("A", 1.0), ("B", 1.0), ("C", 0.5)):
        s.add_species(nm, d)
    for d in range(3):
        s.boundary(d, -1, wall)
    s.set_times(0, 1e6, dt)
    s.seed(seed)
    s.add_reaction("fwd", "A", "B", ["C"], kf)
    if kr is not None:
        s.add_reaction("rev", "C", None, ["A", "B"], kr)
    return s


def test_per_replicate_radii_device_host_single():
    R = 64
    rng = np.random.default_rng(2)
    kf = 10 ** rng.uniform(-3, 0, R)
    kr = 10 ** rng.uniform(-3, 0, R)
    t = template(20.0, 0.05, 0.1)
    e = sb.Ensemble(t, R)
    e.set_rates("fwd", kf)
    e.set_rates("rev", kr)
    e.radius_mode(1)
    b_dev, u_dev = e.reaction_params("fwd")
    e.radius_mode(0)
    b_host, u_host = e.reaction_params("fwd")
    assert np.allclose(b_dev, b_host, rtol=1e-9, atol=0)
    assert np.allclose(u_dev, u_host, rtol=1e-9, atol=1e-300)
    for k in range(0, R, 9):
        single = template(20.0, kf[k], kr[k])
        b, u, _ = single.reaction_params("fwd")
        _, ur, _ = single.reaction_params("rev")
        assert abs(b - b_dev[k]) <= 1e-9 * b
        assert abs(ur - u_dev[k]) <= 1e-9 * max(ur, 1e-300)


def ref_config(path, side, n, kf, steps, dt, seed, out):
    with open(path, "w") as f:
        f.write("""dim 3
species A B C
difc A 1
difc B 1
difc C 0.5
boundaries 0 0 %.10g r
boundaries 1 0 %.10g r
boundaries 2 0 %.10g r
time_start 0
time_stop %g
time_step %g
random_seed %d
reaction fwd A + B -> C %g
mol %d A u u u
mol %d B u u u
output_files %s
cmd a molcount %s
end_file
""" % (side, side, side, steps * dt, dt, seed, kf, n, n, out, out))


def test_ensemble_matches_reference_ensemble():
    if not os.path.exists(REF_EXE):
        pytest.skip("reference binary not built")
    n, kf, dt, steps = 1000, 1.0, 0.01, 200
    side = (2 * n / 0.1) ** (1 / 3)
    ref = []
    env = dict(os.environ, SMOLDYN_NO_PROMPT="1")
    with tempfile.TemporaryDirectory() as d:
        for seed in range(1, 17):
            out = "o%d.txt" % seed
            ref_config(os.path.join(d, "c%d.txt" % seed), side, n, kf, steps, dt, seed, out)
            subprocess.check_call([REF_EXE, "c%d.txt" % seed, "-qt"], cwd=d, stdout=subprocess.DEVNULL,
                                  stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, env=env, timeout=300)
            rows = [ln.split() for ln in open(os.path.join(d, out)) if ln.strip()]
            ref.append(float(rows[-1][1]))
    ref = np.array(ref)
    # 192 replicates: 128 with the reference parameters, 64 with other boxes/rates
    R = 192
    t = template(side, kf, None, dt=dt)
    e = sb.Ensemble(t, R)
    rates = np.full(R, kf)
    rates[128:] = 0.2
    e.set_rates("fwd", rates)
    lo = np.zeros((R, 3))
    hi = np.full((R, 3), side)
    hi[128:] = side * 1.3
    e.set_boxes(lo, hi)
    e.add_molecules("A", np.full(R, n))
    e.add_molecules("B", np.full(R, n))
    e.update()
    e.run_steps(steps)
    c = e.counts(4)
    gpu = c[:128, 1].astype(float)
    assert (c[:, 1] == c[:, 2]).all()  # A and B consumed in pairs
    assert (c[:, 1] + c[:, 3] == n).all()  # A + C conserved per replicate
    se = np.sqrt(ref.var(ddof=1) / len(ref) + gpu.var(ddof=1) / len(gpu))
    assert abs(ref.mean() - gpu.mean()) < 3 * se + 1, (ref.mean(), gpu.mean(), se)
    # the slower replicates reacted less
    assert c[128:, 3].mean() < c[:128, 3].mean()

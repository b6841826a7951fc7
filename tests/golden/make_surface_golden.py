"""Generate tests/golden/surface_probs.npz from the reference engine itself.

For a set of seeded random surface configurations (adsorption, desorption,
flips and one- and two-way transmission rates between the solution, front and back
states of two species on one rectangle), runs oracle/_ref/ref_harness in its
"surfprobs" mode: the reference loads the configuration, runs its
surfupdateparams (smolsurface.c:3735-3800) and prints every surface action
and, for rate-based ones, the derived probabilities, cumulative
probabilities and reverse probabilities by destination state.
Stored: the configuration texts, the A lines (case, surface, species, state,
face, action) and the S lines (case, the same keys, then 18 values).
Usage: python tests/golden/make_surface_golden.py   (needs `make -C oracle ref`)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
NCASE = 48


def make_config(rng):
    dt = 10 ** rng.uniform(-4, -1)
    da, db = 10 ** rng.uniform(-1, 1, 2)
    lines = ["dim 3", "species A B", "difc A %.6g" % da, "difc B %.6g" % db,
             "difc A(front) %.6g" % (0.1 * da), "difc B(back) %.6g" % (0.2 * db),
             "time_start 0", "time_stop 1", "time_step %.6g" % dt]
    lines += ["boundaries %d 0 10 r" % d for d in range(3)]
    lines += ["random_seed 1", "start_surface s1", "panel rect +0 5 0 0 10 10 r1"]

    def k(lo, hi):
        return "-1" if rng.random() < 0.08 else "%.6g" % (10 ** rng.uniform(lo, hi))

    pool = [
        lambda: "rate A fsoln front %s" % k(-2, 2),
        lambda: "rate A front fsoln %s" % k(-1, 3),
        lambda: "rate A bsoln back %s" % k(-2, 2),
        lambda: "rate A back bsoln %s" % k(-1, 3),
        lambda: "rate A front back %s" % k(-1, 3),
        lambda: "rate A back front %s" % k(-1, 3),
        lambda: "rate B fsoln front %s" % k(-2, 2),
        lambda: "rate B front fsoln %s" % k(-1, 3),
        lambda: "rate B fsoln back %s" % k(-2, 2),
        lambda: "rate B back bsoln %s" % k(-1, 3),
        lambda: "rate B fsoln bsoln %s" % k(-2, 2),
        lambda: "rate A fsoln bsoln %s\nrate A bsoln fsoln %s" % (k(-2, 1), k(-2, 1)),
        lambda: "rate_internal A front fsoln %.4g" % rng.uniform(0, 1),
        lambda: "rate_internal B fsoln front %.4g" % rng.uniform(0, 1),
    ]
    pick = rng.choice(len(pool), size=rng.integers(2, 8), replace=False)
    lines += [pool[j]() for j in sorted(pick)]
    lines += ["end_surface", "end_file"]
    return "\n".join(lines) + "\n"


def run_case(text):
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(text)
        out = os.path.join(d, "o.txt")
        subprocess.run([HARNESS, d + "/", "c.txt", out, "surfprobs"], check=True, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL, env=dict(os.environ, SMOLDYN_NO_PROMPT="1"), timeout=120)
        acts, probs = [], []
        for ln in open(out):
            w = ln.split()
            if w[0] == "A":
                acts.append([int(x) for x in w[1:6]])
            elif w[0] == "S":
                probs.append([float(x) for x in w[1:]])
    return np.array(acts, dtype=np.int32), np.array(probs, dtype=np.float64).reshape(-1, 22)


def main():
    if not os.path.exists(HARNESS):
        sys.exit("build the reference harness first: make -C oracle ref")
    rng = np.random.default_rng(2024)
    configs, acts, probs = [], [], []
    for _ in range(NCASE):
        t = make_config(rng)
        a, p = run_case(t)
        configs.append(t)
        acts.append(a)
        probs.append(p)
    out = os.path.join(HERE, "surface_probs.npz")
    # one row per line, the case index first
    acts_all = np.concatenate([np.column_stack([np.full(len(a), c), a]) for c, a in enumerate(acts)])
    probs_all = np.concatenate([np.column_stack([np.full(len(p), c), p]) for c, p in enumerate(probs) if len(p)])
    np.savez_compressed(out, configs=np.array(configs), acts=acts_all.astype(np.int32), probs=probs_all)
    print("wrote", out, len(probs_all), "rate-based rules")


if __name__ == "__main__":
    main()

"""Whole reaction networks against reference ensembles (statistical parity).

Each case is one text configuration run through the reference binary
(oracle/_ref/smoldyn, 32 seeds in parallel, molcount every `every` steps) and
through this library's config reader as 32 single simulations (the plain
engine path, one replicate each, seeds 1..32).  Checks on every species:
  - the mean count agrees at every recorded time within 3 combined standard
    errors (+1 molecule for the discreteness of counts);
  - two-sample KS tests on the counts at the last time do not reject
    (p > 0.001).

Cases:
  probability     A + B -> C with reaction_probability 0.3: the binding
                  radius comes from bindingradiusprob's 1-D search
                  (rxnparam.c:612-636) and each in-radius pair reacts with
                  probability 0.3 (bireact, smolreact.c:3231);
  chi             A + B <-> C with reaction_chi 0.05 on the forward reaction
                  and unbinding ratio 1.5: radius and probability both from
                  the 2-D search (rxnparam.c:638-676);
  scaleup_reduced the scale-up network at its density (0.01 molecules per
                  unit volume) in a periodic cube of side 126 (2e4
                  molecules, 45% A, 45% B, 10% C): A + B -> C 0.05,
                  C -> A + B 0.1, 0 -> A 1e-4 per unit volume per unit time,
                  D = 1, 1, 0.5, dt = 0.01, 500 steps;
  surfaces_reduced the surfaces network at its density (0.5 per unit
                  volume) scaled to a cube of side 40 closed by reflective
                  panels: a reflective sphere of radius 16 at the centre, an
                  absorbing plane at x = 38, 32,000 molecules in thirds A/B/C
                  (D = 2, 1, 0.2), 60% inside the sphere (compartment_mol)
                  and 40% outside; A + B -> C 0.05, C -> 0 0.01; dt = 0.005,
                  400 steps.
"""
import ctypes as C
import os
import subprocess
import tempfile
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest
from scipy import stats

import smoldyn_b200 as sb
from tests import oracle_lib

pytestmark = pytest.mark.gpu

REF_EXE = os.path.join(oracle_lib.REF_DIR, "smoldyn")
SEEDS = 32

HEAD = """dim 3
species A B C
difc A {dA}
difc B {dB}
difc C {dC}
time_start 0
time_stop {tstop}
time_step {dt}
random_seed {seed}
"""

CASES = {
    "probability": dict(dA=1, dB=1, dC=0.5, dt=0.01, steps=400, every=40, body="""boundaries 0 0 40 r
boundaries 1 0 40 r
boundaries 2 0 40 r
reaction fwd A + B -> C 5
reaction_probability fwd 0.3
mol 3000 A u u u
mol 3000 B u u u
"""),
    "chi": dict(dA=1, dB=1, dC=0.5, dt=0.01, steps=400, every=40, body="""boundaries 0 0 40 r
boundaries 1 0 40 r
boundaries 2 0 40 r
reaction fwd A + B -> C 5
reaction rev C -> A + B 1
reaction_chi fwd 0.05
product_placement rev ratio 1.5
mol 3000 A u u u
mol 3000 B u u u
"""),
    "scaleup_reduced": dict(dA=1, dB=1, dC=0.5, dt=0.01, steps=500, every=50, body="""boundaries 0 0 125.99 p
boundaries 1 0 125.99 p
boundaries 2 0 125.99 p
reaction fwd A + B -> C 0.05
reaction rev C -> A + B 0.1
reaction birth 0 -> A 0.0001
mol 9000 A u u u
mol 9000 B u u u
mol 2000 C u u u
"""),
    "surfaces_reduced": dict(dA=2, dB=1, dC=0.2, dt=0.005, steps=400, every=40, body="""boundaries 0 0 40
boundaries 1 0 40
boundaries 2 0 40
start_surface walls
action both all reflect
panel rect +0 0 0 0 40 40
panel rect -0 40 0 0 40 40
panel rect +1 0 0 0 40 40
panel rect -1 0 40 0 40 40
panel rect +2 0 0 0 40 40
panel rect -2 0 0 40 40 40
end_surface
start_surface membrane
action both all reflect
panel sphere 20 20 20 16 30 30
end_surface
start_surface sink
action both all absorb
panel rect +0 38 0 0 40 40
end_surface
start_compartment inside
surface membrane
point 20 20 20
end_compartment
start_compartment outside
surface walls
surface membrane
point 2 2 2
point 37 37 37
end_compartment
reaction fwd A + B -> C 0.05
reaction decay C -> 0 0.01
compartment_mol 6400 A inside
compartment_mol 6400 B inside
compartment_mol 6400 C inside
compartment_mol 4267 A outside
compartment_mol 4267 B outside
compartment_mol 4267 C outside
"""),
}


def config(case, seed, out=None):
    c = CASES[case]
    txt = HEAD.format(tstop=c["steps"] * c["dt"], seed=seed, **c) + c["body"]
    if out:
        txt += "output_files %s\ncmd N %d molcount %s\n" % (out, c["every"], out)
    return txt + "end_file\n"


def reference_series(case):
    """[seed, time, species A B C] molcount series of the reference."""
    env = dict(os.environ, SMOLDYN_NO_PROMPT="1")
    with tempfile.TemporaryDirectory() as d:
        def one(seed):
            with open(os.path.join(d, "c%d.txt" % seed), "w") as f:
                f.write(config(case, seed, "o%d.txt" % seed))
            r = subprocess.run([REF_EXE, "c%d.txt" % seed, "-qt"], cwd=d, stdout=subprocess.DEVNULL,
                               stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, env=env, timeout=1800)
            assert r.returncode == 0
            rows = [[float(x) for x in ln.split()] for ln in open(os.path.join(d, "o%d.txt" % seed)) if ln.strip()]
            return np.array(rows)[:, 1:4]

        with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
            series = list(ex.map(one, range(1, SEEDS + 1)))
    n = min(len(s) for s in series)
    return np.stack([s[:n] for s in series])


def engine_series(case):
    """The same configuration through the C API, one simulation per seed,
    counts read at the reference's molcount times (t = 0, every, 2*every ...)."""
    lib = sb.load()
    c = CASES[case]
    out = []
    for seed in range(1, SEEDS + 1):
        with tempfile.TemporaryDirectory() as d:
            with open(os.path.join(d, "c.txt"), "w") as f:
                f.write(config(case, 1000 + seed))
            simp = C.c_void_p()
            assert lib.smolLoadSimFromFile((d + "/").encode(), b"c.txt", C.byref(simp), b"") == 0, sb.last_error()
        s = sb.Sim(ptr=simp.value)
        s.update()
        rows = [[s.count(nm) for nm in "ABC"]]
        for _ in range(c["steps"] // c["every"]):
            s.run_steps(c["every"])
            rows.append([s.count(nm) for nm in "ABC"])
        s.close()
        out.append(np.array(rows, dtype=float))
    return np.stack(out)


@pytest.mark.parametrize("case", sorted(CASES))
def test_network_matches_reference(case):
    if not os.path.exists(REF_EXE):
        pytest.skip("reference binary not built")
    ref = reference_series(case)
    eng = engine_series(case)
    nt = min(ref.shape[1], eng.shape[1])
    assert nt >= CASES[case]["steps"] // CASES[case]["every"]
    for k, nm in enumerate("ABC"):
        r, g = ref[:, :nt, k], eng[:, :nt, k]
        se = np.sqrt(r.var(axis=0, ddof=1) / len(r) + g.var(axis=0, ddof=1) / len(g))
        dev = np.abs(r.mean(0) - g.mean(0))
        print("%s %s: reference %s engine %s" % (case, nm, np.round(r.mean(0)[::2], 1), np.round(g.mean(0)[::2], 1)))
        bad = np.nonzero(dev > 3 * se + 1)[0]
        assert not len(bad), (case, nm, bad, r.mean(0)[bad], g.mean(0)[bad], se[bad])
        if r[:, -1].std() > 0 or g[:, -1].std() > 0:
            p = stats.ks_2samp(r[:, -1], g[:, -1]).pvalue
            assert p > 1e-3, (case, nm, p)

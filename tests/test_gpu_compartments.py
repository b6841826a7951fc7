"""Compartment-restricted reactions on the GPU against the reference binary.

A cube of side 20 closed by reflective rectangle panels holds a transparent
sphere of radius 6 at its centre; the compartment "inside" is bounded by the
sphere with an interior point at the centre (smolcomparts.c:119
posincompart).  Each case runs the same configuration through the reference
(oracle/_ref/smoldyn) and through this library's config reader, 8 seeds each,
and compares the mean end counts within 4 combined standard errors (+2 for
the discreteness of counts):
- first order: A -> B only inside;
- competing first-order reactions, the first restricted: A -> B inside,
  A -> C anywhere (a molecule outside whose coin picked the first reaction
  passes the decision on, smolreact.c:3040-3050);
- zeroth order: births inside at rate x compartment volume; with D = 0 every
  born molecule must also sit inside the sphere;
- second order: A + B -> C only when both reactants are inside.
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
SEEDS = 8

HEAD = """dim 3
species A B C
difc A {da}
difc B 1
difc C 1
boundaries 0 0 20
boundaries 1 0 20
boundaries 2 0 20
time_start 0
time_stop 2
time_step 0.01
random_seed {seed}
start_surface walls
action both all reflect
panel rect +0 0 0 0 20 20
panel rect -0 20 0 0 20 20
panel rect +1 0 0 0 20 20
panel rect -1 0 20 0 20 20
panel rect +2 0 0 0 20 20
panel rect -2 0 0 20 20 20
end_surface
start_surface ball
action both all transmit
panel sph 10 10 10 6 20 20
end_surface
start_compartment inside
surface ball
point 10 10 10
end_compartment
"""

CASES = {
    "uni": (1, "mol 4000 A u u u\nreaction cmpt=inside conv A -> B 0.5\n"),
    "uni_competing": (1, "mol 4000 A u u u\nreaction cmpt=inside toB A -> B 1\nreaction toC A -> C 0.5\n"),
    "births": (0, "reaction cmpt=inside birth 0 -> A 1\n"),
    "bi": (1, "mol 4000 A u u u\nmol 4000 B u u u\nreaction_cmpt inside fwd A + B -> C 20\n"),
}


def config(case, seed):
    da, body = CASES[case]
    return (HEAD.format(da=da, seed=seed) + body +
            "output_files out.txt\ncmd a molcount out.txt\nend_file\n")


def reference_counts(case):
    env = dict(os.environ, SMOLDYN_NO_PROMPT="1")
    rows = []
    with tempfile.TemporaryDirectory() as d:
        procs = []
        for seed in range(1, SEEDS + 1):
            sd = os.path.join(d, str(seed))
            os.mkdir(sd)
            with open(os.path.join(sd, "c.txt"), "w") as f:
                f.write(config(case, seed))
            procs.append(subprocess.Popen([REF_EXE, "c.txt", "-qt"], cwd=sd, stdout=subprocess.DEVNULL,
                                          stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, env=env))
        for p in procs:
            assert p.wait(timeout=900) == 0
        for seed in range(1, SEEDS + 1):
            last = [ln.split() for ln in open(os.path.join(d, str(seed), "out.txt")) if ln.strip()][-1]
            rows.append([float(x) for x in last[1:4]])
    return np.array(rows)


def engine_run(case, seed):
    lib = sb.load()
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(config(case, 100 + seed))
        simp = C.c_void_p()
        assert lib.smolLoadSimFromFile((d + "/").encode(), b"c.txt", C.byref(simp), b"") == 0, sb.last_error()
    s = sb.Sim(ptr=simp.value)
    s.run()
    return s


def engine_counts(case):
    rows = []
    for seed in range(SEEDS):
        s = engine_run(case, seed)
        rows.append(s.output_data("out.txt")[-1][1:4])
        s.close()
    return np.array(rows)


@pytest.mark.parametrize("case", sorted(CASES))
def test_restricted_reaction_matches_reference(case):
    if not os.path.exists(REF_EXE):
        pytest.skip("reference binary not built")
    ref, eng = reference_counts(case), engine_counts(case)
    moved = False
    for k, nm in enumerate("ABC"):
        r, g = ref[:, k], eng[:, k]
        if r.max() == 0 and g.max() == 0:
            continue
        se = np.sqrt(r.var(ddof=1) / len(r) + g.var(ddof=1) / len(g))
        print("%s %s: reference %.1f +- %.1f, engine %.1f +- %.1f" %
              (case, nm, r.mean(), r.std(ddof=1) / np.sqrt(len(r)), g.mean(), g.std(ddof=1) / np.sqrt(len(g))))
        assert abs(r.mean() - g.mean()) <= 4 * se + 2, (case, nm, r.mean(), g.mean(), se)
        moved = True
    assert moved


def test_births_stay_inside_the_compartment():
    s = engine_run("births", 0)
    pos, sp, _ = s.molecules()
    r = np.linalg.norm(pos - 10.0, axis=1)
    expect = 1.0 * 4 / 3 * np.pi * 6 ** 3 * 2.0
    assert abs(len(pos) - expect) < 5 * np.sqrt(expect), (len(pos), expect)
    assert r.max() <= 6.0 + 1e-4, r.max()
    s.close()


def test_ensemble_keeps_the_compartment():
    """An ensemble built from the template keeps its compartments: A -> B
    inside the sphere only, 16 replicates of 4000 molecules each, against the
    single simulations' mean."""
    ref = engine_counts("uni")
    lib = sb.load()
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(config("uni", 1).replace("mol 4000 A u u u\n", ""))
        simp = C.c_void_p()
        assert lib.smolLoadSimFromFile((d + "/").encode(), b"c.txt", C.byref(simp), b"") == 0, sb.last_error()
    t = sb.Sim(ptr=simp.value)
    e = sb.Ensemble(t, 16)
    e.add_molecules("A", np.full(16, 4000))
    e.update()
    e.run_steps(200)
    b = e.counts(4)[:, 2].astype(float)
    r = ref[:, 1]
    se = np.sqrt(r.var(ddof=1) / len(r) + b.var(ddof=1) / len(b))
    assert abs(b.mean() - r.mean()) <= 4 * se + 2, (b.mean(), r.mean(), se)
    assert b.mean() < 0.2 * 4000  # restricted: far fewer than A -> B everywhere (about 2/3 of 4000)


def test_molcountincmpt_counts_molecules_inside():
    """molcountincmpt (smolcmd.c:1054): per-species counts inside the
    compartment equal a host count of the downloaded positions inside the
    sphere, and agree with the reference's own molcountincmpt output."""
    text = (HEAD.format(da=1, seed=3) + "mol 4000 A u u u\nmol 2000 B u u u\n"
            "output_files cnt.txt\ncmd a molcountincmpt inside cnt.txt\nend_file\n")
    lib = sb.load()
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(text)
        simp = C.c_void_p()
        assert lib.smolLoadSimFromFile((d + "/").encode(), b"c.txt", C.byref(simp), b"") == 0, sb.last_error()
    s = sb.Sim(ptr=simp.value)
    s.run()
    row = s.output_data("cnt.txt")[-1]
    pos, sp, _ = s.molecules()
    inside = np.linalg.norm(pos - 10.0, axis=1) < 6.0
    host = [int(np.count_nonzero(inside & (sp == k))) for k in (1, 2, 3)]
    assert [int(v) for v in row[1:4]] == host, (row, host)
    if not os.path.exists(REF_EXE):
        return
    env = dict(os.environ, SMOLDYN_NO_PROMPT="1")
    ref = []
    with tempfile.TemporaryDirectory() as d:
        for seed in range(1, 5):
            with open(os.path.join(d, "c.txt"), "w") as f:
                f.write(text.replace("random_seed 3", "random_seed %d" % seed))
            subprocess.run([REF_EXE, "c.txt", "-qt"], cwd=d, check=True, stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, env=env, timeout=600)
            last = [ln.replace(",", " ").split() for ln in open(os.path.join(d, "cnt.txt")) if ln.strip()][-1]
            ref.append([float(x) for x in last[1:4]])
    ref = np.array(ref).mean(0)
    expect = np.array([4000, 2000, 0]) * (4 / 3 * np.pi * 216) / 8000
    assert np.all(np.abs(ref - expect) <= 5 * np.sqrt(expect / 4) + 1), (ref, expect)
    assert np.all(np.abs(np.array(host) - expect) <= 5 * np.sqrt(expect) + 1), (host, expect)

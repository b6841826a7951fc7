"""Triangle, cylinder, hemisphere and disk panels (smolsurface.c:2432
surfaddpanel, :4000 lineXpanel) on the GPU.

1. Absorption against the reference: a cube of side 20 closed by reflective
   rectangle panels (walls are transparent once surfaces exist) holds
   molecules of D = 1; one absorbing panel of the shape under test sits in
   it.  The same configuration runs in the reference binary (8 seeds, 4000
   molecules each) and in the engine (32000 molecules); the surviving
   fractions agree within 4 combined binomial standard errors.  One case has
   a one-sided cylinder (outside reflects, inside absorbs), which checks the
   face conventions (front outside for a positive radius).
2. Containment: closed shapes built from the new panels (a cylinder with two
   disk caps, a capsule of a cylinder and two hemispheres, a tetrahedron of
   four triangles), all reflective, keep every molecule that starts inside.
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
SEEDS, NREF = 8, 4000

HEAD = """dim 3
species A
difc A 1
boundaries 0 0 20
boundaries 1 0 20
boundaries 2 0 20
time_start 0
time_stop {tstop}
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
"""

ABSORB = {
    "disk": "action both all absorb\npanel disk 10 10 10 5 1 0.5 0 20",
    "tri": "action both all absorb\npanel tri 4 4 10 16 5 9 9 16 11",
    "cyl": "action both all absorb\npanel cyl 10 10 4 10 12 16 4 20 20",
    "hemi": "action both all absorb\npanel hemi 10 10 10 5 0 0.6 0.8 20 20",
    "cyl_inside_absorbs": "action front all reflect\naction back all absorb\npanel cyl 4 10 10 16 10 10 3 20 20",
}


def absorb_config(case, seed, nmol):
    return (HEAD.format(tstop=2.0, seed=seed) + "start_surface sink\n" + ABSORB[case] + "\nend_surface\n" +
            "mol %d A u u u\noutput_files out.txt\ncmd a molcount out.txt\nend_file\n" % nmol)


def reference_fraction(case):
    env = dict(os.environ, SMOLDYN_NO_PROMPT="1")
    left = []
    with tempfile.TemporaryDirectory() as d:
        procs = []
        for seed in range(1, SEEDS + 1):
            sd = os.path.join(d, str(seed))
            os.mkdir(sd)
            with open(os.path.join(sd, "c.txt"), "w") as f:
                f.write(absorb_config(case, seed, NREF))
            procs.append(subprocess.Popen([REF_EXE, "c.txt", "-qt"], cwd=sd, stdout=subprocess.DEVNULL,
                                          stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, env=env))
        for p in procs:
            assert p.wait(timeout=900) == 0
        for seed in range(1, SEEDS + 1):
            rows = [ln.split() for ln in open(os.path.join(d, str(seed), "out.txt")) if ln.strip()]
            left.append(float(rows[-1][1]))
    return sum(left) / (SEEDS * NREF)


def load(text):
    lib = sb.load()
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "c.txt"), "w") as f:
            f.write(text)
        simp = C.c_void_p()
        assert lib.smolLoadSimFromFile((d + "/").encode(), b"c.txt", C.byref(simp), b"") == 0, sb.last_error()
    return sb.Sim(ptr=simp.value)


@pytest.mark.parametrize("case", sorted(ABSORB))
def test_absorbing_panel_matches_reference(case):
    if not os.path.exists(REF_EXE):
        pytest.skip("reference binary not built")
    n = SEEDS * NREF
    s = load(absorb_config(case, 5, n))
    s.run()
    fe = s.output_data("out.txt")[-1][1] / n
    fr = reference_fraction(case)
    se = np.sqrt(fr * (1 - fr) * (1.0 / n + 1.0 / n))
    print("%s: reference %.4f engine %.4f (se %.4f)" % (case, fr, fe, se))
    assert 0.02 < 1 - fr < 0.98, "the case should absorb a fair part of the molecules"
    assert abs(fe - fr) <= 4 * se + 0.002, (case, fe, fr, se)


def closed_config(body):
    return HEAD.format(tstop=100.0, seed=3) + "start_surface shell\naction both all reflect\n" + body + \
        "\nend_surface\nend_file\n"


def run_inside(text, pos, steps=300):
    s = load(text)
    s.set_molecules(pos, np.ones(len(pos), dtype=np.int32))
    s.run_steps(steps)
    p, _, _ = s.molecules()
    assert len(p) == len(pos)
    return p


def test_cylinder_with_disk_caps_contains():
    rng = np.random.default_rng(1)
    n = 20000
    r = 5 * np.sqrt(rng.random(n)) * 0.999
    th = rng.uniform(0, 2 * np.pi, n)
    pos = np.stack([10 + r * np.cos(th), 10 + r * np.sin(th), rng.uniform(2.01, 17.99, n)], axis=1)
    p = run_inside(closed_config("panel cyl 10 10 2 10 10 18 5 20 20\npanel disk 10 10 2 5 0 0 1 20\n"
                                 "panel disk 10 10 18 5 0 0 -1 20"), pos)
    rad = np.hypot(p[:, 0] - 10, p[:, 1] - 10)
    assert rad.max() <= 5 + 1e-5 and p[:, 2].min() >= 2 - 1e-5 and p[:, 2].max() <= 18 + 1e-5


def test_capsule_contains():
    rng = np.random.default_rng(2)
    n = 20000
    r = 4 * np.sqrt(rng.random(n)) * 0.999
    th = rng.uniform(0, 2 * np.pi, n)
    pos = np.stack([10 + r * np.cos(th), 10 + r * np.sin(th), rng.uniform(5.01, 14.99, n)], axis=1)
    body = ("panel cyl 10 10 5 10 10 15 4 20 20\n"
            "panel hemi 10 10 15 4 0 0 -1 20 20\n"   # open side down, into the cylinder
            "panel hemi 10 10 5 4 0 0 1 20 20")
    p = run_inside(closed_config(body), pos)
    rad = np.hypot(p[:, 0] - 10, p[:, 1] - 10)
    z = p[:, 2]
    top = np.linalg.norm(p - [10, 10, 15], axis=1)
    bot = np.linalg.norm(p - [10, 10, 5], axis=1)
    inside = ((z >= 5 - 1e-5) & (z <= 15 + 1e-5) & (rad <= 4 + 1e-5)) | (top <= 4 + 1e-5) | (bot <= 4 + 1e-5)
    assert inside.all(), np.count_nonzero(~inside)


def test_tetrahedron_contains():
    v = np.array([[4, 4, 4], [16, 4, 4], [10, 16, 4], [10, 10, 16]], dtype=float)
    faces = [(0, 2, 1), (0, 1, 3), (1, 2, 3), (2, 0, 3)]  # right-hand normals point outward
    body = "\n".join("panel tri " + " ".join("%g" % x for k in f for x in v[k]) for f in faces)
    rng = np.random.default_rng(3)
    w = rng.dirichlet(np.ones(4), size=20000) * 0.998 + 0.0005
    pos = w @ v
    p = run_inside(closed_config(body), pos)
    # barycentric coordinates of the end positions
    T = np.column_stack([v[1] - v[0], v[2] - v[0], v[3] - v[0]])
    lam = np.linalg.solve(T, (p - v[0]).T).T
    bary = np.column_stack([1 - lam.sum(1), lam])
    assert bary.min() >= -1e-6, bary.min()


@pytest.mark.parametrize("name", ["onestep_panels", "onestep_panels_actions"])
def test_step_matches_reference_recording(name):
    """One step recorded from the reference (tests/golden/<name>.npz, made by
    make_golden.py with oracle/ref_harness): a cube closed by reflective
    rectangles with a tilted triangle, a cylinder, a hemisphere and a disk
    inside; all reflective, or with mixed actions (triangle front absorbs,
    back reflects; cylinder transmits; hemisphere absorbs).  The reference's
    start state and displacements go in through the injection mode; the same
    molecules must survive, each where the reference put it after its surface
    interactions (checksurfaces, smolsurface.c:5114), to 2e-5 of the side
    (FP32 box-local storage and the surface margin)."""
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name + ".npz"))
    s = load(str(g["config"]))
    s.set_molecules(g["pos0"], g["sp0"], g["serno0"])
    force = np.full((len(g["serno0"]), 1), -1.0)
    s.inject(g["serno0"], np.concatenate([g["disp"], force], axis=1))
    s.run_steps(1)
    pos, sp, sn = s.molecules()
    assert sorted(sn.tolist()) == sorted(g["serno1"].tolist())  # the same molecules absorbed
    ref = {int(k): i for i, k in enumerate(g["serno1"].tolist())}
    idx = np.array([ref[int(k)] for k in sn.tolist()])
    dev = np.linalg.norm(pos - g["pos1"][idx], axis=1)
    moved = g["pos0"] + g["disp"]
    i0 = {int(k): i for i, k in enumerate(g["serno0"].tolist())}
    hit = np.linalg.norm(moved[[i0[int(k)] for k in sn.tolist()]] - g["pos1"][idx], axis=1) > 1e-9
    print("%s: absorbed %d, reflected %d, max deviation %.3g (reflected) %.3g (others)" %
          (name, len(g["serno0"]) - len(sn), hit.sum(), dev[hit].max() if hit.any() else 0, dev[~hit].max()))
    assert hit.sum() > 100
    assert dev.max() <= 2e-5 * float(g["L"]), dev.max()

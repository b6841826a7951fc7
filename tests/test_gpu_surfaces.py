"""Surface parity tests (sphere and rectangle panels) on the GPU.

The same text configuration is run by the engine (through the libsmoldyn C API
config reader) and by the reference Smoldyn binary compiled from the
reference's sources (oracle/_ref/smoldyn, an ensemble of seeds); the
surviving-molecule counts must agree within 3 combined standard deviations.
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


def absorbing_plane_config(path, seed, nmol=5000, steps=400, dt=0.005, out="out.txt"):
    # walls are transparent once surfaces exist (smolwall.c:328), so the box
    # is closed by reflective rectangle panels; the plane x=15 absorbs
    with open(path, "w") as f:
        f.write("""dim 3
species A
difc A 1
boundaries 0 0 20
boundaries 1 0 20
boundaries 2 0 20
time_start 0
time_stop %g
time_step %g
random_seed %d
start_surface walls
action both all reflect
panel rect +0 0 0 0 20 20
panel rect -0 20 0 0 20 20
panel rect +1 0 0 0 20 20
panel rect -1 0 20 0 20 20
panel rect +2 0 0 0 20 20
panel rect -2 0 0 20 20 20
end_surface
start_surface sink
action both all absorb
panel rect +0 15 0 0 20 20
end_surface
mol %d A 0-15 u u
output_files %s
cmd a molcount %s
end_file
""" % (steps * dt, dt, seed, nmol, out, out))


def run_reference(cfg_dir, cfg_name, out="out.txt"):
    path = os.path.join(cfg_dir, out)
    if os.path.exists(path):
        os.remove(path)
    env = dict(os.environ, SMOLDYN_NO_PROMPT="1")
    subprocess.check_call([REF_EXE, cfg_name, "-qt"], cwd=cfg_dir, stdout=subprocess.DEVNULL,
                          stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, timeout=300, env=env)
    with open(path) as f:
        rows = [ln.split() for ln in f if ln.strip()]
    return float(rows[-1][1])


def run_engine(cfg_dir, cfg_name, out="out.txt"):
    import ctypes as C
    lib = sb.load()
    simp = C.c_void_p()
    assert lib.smolLoadSimFromFile(cfg_dir.encode(), cfg_name.encode(), C.byref(simp), b"") == 0, sb.last_error()
    s = sb.Sim(ptr=simp.value)
    s.run()
    data = s.output_data(out)
    return float(data[-1][1]), s


def test_absorbing_plane_matches_reference():
    if not os.path.exists(REF_EXE):
        pytest.skip("reference binary not built")
    from concurrent.futures import ThreadPoolExecutor
    seeds = range(1, 33)  # 32 seeds each
    ref, eng = [], []
    with tempfile.TemporaryDirectory() as d:
        for seed in seeds:
            absorbing_plane_config(os.path.join(d, "c%d.txt" % seed), seed, out="out%d.txt" % seed)
        with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
            ref = list(ex.map(lambda k: run_reference(d, "c%d.txt" % k, "out%d.txt" % k), seeds))
        for seed in seeds:
            n, s = run_engine(d, "c%d.txt" % seed, "out%d.txt" % seed)
            eng.append(n)
            s.close()
    ref, eng = np.array(ref), np.array(eng)
    se = np.sqrt(ref.var(ddof=1) / len(ref) + eng.var(ddof=1) / len(eng))
    assert 3000 < ref.mean() < 4900, ref.mean()
    assert abs(ref.mean() - eng.mean()) < 3 * se + 2, (ref.mean(), eng.mean(), se)


def test_reflective_sphere_keeps_inside_and_outside_apart():
    L, R = 40.0, 10.0
    s = sb.Sim(3, (0, 0, 0), (L, L, L))
    s.add_species("A", 1.0)
    s.set_times(0, 100, 0.01)
    s.seed(3)
    lib = s.lib
    assert lib.smolAddSurface(s.ptr, b"membrane") == 0
    assert lib.smolSetSurfaceAction(s.ptr, b"membrane", sb.PFboth, b"all", sb.MSsoln, sb.SAreflect, None) == 0
    params = np.array([20.0, 20.0, 20.0, R, 20, 20], dtype=np.float64)
    assert lib.smolAddPanel(s.ptr, b"membrane", sb.PSsph, None, None, sb.dptr(params)) == 0
    assert lib.smolAddSurface(s.ptr, b"box") == 0
    assert lib.smolSetSurfaceAction(s.ptr, b"box", sb.PFboth, b"all", sb.MSsoln, sb.SAreflect, None) == 0
    for ax, sign, c in ((0, "+", 0), (0, "-", L), (1, "+", 0), (1, "-", L), (2, "+", 0), (2, "-", L)):
        corner = [0.0, 0.0, 0.0]
        corner[ax] = c
        pr = np.array(corner + [L, L], dtype=np.float64)
        assert lib.smolAddPanel(s.ptr, b"box", sb.PSrect, None, ("%s%d" % (sign, ax)).encode(), sb.dptr(pr)) == 0
    rng = np.random.default_rng(0)
    # 3000 inside the sphere, 3000 outside it
    pin = []
    while len(pin) < 3000:
        q = rng.uniform(20 - R, 20 + R, 3)
        if np.linalg.norm(q - 20) < R - 0.01:
            pin.append(q)
    pout = []
    while len(pout) < 3000:
        q = rng.uniform(0.01, L - 0.01, 3)
        if np.linalg.norm(q - 20) > R + 0.01:
            pout.append(q)
    pos = np.array(pin + pout)
    sp = np.ones(len(pos), dtype=np.int32)
    sn = np.arange(1, len(pos) + 1, dtype=np.uint64)
    s.set_molecules(pos, sp, sn)
    s.run_steps(800)
    p, _, serno = s.molecules()
    assert len(serno) == 6000
    r = np.linalg.norm(p - 20, axis=1)
    inside0 = serno <= 3000
    assert (r[inside0] < R).all(), r[inside0].max()
    assert (r[~inside0] > R).all(), r[~inside0].min()
    assert p.min() >= 0 and p.max() <= L
    # molecules did move (a reflected walk, not a frozen one)
    assert np.abs(p[:3000] - pos[:3000]).mean() > 1.0

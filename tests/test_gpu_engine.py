"""GPU engine parity and behaviour tests (run on a B200 through the C ABI).

Deterministic parity: one time step with injected displacements and injected
first-order decisions, compared with the oracle's restatement of the
reference step (oracle/engine_oracle.c) on the same inputs: survivor
positions to 1e-5 of the box size (the engine stores FP32 box-local
coordinates), identical sets of molecules consumed by second-order reactions
away from binding-radius ties, identical product multisets.
"""
import numpy as np
import pytest

import smoldyn_b200 as sb
from tests import gpu_cases as gc
from tests import oracle_lib

pytestmark = pytest.mark.gpu


def _one_step_parity(n, L, wall, seed, rev_placement=None, frac=(0.4, 0.4, 0.2), uni_frac=0.1, kf=20.0,
                     molperbox=None):
    rng = np.random.default_rng(seed)
    difc = (1.0, 1.0, 0.5)
    dt = 0.01
    s = gc.make_sim(L=L, wall=wall, kf=kf, difc=difc, dt=dt, rev_placement=rev_placement, molperbox=molperbox)
    pos, sp, serno = gc.random_state(n, L, rng, frac)
    s.set_molecules(pos, sp, serno)
    bind, unb, _ = s.reaction_params("fwd")
    _, unb_rev, _ = s.reaction_params("rev")
    steps = np.sqrt(2 * np.asarray(difc)[sp - 1] * dt)
    disp = rng.normal(size=(n, 3)) * steps[:, None]
    force = np.where((sp == 3) & (rng.uniform(size=n) < uni_frac), 0, -1).astype(np.int32)
    disp4 = np.concatenate([disp, force[:, None].astype(np.float64)], axis=1)
    s.inject(serno, disp4)
    s.run_steps(1)
    gpos, gsp, gsn = s.molecules()
    # oracle
    dA, dB = difc[0], difc[1]
    prdpos = (0.0, 0.0)
    if unb_rev > 0:
        prdpos = (unb_rev * dA / (dA + dB), -unb_rev * dB / (dA + dB))
    net = gc.oracle_net(s, L, wall, difc, bind * bind, prdpos)
    o = oracle_lib.ora_step(net, pos, sp, serno, disp, force)
    return s, dict(pos=pos, sp=sp, serno=serno, disp=disp, bind=bind), (gpos, gsp, gsn), o


def _compare(inp, g, o, L, wall):
    gpos, gsp, gsn = g
    periodic = wall == "p"
    moved = gc.apply_walls_np(inp["pos"] + inp["disp"], L, wall)
    ties = gc.near_threshold(moved, inp["sp"], inp["bind"] ** 2, L, periodic)
    alive = o["fate"] != 2
    amb = gc.ambiguous_set(moved, inp["sp"], inp["bind"] ** 2, L, periodic, alive)
    tie_sn = {int(inp["serno"][i]) for i in ties | amb}
    # survivors: molecules with original serial numbers
    orig = gsn < (1 << 41)
    g_surv = dict(zip(gsn[orig].tolist(), range(int(orig.sum()))))
    gp = gpos[orig]
    o_surv = o["serno"][o["parent"] == 0]
    o_pos = o["pos"][o["parent"] == 0]
    o_set = set(o_surv.tolist())
    g_set = set(g_surv.keys())
    diff = (o_set ^ g_set) - tie_sn
    assert not diff, (len(diff), sorted(diff)[:10])
    common = sorted(o_set & g_set)
    oi = {int(k): i for i, k in enumerate(o_surv.tolist())}
    a = np.array([o_pos[oi[k]] for k in common])
    b = np.array([gp[g_surv[k]] for k in common])
    d = gc.min_image(a - b, L, periodic)
    assert np.abs(d).max() <= 1e-5 * L, np.abs(d).max()
    # products: same count per species (ties excepted), same positions as a multiset
    g_prod = gpos[~orig]
    g_psp = gsp[~orig]
    o_prod = o["pos"][o["parent"] != 0]
    o_psp = o["sp"][o["parent"] != 0]
    if not tie_sn:
        for spc in (1, 2, 3):
            assert (g_psp == spc).sum() == (o_psp == spc).sum(), spc
        for spc in (1, 2, 3):
            A = o_prod[o_psp == spc]
            B = g_prod[g_psp == spc]
            for x in A:
                dd = np.abs(gc.min_image(B - x, L, periodic)).max(1)
                assert dd.min() <= 1e-4 * L
    return len(common)


@pytest.mark.parametrize("wall", ["r", "p"])
def test_deterministic_step_matches_oracle(wall):
    L = 20.0
    s, inp, g, o = _one_step_parity(4000, L, wall, seed=11, rev_placement=(sb.RPirrev, 0.0))
    ncommon = _compare(inp, g, o, L, wall)
    assert ncommon > 2000
    ev = s.events()
    assert ev[3] > 0  # some second-order events happened
    assert ev[2] > 0  # and first-order ones


def test_deterministic_step_small_boxes_and_long_steps():
    # molperbox 0.5: boxes barely above the binding radius; large displacements
    # cross several boxes and reflect off walls
    L = 6.0
    s, inp, g, o = _one_step_parity(1500, L, "r", seed=3, rev_placement=(sb.RPirrev, 0.0), molperbox=0.5)
    _compare(inp, g, o, L, "r")


def test_deterministic_products_with_unbinding_radius():
    """C -> A + B with a fixed unbinding radius: products land at distance
    sigma_u apart, split by D (smolreact.c:1545-1548); orientation is random."""
    L = 20.0
    s, inp, g, o = _one_step_parity(2000, L, "p", seed=8, rev_placement=(sb.RPunbindrad, 0.5), frac=(0.0, 0.0, 1.0),
                                    uni_frac=0.3)
    gpos, gsp, gsn = g
    prod = gsn >= (1 << 41)
    nA = int(((gsp == 1) & prod).sum())
    nB = int(((gsp == 2) & prod).sum())
    nfired = int((o["fate"] == 2).sum())
    assert nA == nfired and nB == nfired and nfired > 400
    # every A product has a B product at distance 0.5 (pairs share the rotation)
    A = gpos[(gsp == 1) & prod]
    B = gpos[(gsp == 2) & prod]
    for x in A[:200]:
        d = np.sqrt((gc.min_image(B - x, L, True) ** 2).sum(1))
        assert np.abs(d - 0.5).min() < 1e-4


def test_counts_conserved_and_positions_inside_reflective_box():
    s = gc.make_sim(L=10.0, wall="r", kf=0.0, kr=0.0)
    s.add_molecules("A", 3000)
    s.add_molecules("B", 2000)
    s.update()
    s.run_steps(200)
    pos, sp, sn = s.molecules()
    assert len(sp) == 5000 and s.count("A") == 3000 and s.count("B") == 2000
    assert pos.min() >= 0.0 and pos.max() <= 10.0


def test_free_diffusion_msd():
    """Mean squared displacement of free diffusion = 6 D t within 3 sigma."""
    L = 1000.0
    s = sb.Sim(3, (0, 0, 0), (L, L, L))
    s.add_species("A", 1.0)
    s.set_times(0, 100, 0.01)
    s.seed(99)
    for d in range(3):
        s.boundary(d, -1, "r")
    n = 20000
    s.add_molecules("A", n, (450, 450, 450), (550, 550, 550))
    s.update()
    p0, _, sn0 = s.molecules()
    s.run_steps(100)
    p1, _, sn1 = s.molecules()
    assert (sn0 == sn1).all()
    r2 = ((p1 - p0) ** 2).sum(1)
    t = 1.0
    expect = 6 * 1.0 * t
    sd = np.sqrt(24) * 1.0 * t / np.sqrt(n)
    assert abs(r2.mean() - expect) < 3 * sd + 0.01 * expect, (r2.mean(), expect)
    # per-axis displacement distribution is Gaussian with variance 2Dt
    dx = (p1 - p0)[:, 0]
    assert abs(dx.var() - 2.0) < 0.05


def test_runs_are_reproducible():
    out = []
    for _ in range(2):
        s = gc.make_sim(L=15.0, wall="p", kf=20.0, kr=5.0)
        s.add_molecules("A", 3000)
        s.add_molecules("B", 3000)
        s.run_steps(50)
        out.append(s.molecules())
    assert len(out[0][1]) == len(out[1][1])
    assert (out[0][2] == out[1][2]).all()
    assert np.abs(out[0][0] - out[1][0]).max() == 0.0


def test_device_radius_solver_matches_reference():
    ref = oracle_lib.reference_rxnparam()
    if ref is None:
        pytest.skip("reference rxnparam not compiled")
    rng = np.random.default_rng(4)
    n = 2000
    rate = 10 ** rng.uniform(-4, 2, n)
    difc = 10 ** rng.uniform(-2, 1, n)
    dt = 0.01
    b = np.where(rng.uniform(size=n) < 0.5, -1.0, rng.uniform(1.1, 10, n))
    out = sb.solve_radii_device(0, rate, dt, difc, b, rel=1)
    exp = np.array([ref.bindingradius(rate[k], dt, difc[k], b[k], 1) for k in range(n)])
    rel = np.abs(out - exp) / np.abs(exp)
    assert rel.max() < 1e-9, rel.max()
    pg = rng.uniform(0.05, 0.5, n)
    uo = sb.solve_radii_device(1, pg, dt, difc, exp)
    ue = np.array([ref.unbindingradius(pg[k], dt, difc[k], exp[k]) for k in range(n)])
    ok = ue > 0
    assert (np.abs(uo[ok] - ue[ok]) / ue[ok]).max() < 1e-9
    assert np.array_equal(uo[~ok] <= 0, ue[~ok] <= 0)


@pytest.mark.parametrize("name", ["onestep_reflect", "onestep_periodic", "onestep_sparse"])
def test_deterministic_step_matches_reference_recording(name):
    """One step against the reference engine's own recorded step
    (tests/golden, made by oracle/ref_harness.c): the reference's start state,
    displacements and first-order outcomes go in through the injection mode;
    the result must equal the reference's state after the step (positions to
    1e-5 of the box side, FP32 box-local storage)."""
    from tests import golden_cases as gd
    g = gd.load(name)
    s = gc.make_sim(L=g["L"], wall=g["wall"], kf=g["kf"], kr=g["kr"], difc=gd.DIFC, dt=gd.DT,
                    rev_placement=(sb.RPirrev, 0.0))
    s.set_molecules(g["pos0"], g["sp0"], g["serno0"])
    force = np.where(g["uni"] == 1, 0, -1).astype(np.float64)
    s.inject(g["serno0"], np.concatenate([g["disp"], force[:, None]], axis=1))
    s.run_steps(1)
    gpos, gsp, gsn = s.molecules()
    act = dict(pos=gpos, sp=gsp, serno=gsn, orig=gsn < (1 << 41))
    ncommon, nprod, nties = gd.compare(g, gd.reference_state(g), act, 1e-5)
    assert ncommon > 2500 and nprod >= 10


@pytest.mark.parametrize("name", ["onestep_confspread", "onestep_bounce"])
def test_bimolecular_placement_matches_reference_recording(name):
    """confspread and bounce product placement (doreact, smolreact.c:2736-2805)
    against one step recorded from the reference: every molecule keeps its
    serial number in both placements, so each one is compared by serial
    number — species and position (1e-5 of the side) — away from ambiguous
    multi-candidate groups and binding-radius ties."""
    import ctypes as C
    import tempfile
    from tests import golden_cases as gd
    g = gd.load(name)
    with tempfile.TemporaryDirectory() as d:
        with open(d + "/cfg.txt", "w") as f:
            f.write(str(g["config"]))
        lib = sb.load()
        simp = C.c_void_p()
        assert lib.smolLoadSimFromFile((d + "/").encode(), b"cfg.txt", C.byref(simp), b"") == 0, sb.last_error()
    s = sb.Sim(ptr=simp.value)
    s.set_molecules(g["pos0"], g["sp0"], g["serno0"])
    s.inject(g["serno0"], np.concatenate([g["disp"], np.full((len(g["sp0"]), 1), -1.0)], axis=1))
    s.run_steps(1)
    gpos, gsp, gsn = s.molecules()
    L, periodic = g["L"], True
    idx, moved = gd.tie_set(g)
    tie_sn = {int(g["serno0"][i]) for i in idx}
    ref = {int(k): i for i, k in enumerate(g["serno1"].tolist())}
    eng = {int(k): i for i, k in enumerate(gsn.tolist())}
    assert set(ref) == set(eng)  # nobody is created or removed
    changed = 0
    for k in ref:
        if k in tie_sn:
            continue
        i, j = ref[k], eng[k]
        assert g["sp1"][i] == gsp[j], (k, g["sp1"][i], gsp[j])
        dpos = gc.min_image(g["pos1"][i] - gpos[j], L, periodic)
        assert np.abs(dpos).max() <= 1e-5 * L, (k, g["pos1"][i], gpos[j])
        i0 = int(np.where(g["serno0"] == k)[0][0])
        changed += int(np.abs(gc.min_image(g["pos1"][i] - moved[i0], L, periodic)).max() > 1e-6 or
                       g["sp1"][i] != g["sp0"][i0])
    assert changed > 10  # reactions did happen away from ties


def test_anisotropic_diffusion_covariance():
    """difm (smolmolec.c:3158-3162): each step is M * sqrt(2 dt) * g, so the
    displacement covariance after time t is 2 t M M^T.  20000 molecules in a
    box too large for the walls to matter; every entry within 5 % of the
    largest (the sampling error of a variance at this count is about 1 %)."""
    import ctypes as C
    L, n, dt, steps = 1000.0, 20000, 0.01, 100
    s = sb.Sim(3, (0, 0, 0), (L, L, L))
    s.add_species("A", 1.0)
    for d in range(3):
        s.boundary(d, -1, "r")
    s.set_times(0, 1e6, dt)
    s.seed(17)
    M = np.array([[1.0, 0.5, 0.0], [0.0, 2.0, 0.0], [0.0, 0.0, 0.5]])
    mflat = np.ascontiguousarray(M.ravel())
    assert s.lib.smolSetSpeciesMobility(s.ptr, b"A", sb.MSsoln, -1.0, None, sb.dptr(mflat)) == 0
    rng = np.random.default_rng(5)
    pos0 = rng.uniform(400, 600, size=(n, 3))
    s.set_molecules(pos0, np.ones(n, dtype=np.int32), np.arange(1, n + 1, dtype=np.uint64))
    s.run_steps(steps)
    pos1, _, sn = s.molecules()
    disp = pos1[np.argsort(sn)] - pos0
    cov = disp.T @ disp / n
    expect = 2 * steps * dt * M @ M.T
    assert np.abs(cov - expect).max() <= 0.05 * np.abs(expect).max(), (cov, expect)

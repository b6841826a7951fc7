"""The oracle's radial-distribution-function solver against the reference
(CPU only).

1. The primitives (rdfdiffuse, rdfabsorb, rdfreverserxn, rdfsteadystate;
   rxnparam.c:784-912) of the oracle restatement (oracle/rdf_oracle.c) agree
   bit for bit with the reference's own functions compiled from rxnparam.c
   (oracle/_ref/librxnparam_ref.so) on the same grids and profiles.
2. The oracle's sweeps reproduce the tables that the reference computed with
   the same method and embedded in numrxnrate / numrxnrateprob (read here from
   this library's compiled-in copies): the downward sweeps of yb (100 points,
   eps 1e-5) and kb (200 points, eps 1e-6), over the large-step head of each
   sweep where every solve takes a few dozen iterations.
3. The device entry points reject bad arguments before touching the GPU.
"""
import ctypes as C
import os

import numpy as np
import pytest

import smoldyn_b200 as sb
from tests import oracle_lib

_dp = C.POINTER(C.c_double)
PVECT = [0, 0.01, 0.02, 0.05, 0.1, 0.2, 0.5, 1.0]   # rxnparam.c:1012


def dptr(a):
    return a.ctypes.data_as(_dp)


def ora():
    lib = C.CDLL(oracle_lib.ensure_built())
    for f in ("ora_rdf_absorb", "ora_rdf_steady", "ora_erfc_nr"):
        getattr(lib, f).restype = C.c_double
    return lib


def ref():
    so = os.path.join(oracle_lib.REF_DIR, "librxnparam_ref.so")
    if not os.path.exists(so):
        pytest.skip("reference rxnparam library not built")
    lib = C.CDLL(so)
    for f in ("rdfabsorb", "rdfsteadystate", "rxnparam_erfccD"):
        getattr(lib, f).restype = C.c_double
    return lib


def grid(lib, mode, n, b, shift=0.0):
    r = np.zeros(n)
    assert lib.ora_rdf_grid(ord(mode), n, C.c_double(b), dptr(r)) == 0
    return r + shift


def profile(r, seed):
    rng = np.random.default_rng(seed)
    g = np.where(r < 1, 0.05 * rng.random(len(r)), 1 - 0.8 / np.maximum(r, 1e-3) * rng.random(len(r)))
    return np.ascontiguousarray(g)


CASES = [("i", 150, -1.0, 0.0), ("r", 150, 2.0, 0.0), ("b", 150, 0.5, 0.0), ("i", 120, -1.0, 0.003)]


@pytest.mark.parametrize("mode,n,b,shift", CASES)
def test_primitives_bit_exact(mode, n, b, shift):
    o, R = ora(), ref()
    r = grid(o, mode, n, b if b > 0 else 1.0, shift)
    for k, step in enumerate((0.07, 0.6, 3.0)):
        g = profile(r, k)
        d1, d2 = np.zeros(n), np.zeros(n)
        o.ora_rdf_diffuse(dptr(r), dptr(g), dptr(d1), n, C.c_double(step))
        R.rdfdiffuse(dptr(r), dptr(g), dptr(d2), n, C.c_double(step))
        assert np.array_equal(d1, d2)
        for prob in (1.0, 0.3):
            a1, a2 = d1.copy(), d1.copy()
            f1 = o.ora_rdf_absorb(dptr(r), dptr(a1), n, C.c_double(1.0), C.c_double(prob))
            f2 = R.rdfabsorb(dptr(r), dptr(a2), n, C.c_double(1.0), C.c_double(prob))
            assert f1 == f2 and np.array_equal(a1, a2)
        for bb in (0.0, 0.7, 2.5):
            v1, v2 = d1.copy(), d1.copy()
            o.ora_rdf_reverse(dptr(r), dptr(v1), n, C.c_double(step), C.c_double(bb), C.c_double(0.4))
            R.rdfreverserxn(dptr(r), dptr(v2), n, C.c_double(step), C.c_double(bb), C.c_double(0.4))
            assert np.array_equal(v1, v2)
    for x in np.linspace(-4, 6, 41):
        assert o.ora_erfc_nr(C.c_double(x)) == R.rxnparam_erfccD(C.c_double(x))


@pytest.mark.parametrize("mode,b,prob,step", [("i", -1.0, 1.0, 0.5), ("i", -1.0, 0.2, 2.0), ("r", 2.0, 1.0, 0.4),
                                             ("b", 0.5, 1.0, 3.0), ("b", 0.0, 0.5, 1.5)])
def test_steady_state_bit_exact(mode, b, prob, step):
    o, R = ora(), ref()
    n = 100
    r = grid(o, mode, n, b)
    g1 = np.where(r < 1, 0.0, 1.0)
    g2 = g1.copy()
    d1, d2 = np.zeros(n), np.zeros(n)
    it = C.c_int()
    f1 = o.ora_rdf_steady(dptr(r), dptr(g1), dptr(d1), n, C.c_double(step), C.c_double(1), C.c_double(b),
                          C.c_double(1e-5), C.c_double(prob), C.byref(it))
    f2 = R.rdfsteadystate(dptr(r), dptr(g2), dptr(d2), n, C.c_double(step), C.c_double(1), C.c_double(b),
                          C.c_double(1e-5), C.c_double(prob))
    assert it.value >= 30
    assert f1 == f2 and np.array_equal(g1, g2) and np.array_equal(d1, d2)


def down_sweep_head(o, mode, n, eps, b, prob, count):
    r = grid(o, mode, n, b)
    g = np.ascontiguousarray(np.where(r < 1, 0.0, 1.0))
    d = np.zeros(n)
    sv = np.zeros(40)
    assert o.ora_rdf_steps(ord("d"), dptr(sv)) == 31
    out = []
    for k in range(count):
        out.append(o.ora_rdf_steady(dptr(r), dptr(g), dptr(d), n, C.c_double(sv[k]), C.c_double(1), C.c_double(b),
                                    C.c_double(eps), C.c_double(prob), None))
    return np.array(out)


@pytest.mark.parametrize("row", [0, 5, 10])
def test_oracle_sweep_reproduces_yb_head(row):
    """yb: 100 points, eps 1e-5, downward sweep; rows b = 0, 0.1, ... 1;
    within a row decreasing step (rxnparam.c:61-64)."""
    o = ora()
    yb = sb.rxn_table("yb").reshape(11, 31)
    got = down_sweep_head(o, "b", 100, 1e-5, 0.1 * row, 1.0, 12)
    assert np.all(np.abs(got - yb[row, :12]) <= 1e-6 + 1e-9 * np.abs(yb[row, :12])), (got, yb[row, :12])


@pytest.mark.parametrize("brow,pi", [(0, 3), (4, 6), (10, 1)])
def test_oracle_sweep_reproduces_kb_head(brow, pi):
    """kb: 200 points, eps 1e-6, downward sweep; groups b = 0 .. 1, rows over
    the probabilities (rxnparam.c:302-304).  Within a row the values run in
    the sweep's decreasing-step order (its comment says increasing, but the
    data start at the large-step limit 4 pi/3 prob and end with the -1 of
    failed small-step solves, as yb does)."""
    o = ora()
    kb = sb.rxn_table("kb").reshape(11, 8, 31)
    want = kb[brow, pi, :8]
    got = down_sweep_head(o, "b", 200, 1e-6, [0.1 * k for k in range(11)][brow], PVECT[pi], 8)
    assert np.all(np.abs(got - want) <= 1e-6 + 1e-9 * np.abs(want)), (got, want)


def test_row_and_step_values_match_reference_sweeps():
    o = ora()
    bv = np.zeros(32)
    assert o.ora_rdf_rows(ord("r"), dptr(bv)) == 16
    assert abs(bv[15] - np.exp(3.0)) < 1e-9
    assert o.ora_rdf_rows(ord("b"), dptr(bv)) == 11
    sv = np.zeros(40)
    assert o.ora_rdf_steps(ord("u"), dptr(sv)) == 31
    assert abs(sv[0] - np.exp(-3)) < 1e-15 and abs(sv[30] / np.exp(3) - 1) < 1e-12


def test_tables_are_compiled_in():
    sizes = {"yi": 31, "yr": 16 * 31, "yb": 11 * 31, "kirr": 8 * 31, "krev": 16 * 8 * 31, "kb": 11 * 8 * 31}
    lib = sb.load()
    for name, size in sizes.items():
        assert len(sb.rxn_table(name)) == size
    assert lib.smolgpuRxnTable(b"nope", None, 0) == -1


def test_device_entry_points_reject_bad_arguments():
    lib = sb.load()
    flux = np.zeros(16 * 31)
    nr = C.c_int()
    assert lib.smolgpuRdfTable(b"x", 100, 1e-5, b"u", 1, None, sb.dptr(flux), None, C.byref(nr)) == sb.ECbounds
    assert lib.smolgpuRdfTable(b"i", 100, 1e-5, b"q", 1, None, sb.dptr(flux), None, C.byref(nr)) == sb.ECbounds
    assert lib.smolgpuRdfTable(b"i", 5, 1e-5, b"u", 1, None, sb.dptr(flux), None, C.byref(nr)) == sb.ECbounds
    assert lib.smolgpuRdfTable(b"i", 100, 0.0, b"u", 1, None, sb.dptr(flux), None, C.byref(nr)) == sb.ECbounds
    bad = np.array([1.5])
    assert lib.smolgpuRdfTable(b"i", 100, 1e-5, b"u", 1, sb.dptr(bad), sb.dptr(flux), None, C.byref(nr)) == sb.ECbounds
    r = np.linspace(0, 5, 20)
    r[3] = 0.0
    g = np.ones(20)
    one = np.ones(1)
    assert lib.smolgpuRdfSteadyState(1, 20, sb.dptr(r), sb.dptr(g), None, sb.dptr(one), sb.dptr(one), sb.dptr(one),
                                     sb.dptr(one), 1e-5, sb.dptr(one), None) == sb.ECbounds

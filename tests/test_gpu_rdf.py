"""The device radial-distribution-function solver (smolgpuRdfSteadyState,
smolgpuRdfTable) against the oracle and against the reference's tables.

1. Single steady states (rdfsteadystate, rxnparam.c:898-912) on the device
   agree with the oracle restatement (itself bit-identical to the reference,
   tests/test_oracle_rdf.py) on the same grids, trial profiles, step lengths,
   unbinding radii and probabilities: same iteration counts, fluxes within
   1e-9 relative, profiles within 1e-9 absolute.  The device sums the
   trapezoid segments in a different order and uses the GPU's exp, so the
   agreement is to rounding, not bitwise.
2. Whole sweeps regenerate the rate tables that the reference computed with
   this method and compiled into numrxnrate / numrxnrateprob (rxnparam.c:58-76,
   162-304), with the point counts, tolerances and sweep directions named in
   the tables' comments; values printed by the reference to 6 decimals (the
   "up&down" tables are means of two such values) agree within 1.5e-6, and the
   -1 entries (solves that gave up) fall on the same places.
"""
import ctypes as C

import numpy as np
import pytest

import smoldyn_b200 as sb
from tests import oracle_lib

pytestmark = pytest.mark.gpu

_dp = C.POINTER(C.c_double)
PVECT = [0, 0.01, 0.02, 0.05, 0.1, 0.2, 0.5, 1.0]   # rxnparam.c:1012


def dptr(a):
    return a.ctypes.data_as(_dp)


def ora():
    lib = C.CDLL(oracle_lib.ensure_built())
    lib.ora_rdf_steady.restype = C.c_double
    return lib


def grid(o, mode, n, b):
    r = np.zeros(n)
    assert o.ora_rdf_grid(ord(mode), n, C.c_double(b), dptr(r)) == 0
    return r


SOLVES = [  # mode, b, prob, step
    ("i", -1.0, 1.0, 0.06), ("i", -1.0, 1.0, 0.8), ("i", -1.0, 1.0, 9.0), ("i", -1.0, 0.05, 0.3),
    ("r", 1.5, 1.0, 0.2), ("r", 4.0, 0.5, 2.0), ("b", 0.0, 1.0, 3.0), ("b", 0.6, 1.0, 1.2),
    ("b", 0.3, 0.2, 0.5), ("i", -1.0, 0.0, 1.0),
]


def test_steady_states_match_oracle():
    o = ora()
    n, eps = 128, 1e-6
    r = np.array([grid(o, m, n, b if m == "r" else 1.0) for m, b, _, _ in SOLVES])
    trial = np.where(r < 1, 0.0, 1.0)
    b = np.array([s[1] for s in SOLVES])
    prob = np.array([s[2] for s in SOLVES])
    step = np.array([s[3] for s in SOLVES])
    flux, ga, gd, iters = sb.rdf_steady_state(r, trial, step, 1.0, b, prob, eps)
    for k in range(len(SOLVES)):
        ra = np.ascontiguousarray(trial[k].copy())
        rd = np.zeros(n)
        it = C.c_int()
        f = o.ora_rdf_steady(dptr(np.ascontiguousarray(r[k])), dptr(ra), dptr(rd), n, C.c_double(step[k]),
                             C.c_double(1.0), C.c_double(b[k]), C.c_double(eps), C.c_double(prob[k]), C.byref(it))
        assert iters[k] == it.value, (SOLVES[k], iters[k], it.value)
        assert abs(flux[k] - f) <= 1e-9 * max(abs(f), 1e-12), (SOLVES[k], flux[k], f)
        assert np.max(np.abs(ga[k] - ra)) <= 1e-9, SOLVES[k]
        assert np.max(np.abs(gd[k] - rd)) <= 1e-9, SOLVES[k]


def check_table(got, want):
    fail_g, fail_w = got < 0, want < 0
    assert np.array_equal(fail_g, fail_w), (np.argwhere(fail_g != fail_w)[:5], got[fail_g != fail_w][:5])
    ok = ~fail_w
    dev = np.abs(got[ok] - want[ok])
    assert dev.max() <= 1.5e-6 + 1e-9 * np.abs(want[ok]).max(), (dev.max(), np.argmax(dev))


def test_regenerates_yi():
    """yi: 600 points, eps 1e-5, up and down averaged, decreasing step."""
    flux, _ = sb.rdf_table("i", 600, 1e-5, "a")
    check_table(flux.reshape(-1), sb.rxn_table("yi"))


def test_regenerates_yb():
    """yb: 100 points, eps 1e-5, down only, decreasing step."""
    flux, _ = sb.rdf_table("b", 100, 1e-5, "d")
    check_table(flux.reshape(-1), sb.rxn_table("yb"))


def test_regenerates_yr():
    """yr: 500 points, eps 1e-5, up and down averaged, decreasing step."""
    flux, _ = sb.rdf_table("r", 500, 1e-5, "a")
    check_table(flux.reshape(-1), sb.rxn_table("yr"))


def test_regenerates_kirr():
    """kirr: 200 points, eps 1e-6, up and down averaged, increasing step."""
    flux, _ = sb.rdf_table("i", 200, 1e-6, "a", PVECT)
    check_table(flux[:, :, ::-1].reshape(-1), sb.rxn_table("kirr"))


def test_regenerates_krev():
    """krev: 200 points, eps 1e-6, up and down averaged, increasing step."""
    flux, _ = sb.rdf_table("r", 200, 1e-6, "a", PVECT)
    check_table(flux[:, :, ::-1].reshape(-1), sb.rxn_table("krev"))


def test_regenerates_kb():
    """kb: 200 points, eps 1e-6, down only, decreasing step."""
    flux, _ = sb.rdf_table("b", 200, 1e-6, "d", PVECT)
    check_table(flux.reshape(-1), sb.rxn_table("kb"))

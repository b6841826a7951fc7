"""Binding/unbinding radius solver parity (CPU).

1. The oracle's C restatement equals the reference's own rxnparam.c
   (compiled unchanged by oracle/Makefile) on randomized inputs covering every
   table branch of numrxnrate / numrxnrateprob (rxnparam.c:57-518).
2. The product's host FP64 solver (the one simupdate-equivalent code uses)
   matches the reference to 1e-9 relative.
"""
import ctypes as C

import numpy as np
import pytest

import smoldyn_b200 as sb
from tests import oracle_lib

REL = 1e-9


def _inputs(n=4000, seed=12345):
    rng = np.random.default_rng(seed)
    rate = 10 ** rng.uniform(-4, 2, n)
    dt = 10 ** rng.uniform(-4, 0, n)
    difc = 10 ** rng.uniform(-2, 1, n)
    mode = rng.integers(0, 4, n)  # 0 irreversible, 1 unbind radius, 2 ratio<1, 3 ratio>1
    b = np.where(mode == 0, -1.0, np.where(mode == 1, 10 ** rng.uniform(-3, 0, n),
                 np.where(mode == 2, rng.uniform(0.01, 0.99, n), rng.uniform(1.01, 20, n))))
    rel = np.where(mode >= 2, 1, 0)
    return rate, dt, difc, b, rel


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.fixture(scope="module")
def ref():
    lib = oracle_lib.reference_rxnparam()
    if lib is None:
        pytest.skip("reference rxnparam not compiled (make -C oracle ref)")
    return lib


def test_oracle_numrxnrate_equals_reference(ref):
    ora = oracle_lib.oracle()
    rng = np.random.default_rng(1)
    for _ in range(3000):
        step = 10 ** rng.uniform(-3, 2)
        a = 10 ** rng.uniform(-3, 1)
        kind = rng.integers(0, 3)
        b = -1.0 if kind == 0 else a * (rng.uniform(0, 1) if kind == 1 else rng.uniform(1, 25))
        assert ora.ora_numrxnrate(step, a, b) == ref.numrxnrate(step, a, b)
        p = rng.uniform(0.001, 0.999)
        x, y = ora.ora_numrxnrateprob(step, a, b, p), ref.numrxnrateprob(step, a, b, p)
        assert x == y or _rel(x, y) < 1e-14, (step, a, b, p, x, y)


def test_oracle_radii_equal_reference(ref):
    ora = oracle_lib.oracle()
    rate, dt, difc, b, rel = _inputs(1500)
    for k in range(len(rate)):
        x = ora.ora_bindingradius(rate[k], dt[k], difc[k], b[k], int(rel[k]))
        y = ref.bindingradius(rate[k], dt[k], difc[k], b[k], int(rel[k]))
        assert x == y, (k, x, y)
        if y > 0:
            pg = 0.05 + 0.5 * (k % 7) / 7
            assert ora.ora_unbindingradius(pg, dt[k], difc[k], y) == ref.unbindingradius(pg, dt[k], difc[k], y)


def test_oracle_bindingradiusprob_equals_reference(ref):
    ora = oracle_lib.oracle()
    rng = np.random.default_rng(3)
    for _ in range(150):
        rate, dt, difc = 10 ** rng.uniform(-3, 1), 10 ** rng.uniform(-3, -1), 10 ** rng.uniform(-1, 1)
        p = C.c_double(rng.uniform(0.05, 0.9))
        q = C.c_double(p.value)
        x = ora.ora_bindingradiusprob(rate, dt, difc, -1.0, 0, -1.0, C.byref(p))
        y = ref.bindingradiusprob(rate, dt, difc, -1.0, 0, -1.0, C.byref(q))
        assert x == y


def test_product_host_solver_matches_reference(ref):
    lib = sb.load()
    rate, dt, difc, b, rel = _inputs(4000, seed=7)
    worst = 0.0
    for k in range(len(rate)):
        y = ref.bindingradius(rate[k], dt[k], difc[k], b[k], int(rel[k]))
        x = lib.smolgpuBindingRadiusHost(rate[k], dt[k], difc[k], b[k], int(rel[k]))
        if y == 0 or not np.isfinite(y):
            assert x == y
            continue
        worst = max(worst, _rel(x, y))
        if y > 0:
            pg = 0.02 + 0.9 * (k % 11) / 11
            u_ref = ref.unbindingradius(pg, dt[k], difc[k], y)
            u = lib.smolgpuUnbindingRadiusHost(pg, dt[k], difc[k], y)
            assert u == u_ref or _rel(u, u_ref) < REL
    assert worst < REL, worst


def test_edge_inputs(ref):
    lib = sb.load()
    cases = [(0.0, 0.01, 1.0, -1.0, 0), (1.0, 0.0, 1.0, -1.0, 0), (1.0, 0.0, 1.0, 2.0, 1), (1.0, 0.0, 1.0, 0.5, 1),
             (1.0, 0.0, 1.0, 0.3, 0), (-1.0, 0.1, 1.0, -1.0, 0), (1.0, 0.1, 0.0, -1.0, 0), (1e3, 1e-2, 1.0, -1.0, 0)]
    for c in cases:
        assert lib.smolgpuBindingRadiusHost(*c) == ref.bindingradius(*c)
    for c in [(0.0, 0.01, 1.0, 0.1), (1.0, 0.01, 1.0, 0.1), (0.5, 0.0, 1.0, 0.1), (0.2, 0.01, 1.0, 0.0)]:
        assert lib.smolgpuUnbindingRadiusHost(*c) == ref.unbindingradius(*c)


def _prob_inputs(n, seed):
    """Random (rate, dt, difc, b, rel, p) over every branch of numrxnrateprob:
    irreversible, unbinding radius b >= a (log-b table) and b < a (linear-b
    table), known probabilities between the table's grid values."""
    rng = np.random.default_rng(seed)
    rate = 10 ** rng.uniform(-3, 1.5, n)
    dt = 10 ** rng.uniform(-3, -0.5, n)
    difc = 10 ** rng.uniform(-1, 1, n)
    mode = rng.integers(0, 3, n)
    b = np.where(mode == 0, -1.0, np.where(mode == 1, rng.uniform(1.05, 15, n), rng.uniform(0.05, 0.95, n)))
    rel = np.where(mode == 0, 0, 1)
    p = rng.uniform(0.02, 0.98, n)
    return rate, dt, difc, b, rel, p


def test_product_numrxnrateprob_matches_reference(ref):
    """smolgpuNumRxnRateProbHost (the product's numrxnrateprob, every
    second-order reaction with p < 1 goes through it) equals rxnparam.c."""
    lib = sb.load()
    rng = np.random.default_rng(11)
    worst = 0.0
    for _ in range(4000):
        step = 10 ** rng.uniform(-3, 2)
        a = 10 ** rng.uniform(-3, 1)
        kind = rng.integers(0, 3)
        b = -1.0 if kind == 0 else a * (rng.uniform(0, 1) if kind == 1 else rng.uniform(1, 25))
        p = rng.choice([rng.uniform(0.001, 0.999), 0.01, 0.05, 0.5, 1.0, 0.0])
        x, y = lib.smolgpuNumRxnRateProbHost(step, a, b, p), ref.numrxnrateprob(step, a, b, p)
        if x != y:
            worst = max(worst, _rel(x, y))
    assert worst < REL, worst


def test_product_bindingradiusprob_known_probability(ref):
    """bindingradiusprob with a given probability (the 1-D multiplicative
    search, rxnparam.c:612-636) on the product's host path equals the
    reference to 1e-9 relative, probability passed through unchanged."""
    lib = sb.load()
    rate, dt, difc, b, rel, p = _prob_inputs(600, 12)
    worst = 0.0
    for k in range(len(rate)):
        px, py = C.c_double(p[k]), C.c_double(p[k])
        x = lib.smolgpuBindingRadiusProbHost(rate[k], dt[k], difc[k], b[k], int(rel[k]), -1.0, C.byref(px))
        y = ref.bindingradiusprob(rate[k], dt[k], difc[k], b[k], int(rel[k]), -1.0, C.byref(py))
        assert px.value == py.value == p[k]
        if x != y:
            worst = max(worst, _rel(x, y))
    assert worst < REL, worst


def test_product_bindingradiusprob_chi_search(ref):
    """bindingradiusprob with a requested chi (the 2-D search over radius and
    probability, rxnparam.c:638-676): radius and the probability found equal
    the reference's to 1e-9 relative; includes chi values too large to need
    the search (p stays 1) and the dt = 0 closed form."""
    lib = sb.load()
    rate, dt, difc, b, rel, _ = _prob_inputs(300, 13)
    rng = np.random.default_rng(14)
    chi = 10 ** rng.uniform(-3, -0.05, len(rate))
    dt = np.where(rng.uniform(size=len(rate)) < 0.05, 0.0, dt)
    worst, searched = 0.0, 0
    for k in range(len(rate)):
        px, py = C.c_double(-1.0), C.c_double(-1.0)
        x = lib.smolgpuBindingRadiusProbHost(rate[k], dt[k], difc[k], b[k], int(rel[k]), chi[k], C.byref(px))
        y = ref.bindingradiusprob(rate[k], dt[k], difc[k], b[k], int(rel[k]), chi[k], C.byref(py))
        searched += py.value < 1.0
        for u, v in ((x, y), (px.value, py.value)):
            if u != v:
                worst = max(worst, _rel(u, v))
    assert searched > 50, searched
    assert worst < REL, worst


def test_product_bindingradiusprob_edges(ref):
    lib = sb.load()
    cases = [(0.0, 0.01, 1.0, -1.0, 0, -1.0, 0.5), (1.0, 0.01, 1.0, -1.0, 0, -1.0, 0.0),
             (1.0, 0.01, 1.0, -1.0, 0, -1.0, 1.0), (1.0, 0.01, 0.0, -1.0, 0, -1.0, 0.5),
             (1.0, 0.01, 1.0, -1.0, 0, 1.5, 0.5), (1.0, 0.0, 1.0, -1.0, 0, 0.3, -1.0),
             (1.0, 0.0, 1.0, 2.0, 1, 0.3, -1.0), (1.0, 0.0, 1.0, 0.5, 0, 0.3, -1.0), (1.0, 0.0, 1.0, 0.5, 1, 0.3, -1.0)]
    for rate, dt, difc, b, rel, chi, p in cases:
        px, py = C.c_double(p), C.c_double(p)
        x = lib.smolgpuBindingRadiusProbHost(rate, dt, difc, b, rel, chi, C.byref(px))
        y = ref.bindingradiusprob(rate, dt, difc, b, rel, chi, C.byref(py))
        assert x == y and px.value == py.value, (rate, dt, difc, b, rel, chi, p, x, y, px.value, py.value)

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

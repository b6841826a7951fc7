"""bindingradiusprob on the device (smolgpuSolveRadiiProb, one thread per
problem, the same rxnparam.cuh code as the host path) against the reference's
own rxnparam.c (oracle/_ref/librxnparam_ref.so).

Known probability (the 1-D multiplicative search, rxnparam.c:612-636) and
requested chi (the 2-D search over radius and probability,
rxnparam.c:638-676).  The searches stop at a squared relative error of 1e-6
after up to 200 / 300 multiplicative moves, and each move compares two
errors, so a device exp/log that differs from glibc's in the last bit can
send a search down another path where the search has not converged.  Known
probability: every radius equals the reference's within 1e-9 relative.
Chi: see test_device_chi_search.
"""
import ctypes as C

import numpy as np
import pytest

import smoldyn_b200 as sb
from tests import oracle_lib
from tests.test_oracle_rxnparam import _prob_inputs

pytestmark = pytest.mark.gpu
REL = 1e-9


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


@pytest.fixture(scope="module")
def ref():
    lib = oracle_lib.reference_rxnparam()
    if lib is None:
        pytest.skip("reference rxnparam not compiled (make -C oracle ref)")
    return lib


def _reference(ref, rate, dt, difc, b, rel, chi, prob):
    out, pout = np.zeros(len(rate)), np.zeros(len(rate))
    for k in range(len(rate)):
        p = C.c_double(prob[k])
        out[k] = ref.bindingradiusprob(rate[k], dt, difc[k], b[k], rel, chi[k], C.byref(p))
        pout[k] = p.value
    return out, pout


@pytest.mark.parametrize("rel", [0, 1])
def test_device_known_probability(ref, rel):
    rate, _, difc, b, _, p = _prob_inputs(3000, 31 + rel)
    if rel == 0:
        b = np.where(b > 0, b * 0.05, b)  # absolute unbinding radii
    dt = 0.01
    chi = np.full(len(rate), -1.0)
    a_ref, p_ref = _reference(ref, rate, dt, difc, b, rel, chi, p)
    a, pp = sb.solve_radii_prob_device(rate, dt, difc, b, rel, chi, p)
    assert np.array_equal(pp, p_ref)
    same = np.sum(a == a_ref)
    print("known probability, rel=%d: %d of %d bit-identical" % (rel, same, len(a)))
    assert np.all(_rel(a, a_ref) <= REL), np.max(_rel(a, a_ref))


def _chi_objective(ref, rate, dt, difc, b, chi, a, p):
    """The 2-D search's own objective (rxnparam.c:648-664): squared relative
    errors of the rate and of chi at (a, p), evaluated with the reference's
    numrxnrateprob (ratio unbinding radius b * a)."""
    step = np.sqrt(2 * difc * dt)
    out = np.zeros(len(rate))
    for k in range(len(rate)):
        ub = b[k] * a[k]
        rt = ref.numrxnrateprob(step[k], a[k], ub, p[k]) / dt
        ch = rate[k] / (4 * np.pi * difc[k] * a[k] * ub / (ub - a[k])) if ub >= 0 else \
            rate[k] / (4 * np.pi * difc[k] * a[k])
        out[k] = (rt / rate[k] - 1) ** 2 + (ch / chi[k] - 1) ** 2
    return out


def test_device_chi_search(ref):
    """The 2-D search stops when its objective falls below 1e-6 or after 300
    rounds; on these inputs the reference itself ends above 1e-6 (not
    converged) in about two thirds of the searched cases, and there the
    answer is wherever its path stood.  Where the reference converged, the
    device result equals it to 1e-9; where it did not, a last-bit difference
    of a device exp/log can move the path, so those results are reported
    (objective of the device's point against the reference's) and at least
    90% of all problems must still be bit-identical."""
    rate, _, difc, b, _, _ = _prob_inputs(1500, 33)
    rng = np.random.default_rng(34)
    chi = 10 ** rng.uniform(-3, -0.05, len(rate))
    dt = 0.01
    p0 = np.full(len(rate), -1.0)
    a_ref, p_ref = _reference(ref, rate, dt, difc, b, 1, chi, p0)
    a, pp = sb.solve_radii_prob_device(rate, dt, difc, b, 1, chi, p0)
    searched = p_ref < 1
    e_ref = _chi_objective(ref, rate, dt, difc, b, chi, a_ref, p_ref)
    e_dev = _chi_objective(ref, rate, dt, difc, b, chi, a, pp)
    conv = e_ref <= 1e-6
    same = (a == a_ref) & (pp == p_ref)
    print("chi search: %d searched, reference converged in %d; %d of %d bit-identical; differing: %d converged, "
          "%d not" % (searched.sum(), (searched & conv).sum(), same.sum(), len(a), (~same & conv).sum(),
                      (~same & ~conv).sum()))
    assert searched.sum() > 200
    assert np.all(_rel(a[conv], a_ref[conv]) <= REL) and np.all(_rel(pp[conv], p_ref[conv]) <= REL)
    d = ~same & ~conv
    if d.any():
        print("not converged and differing: objective device/reference median %.3g, max %.3g" %
              (np.median(e_dev[d] / e_ref[d]), np.max(e_dev[d] / e_ref[d])))
    assert same.mean() > 0.9

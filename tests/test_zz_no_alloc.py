"""smolgpuSolveRadiiNoAlloc, the radius solve for callers that cannot allocate
device memory (for example a rate update issued while an ensemble steps on
another stream, where a cudaMalloc/cudaFree could synchronise the device and
stall the steps), against the allocating smolgpuSolveRadii.

Two calls in a row through the fixed device scratch — a larger
binding-radius solve, then a smaller unbinding-radius solve, so stale scratch
left by the first call would show in the second — must equal the allocating
entry point bit for bit (both run the same FP64 kernel).  A call above the
65536-problem limit is rejected with ECbounds.
"""
import numpy as np
import pytest

import smoldyn_b200 as sb

pytestmark = pytest.mark.gpu

LIMIT = 65536


def _binding_case(n, seed):
    rng = np.random.default_rng(seed)
    rate = 10 ** rng.uniform(-4, 1, n)
    difc = rng.uniform(0.2, 3.0, n)
    b = np.where(rng.uniform(size=n) < 0.5, rng.uniform(0.0, 2.0, n), -1.0)
    return rate, difc, b


def test_two_calls_match_allocating_solver():
    dt = 0.01
    rate, difc, b = _binding_case(40000, 21)
    a_ref = sb.solve_radii_device(0, rate, dt, difc, b, rel=1)
    a_new = sb.solve_radii_device_noalloc(0, rate, dt, difc, b, rel=1)
    assert np.array_equal(a_ref, a_new, equal_nan=True)

    # second call, smaller: unbinding radii from the radii just computed
    rng = np.random.default_rng(22)
    m = 9000
    pgem = rng.uniform(0.01, 0.5, m)
    difc2 = difc[:m]
    a = np.where(np.isfinite(a_ref[:m]) & (a_ref[:m] > 0), a_ref[:m], 0.05)
    u_ref = sb.solve_radii_device(1, pgem, dt, difc2, a)
    u_new = sb.solve_radii_device_noalloc(1, pgem, dt, difc2, a)
    assert np.array_equal(u_ref, u_new, equal_nan=True)


def test_limit_and_bad_arguments_rejected():
    lib = sb.load()
    z = np.zeros(LIMIT + 1)
    dp = sb.dptr
    assert lib.smolgpuSolveRadiiNoAlloc(0, LIMIT + 1, dp(z), 0.01, dp(z), dp(z), 0, dp(z)) == sb.ECbounds
    assert "exceeds" in sb.last_error()[2]
    assert lib.smolgpuSolveRadiiNoAlloc(2, 10, dp(z), 0.01, dp(z), dp(z), 0, dp(z)) == sb.ECbounds
    # exactly the limit is accepted
    rate, difc, b = _binding_case(LIMIT, 23)
    out = sb.solve_radii_device_noalloc(0, rate, 0.01, difc, b, rel=1)
    assert np.array_equal(out, sb.solve_radii_device(0, rate, 0.01, difc, b, rel=1), equal_nan=True)


def test_call_after_setup_allocates_nothing():
    """The property the entry point exists for: once the first call has set
    up the scratch, a full-size call leaves the device's free memory as it
    was (cudaMemGetInfo before and after)."""
    import torch

    rate, difc, b = _binding_case(LIMIT, 24)
    first = sb.solve_radii_device_noalloc(0, rate, 0.01, difc, b, rel=1)  # set-up call
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    again = sb.solve_radii_device_noalloc(0, rate, 0.01, difc, b, rel=1)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert np.array_equal(first, again, equal_nan=True)

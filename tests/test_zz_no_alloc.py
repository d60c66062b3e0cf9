"""GPU: the allocation-free OC entry point against the regular one.

pf_oc_update_noalloc_f64 exists for callers that cannot allocate device memory where they
run the OC step (a plugin under a framework that owns the device memory, a latency-bound
per-iteration callback where cudaMalloc would synchronise the device); it takes its
scratch from a static device array instead of a caller workspace.  Its
results must equal pf_oc_update_f64's on the same inputs, on consecutive calls (the array
keeps the previous call's contents), and sizes beyond the array must be refused.  This
file sorts last so that a run stopping at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from pyfantom_b200 import _lib
    _lib.require_cuda()
    return _lib


def _problem(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, 1.0, n)
    df = -np.abs(rng.standard_normal(n)) * rng.uniform(0.01, 10.0)
    df[::13] = 0.0
    return (torch.as_tensor(x, device="cuda"), torch.as_tensor(df, device="cuda"),
            torch.full((n,), 1.0 / n, dtype=torch.float64, device="cuda"))


def _regular(lib, x, df, dg, vf, move):
    L = lib.load()
    n = x.numel()
    work = torch.empty(int(L.pf_oc_workspace_size(n)), dtype=torch.float64, device="cuda")
    xn = torch.empty_like(x)
    out = (ctypes.c_double * 3)()
    lib.check(L.pf_oc_update_f64(n, lib.ptr(x), lib.ptr(df), lib.ptr(dg), vf, move, lib.ptr(xn), lib.ptr(work),
                                 out, lib.stream()))
    return xn.cpu().numpy(), list(out)


def _noalloc(lib, x, df, dg, vf, move):
    L = lib.load()
    n = x.numel()
    xn = torch.empty_like(x)
    out = (ctypes.c_double * 3)()
    lib.check(L.pf_oc_update_noalloc_f64(n, lib.ptr(x), lib.ptr(df), lib.ptr(dg), vf, move, lib.ptr(xn), out,
                                         lib.stream()))
    return xn.cpu().numpy(), list(out)


def test_noalloc_matches_regular_on_consecutive_calls(lib):
    # two calls in a row on the same inputs, then a smaller problem, then the first again
    cases = [(200_003, 7, 0.3, 0.2), (200_003, 7, 0.3, 0.2), (4_801, 11, 0.5, 0.05), (200_003, 7, 0.3, 0.2)]
    for n, seed, vf, move in cases:
        x, df, dg = _problem(n, seed)
        ref, ref_out = _regular(lib, x, df, dg, vf, move)
        got, got_out = _noalloc(lib, x, df, dg, vf, move)
        assert np.abs(got - ref).max() <= 1e-12
        assert abs(got_out[0] - ref_out[0]) <= 1e-12 * max(1.0, ref_out[0])  # ||x_new - x||
        assert got_out[1] == ref_out[1] and got_out[2] == ref_out[2]      # lambda, bisection steps


def test_noalloc_rejects_sizes_beyond_the_scratch(lib):
    L = lib.load()
    limit = 2097152  # PF_OC_NOALLOC_MAX_ELEMS in include/pyfantom_b200.h
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    status = L.pf_oc_update_noalloc_f64(limit + 1, lib.ptr(x), lib.ptr(x), lib.ptr(x), 0.5, 0.2, lib.ptr(x), None,
                                        lib.stream())
    assert status == lib.PF_BAD_ARG
    assert b"static scratch limit" in L.pf_last_error()

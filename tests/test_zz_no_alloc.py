"""pss_lu_factor_noalloc (device memory owned by the caller, scratch in a fixed device
array) against the allocating entry point pss_lu_solve, both through the C ABI.

The factors from the no-allocation call are applied on the CPU (LAPACK getrs via scipy)
and the solution is compared with pss_lu_solve's FP64 solution of the same system:
relative difference <= 1e-11 on these well-conditioned matrices (both are backward-stable
FP64 LU solves; the bound leaves three orders of magnitude over the observed ~1e-14).
Two factorisations run back to back, so the second reuses the per-device scratch.
"""
import ctypes

import numpy as np
import pytest
import scipy.linalg

from pssfss_b200 import engine

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _system(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3 * np.sqrt(n) * np.eye(n)
    B = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
    return A, B


def _factor_noalloc(A):
    import torch

    n = A.shape[0]
    dA = torch.from_numpy(np.ascontiguousarray(A, dtype=np.complex128)).to("cuda:0")  # row-major, ld = n
    ipiv = torch.full((n,), -1, dtype=torch.int32, device="cuda:0")
    info = torch.full((1,), 7, dtype=torch.int32, device="cuda:0")  # the call must reset it to 0 itself
    stream = torch.cuda.current_stream(0).cuda_stream
    rc = engine.lib().pss_lu_factor_noalloc(n, ctypes.c_void_p(dA.data_ptr()), n, ctypes.c_void_p(ipiv.data_ptr()),
                                            ctypes.c_void_p(info.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 0, engine.lib().pss_last_error().decode()
    torch.cuda.synchronize(0)
    return dA.cpu().numpy(), ipiv.cpu().numpy().astype(np.int64), int(info.cpu().item())


def test_noalloc_factor_matches_allocating_solve_twice():
    for n, seed in ((300, 11), (1100, 12)):
        A, B = _system(n, seed)
        LU, piv, info = _factor_noalloc(A)
        assert info == 0
        assert piv.min() >= 0 and piv.max() < n and np.all(piv >= np.arange(n))
        X_noalloc = scipy.linalg.lu_solve((LU, piv), B)
        X_ref, st = engine.lu_solve(A, B, "fp64")
        assert st == 0
        rel = np.max(np.abs(X_noalloc - X_ref)) / np.max(np.abs(X_ref))
        assert rel < TOL, (n, rel)


def test_noalloc_rejects_order_above_limit():
    import torch

    # rejected on the host before any launch; the buffers are never touched
    buf = torch.zeros(4, dtype=torch.complex128, device="cuda:0")
    piv = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    rc = engine.lib().pss_lu_factor_noalloc(8193, ctypes.c_void_p(buf.data_ptr()), 8193,
                                            ctypes.c_void_p(piv.data_ptr()), ctypes.c_void_p(piv.data_ptr()), None)
    assert rc != 0
    assert "exceeds the no-allocation LU limit of 8192" in engine.lib().pss_last_error().decode()

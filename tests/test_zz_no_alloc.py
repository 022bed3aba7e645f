"""pss_lu_factor_noalloc: the FP64 LU for callers that cannot let a library allocate device
memory (a CUDA.jl or PyTorch pool owns the device, or cudaFree's device-wide synchronisation
would stall a latency-sensitive loop).  Its only scratch is a fixed file-scope device array.

Checked through the C ABI, on two factorisations in a row (the second reuses the scratch):
  * the factors, applied on the CPU (LAPACK getrs via scipy), solve the system as the oracle's
    LAPACK LU solve does, and as the allocating entry point pss_lu_solve does: relative
    difference <= 1e-11 on these well-conditioned matrices (both backward-stable FP64 LU
    solves; observed ~1e-14);
  * the device's free memory (cudaMemGetInfo) is the same before and after a warm call;
  * a padded buffer (leading dimension n + 17) gives the same factors and pivots as ld = n;
  * an order above the limit is rejected before anything is launched.
This file is collected last so that, should it fail, every other test has already run.
"""
import ctypes
import os
import sys

import numpy as np
import pytest
import scipy.linalg

from pssfss_b200 import engine

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import oracle  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _system(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3 * np.sqrt(n) * np.eye(n)
    B = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
    return A, B


def _factor_noalloc(A, pad=0):
    """Factor A (row-major, leading dimension n + pad) through the C ABI; the device buffers
    are made before the call, so nothing in the call itself allocates."""
    import torch

    n = A.shape[0]
    host = np.zeros((n, n + pad), np.complex128)
    host[:, :n] = A
    dA = torch.from_numpy(host).to("cuda:0")
    ipiv = torch.full((n,), -1, dtype=torch.int32, device="cuda:0")
    info = torch.full((1,), 7, dtype=torch.int32, device="cuda:0")  # the call must reset it to 0 itself
    stream = torch.cuda.current_stream(0).cuda_stream
    torch.cuda.synchronize(0)
    free0, _ = torch.cuda.mem_get_info(0)
    rc = engine.lib().pss_lu_factor_noalloc(n, ctypes.c_void_p(dA.data_ptr()), n + pad,
                                            ctypes.c_void_p(ipiv.data_ptr()), ctypes.c_void_p(info.data_ptr()),
                                            ctypes.c_void_p(stream))
    assert rc == 0, engine.lib().pss_last_error().decode()
    torch.cuda.synchronize(0)
    free1, _ = torch.cuda.mem_get_info(0)
    LU = dA.cpu().numpy()[:, :n].copy()
    return LU, ipiv.cpu().numpy().astype(np.int64), int(info.cpu().item()), free0 - free1


def test_noalloc_factor_matches_oracle_and_allocating_solve_twice():
    _factor_noalloc(_system(64, 1)[0])  # warm: module loading and the one-time scratch look-up
    for n, seed in ((300, 11), (1100, 12)):
        A, B = _system(n, seed)
        LU, piv, info, used = _factor_noalloc(A)
        assert info == 0
        assert used == 0, f"free device memory changed by {used} bytes across the call"
        assert piv.min() >= 0 and piv.max() < n and np.all(piv >= np.arange(n))
        X_noalloc = scipy.linalg.lu_solve((LU, piv), B)
        X_oracle = oracle.lu_solve(A, B)
        rel = np.max(np.abs(X_noalloc - X_oracle)) / np.max(np.abs(X_oracle))
        assert rel < TOL, ("vs oracle", n, rel)
        X_alloc, st = engine.lu_solve(A, B, "fp64")
        assert st == 0
        rel = np.max(np.abs(X_noalloc - X_alloc)) / np.max(np.abs(X_alloc))
        assert rel < TOL, ("vs pss_lu_solve", n, rel)


def test_noalloc_padded_leading_dimension():
    A, B = _system(517, 21)
    LU0, piv0, info0, _ = _factor_noalloc(A)
    LU1, piv1, info1, used = _factor_noalloc(A, pad=17)
    assert info0 == info1 == 0 and used == 0
    np.testing.assert_array_equal(piv0, piv1)
    np.testing.assert_allclose(LU1, LU0, rtol=0, atol=1e-13 * np.max(np.abs(LU0)))
    X = scipy.linalg.lu_solve((LU1, piv1), B)
    X_oracle = oracle.lu_solve(A, B)
    assert np.max(np.abs(X - X_oracle)) / np.max(np.abs(X_oracle)) < TOL


def test_noalloc_rejects_order_above_limit():
    import torch

    # rejected on the host before any launch; the buffers are never touched
    buf = torch.zeros(4, dtype=torch.complex128, device="cuda:0")
    piv = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    rc = engine.lib().pss_lu_factor_noalloc(8193, ctypes.c_void_p(buf.data_ptr()), 8193,
                                            ctypes.c_void_p(piv.data_ptr()), ctypes.c_void_p(piv.data_ptr()), None)
    assert rc != 0
    assert "exceeds the no-allocation LU limit of 8192" in engine.lib().pss_last_error().decode()

"""bem_dgesv_noalloc: the allocation-free dense solve on caller-owned device buffers.

It serves callers that cannot allocate device memory when they solve (a host that
owns every device buffer through its own pool, a loop that must not pay for the
synchronisation of cudaMalloc/cudaFree, a fixed memory budget).  Its scratch is a
static device array sized for n <= 4096.  This file is collected last on purpose.

The tests call the entry point through the C ABI and check it against the existing
entry point bem_dgesv on the same systems, within the tolerance the other solve tests
use: two calls in a row (different sizes, same shared scratch), a singular system
(info > 0, pivots still 1-based), a call without right-hand sides, and that a call
after the first one leaves the device's free memory unchanged (allocations come in
2 MiB granules, so any cudaMalloc would show).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_colmajor(torch, a):
    """A flat device buffer holding `a` in column-major order (allocated by the test)."""
    return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).cuda()


def _call(L, torch, n, nrhs, dA, dpiv, dB, stream):
    info = ctypes.c_int(-99)
    rc = L.bem_dgesv_noalloc(n, nrhs, dA.data_ptr(), n, dpiv.data_ptr(),
                             dB.data_ptr() if dB is not None else None, n,
                             ctypes.byref(info), ctypes.c_void_p(stream.cuda_stream))
    stream.synchronize()
    return rc, info.value


def test_noalloc_matches_dgesv_on_two_calls():
    import torch

    from bem3d_elastostatic_b200 import _lib
    from bem3d_elastostatic_b200.api import dgesv

    L = _lib.load()
    rng = np.random.default_rng(20261203)
    stream = torch.cuda.current_stream()
    for n, nrhs in ((1000, 2), (517, 1)):
        A = rng.standard_normal((n, n)) + 0.1 * n * np.eye(n)
        B = rng.standard_normal((n, nrhs))
        _, ipiv_ref, X_ref, info_ref = dgesv(A, B)
        assert info_ref == 0

        dA = _device_colmajor(torch, A)
        dB = _device_colmajor(torch, B)
        dpiv = torch.zeros(n, dtype=torch.int32, device="cuda")
        rc, info = _call(L, torch, n, nrhs, dA, dpiv, dB, stream)
        assert rc == 0 and info == 0
        X = dB.cpu().numpy().reshape(nrhs, n).T
        # same tolerance as the other solve tests: normwise backward error 1e-14 ...
        res = np.abs(A @ X - B).max() / (np.abs(A).sum(1).max() * np.abs(X).max())
        assert res < 1e-14
        # ... and agreement with the existing entry point
        assert np.abs(X - X_ref).max() <= 1e-12 * np.abs(X_ref).max()
        assert np.array_equal(dpiv.cpu().numpy(), ipiv_ref)


def test_noalloc_allocates_nothing():
    import torch

    from bem3d_elastostatic_b200 import _lib

    L = _lib.load()
    rng = np.random.default_rng(7)
    stream = torch.cuda.current_stream()
    n, nrhs = 2048, 3
    A = rng.standard_normal((n, n)) + 0.1 * n * np.eye(n)
    B = rng.standard_normal((n, nrhs))
    bufs = []
    for _ in range(2):  # every buffer of both calls exists before the measurement
        bufs.append((_device_colmajor(torch, A), _device_colmajor(torch, B),
                     torch.zeros(n, dtype=torch.int32, device="cuda")))
    torch.cuda.synchronize()
    rc, info = _call(L, torch, n, nrhs, *bufs[0][:1], bufs[0][2], bufs[0][1], stream)
    assert rc == 0 and info == 0  # warm-up: loads the module and its static array
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc, info = _call(L, torch, n, nrhs, *bufs[1][:1], bufs[1][2], bufs[1][1], stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert rc == 0 and info == 0
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    # and the two calls agree bitwise (same inputs, same scratch, deterministic kernels)
    assert torch.equal(bufs[0][1], bufs[1][1])


def test_noalloc_singular_and_no_rhs():
    import torch

    from bem3d_elastostatic_b200 import _lib
    from bem3d_elastostatic_b200.api import dgesv

    L = _lib.load()
    rng = np.random.default_rng(11)
    stream = torch.cuda.current_stream()
    n = 300
    A = rng.standard_normal((n, n)) + 0.1 * n * np.eye(n)
    A[:, 17] = 0.0  # a zero column: exactly singular, the LU meets an exact zero pivot
    B = rng.standard_normal((n, 1))
    _, ipiv_ref, _, info_ref = dgesv(A, B)
    assert info_ref > 0
    dA, dB = _device_colmajor(torch, A), _device_colmajor(torch, B)
    dpiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    rc, info = _call(L, torch, n, 1, dA, dpiv, dB, stream)
    assert rc == info == info_ref
    assert np.array_equal(dpiv.cpu().numpy(), ipiv_ref)  # 1-based, as bem_dgesv's

    # no right-hand side: factors and pivots only
    A = rng.standard_normal((n, n)) + 0.1 * n * np.eye(n)
    _, ipiv_ref, _, info_ref = dgesv(A, np.zeros((n, 0)))
    dA = _device_colmajor(torch, A)
    rc, info = _call(L, torch, n, 0, dA, dpiv, None, stream)
    assert rc == 0 and info == 0 == info_ref
    assert np.array_equal(dpiv.cpu().numpy(), ipiv_ref)


def test_noalloc_rejects_orders_above_its_limit():
    from bem3d_elastostatic_b200 import _lib

    L = _lib.load()
    info = ctypes.c_int(0)
    n = _lib.NOALLOC_MAX_N + 1
    # the size check comes first: no buffer is touched
    rc = L.bem_dgesv_noalloc(n, 1, None, n, None, None, n, ctypes.byref(info), None)
    assert rc == _lib.BEM_ERR_TOO_LARGE

"""bem_dgesv_noalloc: the allocation-free dense solve on caller-owned device buffers.

It serves callers that cannot allocate device memory when they solve (a host that
owns every device buffer through its own pool, a loop that must not pay for the
synchronisation of cudaMalloc/cudaFree, a fixed memory budget).  Its scratch is a
static device array sized for n <= 4096.  This file is collected last on purpose.

The test calls the entry point through the C ABI twice in a row (different sizes,
same shared scratch) and checks each result against the existing entry point
bem_dgesv on the same system, within the tolerance the other solve tests use.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_colmajor(torch, a):
    """A flat device buffer holding `a` in column-major order (allocated by the test)."""
    return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).cuda()


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
        info = ctypes.c_int(-99)
        rc = L.bem_dgesv_noalloc(n, nrhs, dA.data_ptr(), n, dpiv.data_ptr(), dB.data_ptr(), n,
                                 ctypes.byref(info), ctypes.c_void_p(stream.cuda_stream))
        stream.synchronize()
        assert rc == 0 and info.value == 0
        X = dB.cpu().numpy().reshape(nrhs, n).T
        # same tolerance as the other solve tests: normwise backward error 1e-14 ...
        res = np.abs(A @ X - B).max() / (np.abs(A).sum(1).max() * np.abs(X).max())
        assert res < 1e-14
        # ... and agreement with the existing entry point
        assert np.abs(X - X_ref).max() <= 1e-12 * np.abs(X_ref).max()
        assert np.array_equal(dpiv.cpu().numpy(), ipiv_ref)


def test_noalloc_rejects_orders_above_its_limit():
    from bem3d_elastostatic_b200 import _lib

    L = _lib.load()
    info = ctypes.c_int(0)
    n = _lib.NOALLOC_MAX_N + 1
    # the size check comes first: no buffer is touched
    rc = L.bem_dgesv_noalloc(n, 1, None, n, None, None, n, ctypes.byref(info), None)
    assert rc == _lib.BEM_ERR_TOO_LARGE

"""lu2gpu_lusolve_noalloc: the solve for callers that cannot allocate device
memory when they solve (device memory owned by another allocator or a fixed
budget, or no tolerance for the device-wide synchronization of cudaMalloc /
cudaFree).  Its scratch is a fixed device array inside the library.

Checked through the C ABI against the regular entry point lu2gpu_lusolve on
two calls in a row (the second call finds the first call's leftovers in the
shared array): identical pivots and x within the parity tolerance of the
other GPU tests; no device memory taken by the second call; sizes beyond the
array's limits are refused.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

import lu2_b200 as L

pytestmark = pytest.mark.gpu

XTOL = 1e-12  # the partial-pivoting x bar of tests/test_gpu_lu.py


def _matrix(ctx, n, nrhs, seed):
    import torch

    ld = L.device_ld(n, nrhs)
    a = torch.zeros((n, ld), dtype=torch.float64, device="cuda")
    ctx.generate(a, n, ld, seed, nrhs)
    return a, ld


def test_noalloc_matches_lusolve_on_two_calls():
    import torch

    lib = L.load()
    torch.cuda.set_device(0)
    ctx = L.Context(0)
    stream = torch.cuda.current_stream()
    n, nb, nrhs = 1000, 64, 3
    a_ref, ld = _matrix(ctx, n, nrhs, 1)
    a_na = torch.empty_like(a_ref)
    piv_ref = torch.zeros(n, dtype=torch.int32, device="cuda")
    piv_na = torch.zeros(n, dtype=torch.int32, device="cuda")
    free_after = []
    for call, seed in enumerate((1, 12345)):
        ctx.generate(a_ref, n, ld, seed, nrhs)
        a_na.copy_(a_ref)
        piv_na.fill_(-1)
        torch.cuda.synchronize()
        assert ctx.lusolve(a_ref, n, ld, nb, nrhs, L.PIVOT_PARTIAL, piv_ref) == 0
        rc = lib.lu2gpu_lusolve_noalloc(n, nrhs, a_na.data_ptr(), ld, nb, L.PIVOT_PARTIAL, piv_na.data_ptr(),
                                        ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L._lib.last_error()
        torch.cuda.synchronize()
        free_after.append(torch.cuda.mem_get_info()[0])
        np.testing.assert_array_equal(piv_na.cpu().numpy(), piv_ref.cpu().numpy())
        x_ref = a_ref[:, n:n + nrhs].cpu().numpy()
        x_na = a_na[:, n:n + nrhs].cpu().numpy()
        assert np.abs(x_na - x_ref).max() / np.abs(x_ref).max() < XTOL, call
    assert free_after[1] == free_after[0]
    ctx.close()


def test_noalloc_at_its_limits_without_pivot_output():
    """n = 2048, nrhs = 16, nb = 128 (every limit at once) with ipiv = NULL, so
    the pivots also live in the fixed array."""
    import torch

    lib = L.load()
    torch.cuda.set_device(0)
    ctx = L.Context(0)
    stream = torch.cuda.current_stream()
    n, nb, nrhs = 2048, 128, 16
    a_ref, ld = _matrix(ctx, n, nrhs, 7)
    a_na = a_ref.clone()
    torch.cuda.synchronize()
    assert ctx.lusolve(a_ref, n, ld, nb, nrhs, L.PIVOT_PARTIAL) == 0
    rc = lib.lu2gpu_lusolve_noalloc(n, nrhs, a_na.data_ptr(), ld, nb, L.PIVOT_PARTIAL, None,
                                    ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, L._lib.last_error()
    torch.cuda.synchronize()
    x_ref = a_ref[:, n:n + nrhs].cpu().numpy()
    x_na = a_na[:, n:n + nrhs].cpu().numpy()
    assert np.abs(x_na - x_ref).max() / np.abs(x_ref).max() < XTOL
    ctx.close()


def test_noalloc_refuses_sizes_beyond_its_array():
    import torch

    lib = L.load()
    n = 4096
    a = torch.zeros((n, n + 16), dtype=torch.float64, device="cuda")
    rc = lib.lu2gpu_lusolve_noalloc(n, 1, a.data_ptr(), n + 16, 64, L.PIVOT_PARTIAL, None, None)
    assert rc == -1
    assert "n <= 2048" in L._lib.last_error()
    rc = lib.lu2gpu_lusolve_noalloc(256, 1, a.data_ptr(), n + 16, 256, L.PIVOT_PARTIAL, None, None)
    assert rc == -1

"""Edge cases of the device path: empty and degenerate systems, exact zeros,
NaN input (the pivot search must finish and report, not hang), identity
matrices, and a NaN system inside a batch leaving the others untouched."""
import numpy as np
import pytest

import lu2_b200 as L

pytestmark = pytest.mark.gpu


def _dev(n, ld, fill=0.0):
    import torch

    return torch.full((n, ld), fill, dtype=torch.float64, device="cuda")


def test_empty_system_is_an_argument_error(ctx):
    import torch

    a = torch.zeros((1, 32), dtype=torch.float64, device="cuda")
    with pytest.raises(L.Lu2GpuError):
        ctx.lusolve(a, 0, 32, 16)


def test_all_zero_matrix_reports_first_column(ctx):
    n = 300
    ld = L.device_ld(n)
    a = _dev(n, ld)
    assert ctx.lusolve(a, n, ld, 64) == 1  # zero pivot at column 0


@pytest.mark.parametrize("n", [1, 64, 1000])
def test_identity_solves_exactly(ctx, n):
    import torch

    ld = L.device_ld(n)
    a = _dev(n, ld)
    a[:, :n] = torch.eye(n, dtype=torch.float64, device="cuda")
    b = torch.arange(1, n + 1, dtype=torch.float64, device="cuda") * 0.5
    a[:, n] = b
    assert ctx.lusolve(a, n, ld, 16) == 0
    assert torch.equal(a[:, n], b)
    assert np.array_equal(ctx.pivots(n), np.arange(n))


def test_singular_matrix_reports_zero_pivot(ctx, oracle):
    """A zero column stays exactly zero through every update (its U entries
    are 0 * 1/pivot), so the factorization meets an exact zero pivot there,
    reports it LAPACK-style (column + 1) and completes.  (Two equal rows
    would only leave rounding-level values, not an exact zero, as in LAPACK.)"""
    import torch

    n = 200
    ld = L.device_ld(n)
    a = torch.from_numpy(oracle.randomsetmat(n, 3, lda=ld)).cuda()
    a[:, 150] = 0.0
    assert ctx.lusolve(a, n, ld, 64) == 151


def test_nan_entry_finishes_without_hanging(ctx, oracle):
    """A NaN makes every later pivot candidate non-comparable; the leaf keeps
    row c as the pivot row and the factorization runs to completion."""
    import torch

    n = 512
    ld = L.device_ld(n)
    a = torch.from_numpy(oracle.randomsetmat(n, 4, lda=ld)).cuda()
    a[7, 3] = float("nan")
    info = ctx.lusolve(a, n, ld, 64)
    assert info >= 0
    assert torch.isnan(a[:, n]).any()


def test_nan_system_in_batch_leaves_others_exact(ctx):
    """Systems are independent: a NaN in one system changes nothing in the
    others (bit-identical to a batch without it)."""
    import ctypes
    import glob

    n = np.array([40, 300, 100, 300], dtype=np.int32)
    cudart = ctypes.CDLL(sorted(glob.glob("/usr/local/cuda/lib64/libcudart.so*"))[0])

    def run(poison):
        b = L.Batch(ctx, n)
        b.generate(50)
        if poison:
            ptr, ld = b.system(1)
            host = np.zeros((300, ld))
            assert cudart.cudaDeviceSynchronize() == 0
            assert cudart.cudaMemcpy(ctypes.c_void_p(host.ctypes.data), ctypes.c_void_p(ptr),
                                     ctypes.c_size_t(host.nbytes), 2) == 0
            host[10, 10] = np.nan
            assert cudart.cudaMemcpy(ctypes.c_void_p(ptr), ctypes.c_void_p(host.ctypes.data),
                                     ctypes.c_size_t(host.nbytes), 1) == 0
        b.solve()
        assert cudart.cudaDeviceSynchronize() == 0
        out = []
        for i in range(4):
            ptr, ld = b.system(i)
            h = np.zeros((int(n[i]), ld))
            assert cudart.cudaMemcpy(ctypes.c_void_p(h.ctypes.data), ctypes.c_void_p(ptr),
                                     ctypes.c_size_t(h.nbytes), 2) == 0
            out.append(h[:, int(n[i])].copy())
        b.close()
        return out

    clean, poisoned = run(False), run(True)
    for i in (0, 2, 3):
        assert np.array_equal(clean[i], poisoned[i])
    assert np.isnan(poisoned[1]).any()

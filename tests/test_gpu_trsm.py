"""The block-row solve of lu2's right part (solve_triangle, lu2.c:485-521:
U12 = L11^{-1} A12) through lu2gpu_solve_triangle_dev, against
scipy.linalg.solve_triangular in FP64 on the unit lower triangles of real LU
panels (partial pivoting: |l| <= 1).  Both the tensor-pipe path (K a
multiple of 16 up to 256, aligned) and the CUDA-core path (other K, odd
strides) are covered; the transposed, negated copy -U12^T is checked bit for
bit against the solved block."""
import numpy as np
import pytest

import lu2_b200 as L

pytestmark = pytest.mark.gpu


def unit_lower(K, seed):
    import scipy.linalg as sl

    rng = np.random.default_rng(seed)
    _, lo, _ = sl.lu(rng.uniform(-0.5, 0.5, (K, K)))
    return lo


@pytest.mark.parametrize("K,ncols,ldx_pad", [(256, 1000, 16), (256, 64, 0), (256, 7, 1), (128, 300, 4), (16, 33, 2),
                                             (240, 129, 0), (48, 5000, 8), (200, 100, 0), (512, 70, 6), (256, 1, 0)])
def test_solve_triangle_matches_scipy(ctx, parity, K, ncols, ldx_pad):
    import scipy.linalg as sl
    import torch

    lo = unit_lower(K, K + ncols)
    rng = np.random.default_rng(ncols)
    x0 = rng.uniform(-1, 1, (K, ncols))
    want = sl.solve_triangular(lo, x0, lower=True, unit_diagonal=True)
    ldt = K + 2
    t = np.zeros((K, ldt))
    t[:, :K] = np.tril(lo, -1) + np.triu(rng.uniform(5, 9, (K, K)))  # the upper part must not be read
    ldx = ncols + ldx_pad
    x = np.zeros((K, ldx))
    x[:, :ncols] = x0
    td = torch.tensor(t, device="cuda")
    xd = torch.tensor(x, device="cuda")
    bt = torch.full((ncols, K), np.nan, dtype=torch.float64, device="cuda")
    ctx.solve_triangle(K, td, ldt, xd, ldx, ncols, bt)
    got = xd.cpu().numpy()
    err = np.abs(got[:, :ncols] - want).max() / np.abs(want).max()
    parity("solve_triangle K=%d ncols=%d ldx=%d" % (K, ncols, ldx), err, 1e-13)
    np.testing.assert_array_equal(got[:, ncols:], x[:, ncols:])  # padding untouched
    np.testing.assert_array_equal(bt.cpu().numpy(), -got[:, :ncols].T)

"""backward_sub (lu2.c:110-116: x_j = y_j - sum_{k>j} U'_jk x_k, U' unit
upper) through lu2gpu_backsolve, against scipy.linalg.solve_triangular in
FP64.  Orders from 4096 up take the persistent single-launch path (64-row
blocks published in order), smaller ones the blocked launches; covered: a
partial last block, 1 to 11 right-hand sides (two passes past 8), an odd
right-hand-side stride, and the diagonal and lower part never read."""
import numpy as np
import pytest

import lu2_b200 as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,nrhs,ldx_pad", [(4096, 1, 0), (5000, 3, 1), (8192, 8, 0), (4160, 11, 2), (1000, 2, 0),
                                            (64, 1, 0), (4097, 1, 0)])
def test_backsolve_matches_scipy(ctx, parity, n, nrhs, ldx_pad):
    import scipy.linalg as sl
    import torch

    rng = np.random.default_rng(n + nrhs)
    ld = n + 6
    a = np.zeros((n, ld))
    a[:, :n] = np.triu(rng.uniform(-1, 1, (n, n)) / np.sqrt(n), 1)
    a[np.arange(n), np.arange(n)] = 7.0                     # must not be read (unit diagonal)
    a[:, :n] += np.tril(rng.uniform(3, 4, (n, n)), -1)       # must not be read
    y = rng.uniform(-1, 1, (n, nrhs))
    u = np.triu(a[:, :n], 1) + np.eye(n)
    want = sl.solve_triangular(u, y, lower=False, unit_diagonal=True)
    ldx = nrhs + ldx_pad
    x = np.zeros((n, ldx))
    x[:, :nrhs] = y
    ad = torch.tensor(a, device="cuda")
    xd = torch.tensor(x, device="cuda")
    ctx.backsolve(ad, n, ld, xd, ldx, nrhs)
    got = xd.cpu().numpy()
    err = np.abs(got[:, :nrhs] - want).max() / np.abs(want).max()
    parity("backsolve n=%d nrhs=%d ldx=%d" % (n, nrhs, ldx), err, 1e-13)
    np.testing.assert_array_equal(got[:, nrhs:], x[:, nrhs:])

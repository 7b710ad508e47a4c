"""Failure detection without a GPU fault: the panel leaf's cross-CTA waits
are bounded.  Through the test hook lu2gpu_test_leaf_withhold one leaf CTA
skips its publications and the waits give up after 50 ms; the factorization
reports LU2GPU_ERR_TIMEOUT (the kernels after the failed leaf skip work that
depends on the pivots it never wrote), and the same context then solves
normally."""
import numpy as np
import pytest

import lu2_b200 as L

pytestmark = pytest.mark.gpu


def test_leaf_wait_gives_up_and_context_recovers(oracle):
    import torch

    n, nb, seed = 1024, 64, 1
    ctx = L.Context(0)
    try:
        ld = L.device_ld(n)
        a = torch.zeros((n, ld), dtype=torch.float64, device="cuda")
        ctx.generate(a, n, ld, seed)
        ctx.test_leaf_withhold(1, 50.0)  # 1024 rows: the first leaf runs on 8 CTAs
        with pytest.raises(L.Lu2GpuError) as e:
            ctx.lusolve(a, n, ld, nb, 1, L.PIVOT_PARTIAL)
        assert e.value.rc == -4, e.value
        assert "gave up" in str(e.value)
        ctx.test_leaf_withhold(-1, 0.0)
        ctx.generate(a, n, ld, seed)
        assert ctx.lusolve(a, n, ld, nb, 1, L.PIVOT_PARTIAL) == 0
        xo, po = oracle.solve(n, nb, seed)
        np.testing.assert_array_equal(ctx.pivots(n), po)
        x = a[:, n].cpu().numpy()
        assert np.abs(x - xo).max() / np.abs(xo).max() < 1e-11
    finally:
        ctx.close()


def test_withhold_hook_rejects_bad_limits():
    ctx = L.Context(0)
    try:
        with pytest.raises(L.Lu2GpuError):
            ctx.test_leaf_withhold(0, 5000.0)
        with pytest.raises(L.Lu2GpuError):
            ctx.test_leaf_withhold(0, -1.0)
    finally:
        ctx.close()

"""The row exchange of a panel's pivots (lu2.c:251-291,
swaprows_simple_with_scale, applied per panel as lu2.c:541-554 does)
through lu2gpu_swaprows_dev, against the sequential exchanges restated in
numpy: bit-exact (every element is copied once and pivot rows are multiplied
once by the same 1/pivot).  Cases: repeated pivot rows, pivots inside the
panel, no-op pivots, the widest panel (512 pivots), ragged and unaligned
column ranges (scalar path), and refused out-of-range pivots."""
import numpy as np
import pytest

import lu2_b200 as L

pytestmark = pytest.mark.gpu


def swaps_restated(a, k0, k1, piv, dinv, cs, ce):
    """lu2.c:251-291 for k = k0..k1-1: exchange rows k and piv[k] over
    columns cs..ce-1, then scale row k by dinv[k]."""
    a = a.copy()
    for k in range(k0, k1):
        p = int(piv[k])
        if p != k:
            tmp = a[k, cs:ce].copy()
            a[k, cs:ce] = a[p, cs:ce]
            a[p, cs:ce] = tmp
        if dinv is not None:
            a[k, cs:ce] *= dinv[k]
    return a


def pivots(rng, n, k0, k1, style):
    piv = np.zeros(n, dtype=np.int32)
    for k in range(k0, k1):
        if style == "far":
            piv[k] = rng.integers(k, n)
        elif style == "near":
            piv[k] = rng.integers(k, min(n, k + 4))
        elif style == "repeat":  # a handful of rows named again and again
            cand = [x for x in (n - 1, n - 2, k, (k + n) // 2) if x >= k]
            piv[k] = rng.choice(cand)
        else:  # identity
            piv[k] = k
    return piv


@pytest.mark.parametrize("n,ld,k0,k1,cs,ce,style", [
    (600, 640, 0, 256, 256, 601, "far"),
    (600, 640, 64, 128, 0, 64, "near"),
    (1000, 1024, 16, 528, 528, 1000, "far"),   # the widest panel: 512 pivots
    (300, 320, 10, 40, 40, 301, "repeat"),
    (300, 320, 0, 32, 32, 300, "identity"),
    (257, 300, 1, 17, 3, 270, "far"),          # odd column start: scalar path
    (400, 403, 100, 116, 0, 403, "near"),      # odd row stride: scalar path
    (5000, 5016, 0, 256, 256, 5001, "repeat"),
])
def test_swaprows_matches_sequential_exchanges(ctx, n, ld, k0, k1, cs, ce, style):
    import torch

    rng = np.random.default_rng(n + k0 + ce)
    a0 = rng.uniform(-1, 1, (n, ld))
    piv = pivots(rng, n, k0, k1, style)
    dinv = rng.uniform(0.5, 2.0, n)
    want = swaps_restated(a0, k0, k1, piv, dinv, cs, ce)
    a = torch.tensor(a0, device="cuda")
    ctx.swaprows(a, n, ld, k0, k1, torch.tensor(piv, device="cuda"), torch.tensor(dinv, device="cuda"), cs, ce)
    np.testing.assert_array_equal(a.cpu().numpy(), want)
    # without scaling
    a = torch.tensor(a0, device="cuda")
    ctx.swaprows(a, n, ld, k0, k1, torch.tensor(piv, device="cuda"), None, cs, ce)
    np.testing.assert_array_equal(a.cpu().numpy(), swaps_restated(a0, k0, k1, piv, None, cs, ce))


@pytest.mark.parametrize("bad", [-1, 5, 700])
def test_swaprows_refuses_out_of_range_pivots(ctx, bad):
    """A pivot below its own row or beyond the last row is refused on the
    device before anything moves (the matrix is unchanged)."""
    import torch

    n, ld = 600, 640
    rng = np.random.default_rng(1)
    a0 = rng.uniform(-1, 1, (n, ld))
    piv = pivots(rng, n, 0, 64, "far")
    piv[40] = bad  # below its own row (-1, 5) or past the last row (700)
    a = torch.tensor(a0, device="cuda")
    with pytest.raises(L.Lu2GpuError) as e:
        ctx.swaprows(a, n, ld, 0, 64, torch.tensor(piv, device="cuda"), None, 64, n)
    assert e.value.rc == -1
    np.testing.assert_array_equal(a.cpu().numpy(), a0)
    # the context is still usable
    piv[40] = 40
    ctx.swaprows(a, n, ld, 0, 64, torch.tensor(piv, device="cuda"), None, 64, n)
    np.testing.assert_array_equal(a.cpu().numpy(), swaps_restated(a0, 0, 64, piv, None, 64, n))

"""The composition rule the row-exchange kernel (kernels_panel.cu,
laswp_scale_kernel) uses to turn a panel's exchanges into one gather/scatter,
restated in Python and checked against the exchanges applied one by one
(lu2.c:251-291 in the order lu2.c:541-554 applies them).

For exchanges k <-> p_k, k = k0..k1-1 in order (p_k >= k):
  A(k): the original row at position k just before step k -- A(i) for the
        latest i < k with p_i = k, else k (chains resolved by pointer jumping);
  row k finally holds A(k) if p_k = k, else A(j) for the latest j < k with
        p_j = p_k, else the original row p_k;
  row q >= k1 finally holds A(j) for the last j with p_j = q."""
import numpy as np
import pytest


def plan(P, k0, k1):
    npiv = k1 - k0
    A = [-1] * npiv
    for i in range(npiv):
        q = P[i]
        if q != k0 + i and q < k1:
            A[q - k0] = max(A[q - k0], i)
    A = [(-(k0 + t) - 1 if A[t] < 0 else A[t]) for t in range(npiv)]
    span = 1
    while span < npiv:  # the kernel's ceil(log2 npiv) double-buffered rounds
        A = [(A[A[t]] if A[t] >= 0 else A[t]) for t in range(npiv)]
        span <<= 1
    assert all(v < 0 for v in A)
    slots = []
    for t in range(npiv):
        p, k = P[t], k0 + t
        if p == k:
            s = -A[t] - 1
        else:
            earlier = [j for j in range(t) if P[j] == p]
            s = -A[earlier[-1]] - 1 if earlier else p
            if p >= k1 and not any(P[q] == p for q in range(t + 1, npiv)):
                slots.append((-A[t] - 1, p))
        slots.append((s, k))
    return slots


@pytest.mark.parametrize("style", ["far", "mixed", "near"])
def test_plan_equals_sequential_exchanges(style):
    rng = np.random.default_rng({"far": 0, "mixed": 1, "near": 2}[style])
    for _ in range(1500):
        n = int(rng.integers(2, 60))
        k0 = int(rng.integers(0, n - 1))
        k1 = int(rng.integers(k0 + 1, n + 1))
        P = []
        for k in range(k0, k1):
            if style == "far":
                p = int(rng.integers(k, n))
            elif style == "mixed":
                p = int(rng.choice([k, min(n - 1, k + 1), n - 1, int(rng.integers(k, n))]))
            else:
                p = int(rng.integers(k, min(n, k + 3)))
            P.append(p)
        rows = list(range(n))
        for t, p in enumerate(P):
            k = k0 + t
            rows[k], rows[p] = rows[p], rows[k]
        sl = plan(P, k0, k1)
        dst = [d for _, d in sl]
        assert len(set(dst)) == len(dst) and len(sl) <= 2 * (k1 - k0)
        out = list(range(n))
        for s, d in sl:
            out[d] = s
        assert out == rows

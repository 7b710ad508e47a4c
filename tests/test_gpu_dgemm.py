"""The DGEMM offload entry points (mydgemm, gdr_dgemm_, gdrblas_dgemm,
mygdrdgemm, matmul_for_small_nk, gdr_check_and_restart) on the FP64 tensor-core
kernel, against numpy float64.  Tolerance: |C - C_ref| <= 8 k eps |A||B| + eps|C|
elementwise (different summation order)."""
import numpy as np
import pytest

import lu2_b200 as L

pytestmark = pytest.mark.gpu
EPS = 2.0**-52


def bound(a, b, k, c):
    return 8 * max(k, 1) * EPS * (np.abs(a) @ np.abs(b)) + 4 * EPS * np.abs(c) + 1e-300


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (37, 53, 19), (128, 128, 256), (300, 129, 64), (513, 65, 48),
                                   (64, 700, 33), (5, 3, 0)])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.0, 1.0), (0.5, -2.0)])
def test_mydgemm(m, n, k, alpha, beta):
    rng = np.random.default_rng(m * 1000 + n + k)
    na, nb, nc = k + 3, n + 1, n + 5
    a = rng.uniform(-1, 1, (m, na))
    b = rng.uniform(-1, 1, (max(k, 1), nb))
    c = rng.uniform(-1, 1, (m, nc))
    if beta == 0.0:
        c[:, :n] = np.nan  # must not be read
    ref = alpha * a[:, :k] @ b[:k, :n] + (beta * c[:, :n] if beta != 0 else 0)
    cc = c.copy()
    L.mydgemm(m, n, k, alpha, a, na, b, nb, beta, cc, nc)
    assert np.all(np.abs(cc[:, :n] - ref) <= bound(a[:, :k], b[:k, :n], k, ref))
    assert np.array_equal(cc[:, n:], c[:, n:])  # untouched outside C


@pytest.mark.parametrize("nota,notb", [(1, 1), (0, 1), (1, 0), (0, 0)])
def test_gdr_dgemm_colmajor(nota, notb):
    rng = np.random.default_rng(7 + 2 * nota + notb)
    m, n, k = 97, 75, 50
    lda, ldb, ldc = (m if nota else k) + 2, (k if notb else n) + 1, m + 3
    A = np.asfortranarray(rng.uniform(-1, 1, (lda, k if nota else m)))
    B = np.asfortranarray(rng.uniform(-1, 1, (ldb, n if notb else k)))
    Cm = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)))
    opA = A[:m, :k] if nota else A[:k, :m].T
    opB = B[:k, :n] if notb else B[:n, :k].T
    ref = 1.5 * opA @ opB - 0.25 * Cm[:m, :n]
    Cg = Cm.copy(order="F")
    done = L.gdr_dgemm_(nota, notb, m, n, k, 1.5, -0.25, lda, ldb, ldc, A, B, Cg)
    assert done == 1
    assert np.all(np.abs(Cg[:m, :n] - ref) <= bound(opA, opB, k, ref))


@pytest.mark.parametrize("order", [L.CBLAS_ROWMAJOR, L.CBLAS_COLMAJOR])
@pytest.mark.parametrize("ta,tb", [(L.CBLAS_NOTRANS, L.CBLAS_NOTRANS), (L.CBLAS_TRANS, L.CBLAS_NOTRANS),
                                   (L.CBLAS_NOTRANS, L.CBLAS_TRANS)])
def test_gdrblas_dgemm(order, ta, tb):
    rng = np.random.default_rng(11)
    M, N, K = 70, 45, 33
    opA = rng.uniform(-1, 1, (M, K))
    opB = rng.uniform(-1, 1, (K, N))
    C0 = rng.uniform(-1, 1, (M, N))
    # store each operand so that op(X) is the matrix above, in the requested order
    def store(mat, trans):
        s = mat.T if trans == L.CBLAS_TRANS else mat
        s = np.ascontiguousarray(s) if order == L.CBLAS_ROWMAJOR else np.asfortranarray(s)
        ld = s.shape[1] if order == L.CBLAS_ROWMAJOR else s.shape[0]
        return s, ld
    A, lda = store(opA, ta)
    B, ldb = store(opB, tb)
    Cm, ldc = store(C0, L.CBLAS_NOTRANS)
    Cm = Cm.copy(order="C" if order == L.CBLAS_ROWMAJOR else "F")
    L.gdrblas_dgemm(order, ta, tb, M, N, K, -1.0, A, lda, B, ldb, 1.0, Cm, ldc)
    ref = C0 - opA @ opB
    assert np.all(np.abs(np.asarray(Cm) - ref) <= bound(opA, opB, K, ref))


def test_mygdrdgemm_and_small_nk():
    rng = np.random.default_rng(3)
    m, n, k = 200, 13, 16
    a = rng.uniform(-1, 1, (m, k))
    b = rng.uniform(-1, 1, (k, n))
    c = rng.uniform(-1, 1, (m, n))
    c1 = c.copy()
    L.mygdrdgemm(m, n, k, -1.0, a, k, b, n, 1.0, c1, n)
    c2 = c.copy()
    L.load().matmul_for_small_nk(k, a.ctypes.data, n, b.ctypes.data, n, c2.ctypes.data, m, k, n)
    ref = c - a @ b
    assert np.all(np.abs(c1 - ref) <= bound(a, b, k, ref))
    assert np.array_equal(c1, c2)


def test_gdr_check_and_restart_selftest():
    N = 2048
    a = np.zeros((N, N))
    b = np.zeros((N, N))
    c = np.zeros((N, N))
    L.load().gdr_check_and_restart(a.ctypes.data, b.ctypes.data, c.ctypes.data)
    assert np.array_equal(c, b)
    assert b[5, 7] == 5 * N + 7


def test_device_dgemm(ctx):
    import torch

    m, n, k = 260, 190, 80
    g = torch.Generator(device="cuda").manual_seed(0)
    a = torch.rand((m, k), dtype=torch.float64, device="cuda", generator=g) - 0.5
    b = torch.rand((k, n), dtype=torch.float64, device="cuda", generator=g) - 0.5
    c = torch.rand((m, n), dtype=torch.float64, device="cuda", generator=g) - 0.5
    ref = (2.0 * (a @ b) + c).cpu().numpy()
    ctx.dgemm(m, n, k, 2.0, a, k, b, n, 1.0, c, n)
    an, bn = a.cpu().numpy(), b.cpu().numpy()
    assert np.all(np.abs(c.cpu().numpy() - ref) <= 2 * bound(an, bn, k, ref))


def _pinned_like(x):
    """a pinned-host numpy array with x's contents and memory order"""
    import torch

    t = torch.empty(x.size, dtype=torch.float64, pin_memory=True)
    order = "F" if (x.flags.f_contiguous and not x.flags.c_contiguous) else "C"
    out = t.numpy().reshape(x.shape, order=order)
    out[...] = x
    return out, t


@pytest.mark.parametrize("nota,notb", [(1, 1), (0, 1), (1, 0), (0, 0)])
def test_gdr_dgemm_pinned_overlap_is_bit_identical(nota, notb):
    """C in pinned host memory takes the overlapped path (blocks of C's
    columns copied in, multiplied and copied out on three streams); it gives
    the one-pass (pageable) path's result bit for bit."""
    rng = np.random.default_rng(31 + 2 * nota + notb)
    m, n, k = 2048, 2600, 96  # ~16 MB blocks of 1024 columns: 3 blocks, the last ragged
    lda, ldb, ldc = (m if nota else k) + 2, (k if notb else n) + 1, m + 3
    A = np.asfortranarray(rng.uniform(-1, 1, (lda, k if nota else m)))
    B = np.asfortranarray(rng.uniform(-1, 1, (ldb, n if notb else k)))
    C0 = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)))
    Cpg = C0.copy(order="F")
    assert L.gdr_dgemm_(nota, notb, m, n, k, 1.5, -0.25, lda, ldb, ldc, A, B, Cpg) == 1
    Cpin, keep = _pinned_like(C0)
    assert Cpin.flags.f_contiguous
    assert L.gdr_dgemm_(nota, notb, m, n, k, 1.5, -0.25, lda, ldb, ldc, A, B, Cpin) == 1
    assert np.array_equal(Cpin, Cpg)
    opA = A[:m, :k] if nota else A[:k, :m].T
    opB = B[:k, :n] if notb else B[:n, :k].T
    ref = 1.5 * opA @ opB - 0.25 * C0[:m, :n]
    assert np.all(np.abs(Cpin[:m, :n] - ref) <= bound(opA, opB, k, ref))


def test_mydgemm_pinned_overlap_lu2_shape():
    """lu2's trailing update through mydgemm (C -= L21 U12, row-major, k = nb)
    on pinned host buffers: overlapped, bit-identical to the pageable call,
    and beta = 0 never reads C."""
    rng = np.random.default_rng(5)
    m, n, k = 3000, 2100, 256
    na, nb, nc = k + 16, n + 16, n + 16
    a = rng.uniform(-1, 1, (m, na))
    b = rng.uniform(-1, 1, (k, nb))
    c0 = rng.uniform(-1, 1, (m, nc))
    cpg = c0.copy()
    L.mydgemm(m, n, k, -1.0, a, na, b, nb, 1.0, cpg, nc)
    cpin, keep = _pinned_like(c0)
    L.mydgemm(m, n, k, -1.0, a, na, b, nb, 1.0, cpin, nc)
    assert np.array_equal(cpin, cpg)
    cpin[:, :n] = np.nan
    L.mydgemm(m, n, k, 1.0, a, na, b, nb, 0.0, cpin, nc)
    ref = a[:, :k] @ b[:, :n]
    assert np.all(np.abs(cpin[:, :n] - ref) <= bound(a[:, :k], b[:, :n], k, ref))
    assert np.array_equal(cpin[:, n:], c0[:, n:])

"""Parity of the CUDA LU path (through the C ABI) with the oracle and with the
reference's own results (golden vectors, and the compiled reference at
n = 8192).

Bars.  Pivots: equal index for index.  x, relative in the max norm:

* partial pivoting against the fixed reference: XTOL_PARTIAL = 1e-12, the
  agreement asked of the path on well-conditioned inputs.  It holds outright
  on the diagonally dominant systems.  On lu2's uniform random matrices two
  correct FP64 LUs already differ by more at n = 2048 (cond ~ 4e5; the fixed
  reference and LAPACK differ by up to 1.3e-12), so there the bar is
  max(XTOL_PARTIAL, REF_FACTOR d_ref), d_ref being the reference's own
  forward error against the extended-precision solution.  Forward errors of
  correct FP64 LUs of one system scatter by up to about 3x either way
  (LAPACK 0.45-1x the fixed reference's; this repository's C restatement up
  to 2.96x), and a solver whose forward error is at most 3 d_ref lies within
  4 d_ref of the reference (triangle inequality).
* the bug-compatible mode against the shipped reference: REF_FACTOR d_ref as
  well.  That algorithm's poor pivots make its rounding error large
  (1e-12 .. 1e-8), and two evaluation orders differ by about that error.

The GPU's own forward error is reported beside each case.  HPL scaled
residual < 16 in partial-pivoting mode."""
import numpy as np
import pytest

from lu2_b200 import PIVOT_PARTIAL, PIVOT_REF, device_ld, lumcolumn, rdim
from oracle.oracle import RefLib

pytestmark = pytest.mark.gpu

XTOL_PARTIAL = 1e-12
REF_FACTOR = 4.0
GOLDEN_CASES = [(128, 64, 1), (256, 64, 12345), (512, 128, 12345), (1024, 256, 1), (2048, 64, 1),
                (2048, 128, 12345), (2048, 256, 1)]
DD_CASES = [(1024, 64, 1), (2048, 256, 12345), (4096, 256, 1)]


def rel(x, y):
    return float(np.abs(x - y).max() / np.abs(y).max())


def x_bar(mode, d_ref):
    """The bar for x against the reference variant matching `mode`, whose
    forward error is d_ref."""
    return max(XTOL_PARTIAL, REF_FACTOR * d_ref) if mode == PIVOT_PARTIAL else REF_FACTOR * d_ref


def dev_matrix(ctx, n, seed, nrhs=1, kind=0):
    import torch

    ld = device_ld(n, nrhs)
    a = torch.zeros((n, ld), dtype=torch.float64, device="cuda")
    ctx.generate(a, n, ld, seed, nrhs, kind)
    return a, ld


def hpl(a0, x, n):
    """||Ax-b||_inf / (eps (||A||_inf ||x||_inf + ||b||_inf) n), eps = 2^-53, in float64 on the host."""
    A = a0[:, :n]
    b = a0[:, n]
    r = np.abs(A @ x - b).max()
    return r / (2.0**-53 * (np.abs(A).sum(1).max() * np.abs(x).max() + np.abs(b).max()) * n)


def test_generator_bit_exact(ctx, oracle):
    n, nrhs = 301, 3
    a, ld = dev_matrix(ctx, n, 12345, nrhs)
    ref = oracle.randomsetmat(n, 12345, nrhs=nrhs)
    assert np.array_equal(a.cpu().numpy()[:, : n + nrhs], ref[:, : n + nrhs])


def test_generator_diagonally_dominant(ctx, oracle):
    n = 200
    a, ld = dev_matrix(ctx, n, 3, 1, kind=1)
    g = a.cpu().numpy()
    ref = oracle.randomsetmat(n, 3)
    off = ~np.eye(n, dtype=bool)
    assert np.array_equal(g[:, :n][off], ref[:, :n][off])
    np.testing.assert_allclose(np.diag(g[:, :n]), np.abs(ref[:, :n]).sum(1), rtol=1e-13)


@pytest.mark.parametrize("n,nb,seed", GOLDEN_CASES)
@pytest.mark.parametrize("variant,mode", [("fixed", PIVOT_PARTIAL), ("shipped", PIVOT_REF)])
def test_lusolve_matches_reference(ctx, golden, oracle, parity, n, nb, seed, variant, mode):
    a, ld = dev_matrix(ctx, n, seed)
    info = ctx.lusolve(a, n, ld, nb, 1, mode)
    assert info == 0
    piv = ctx.pivots(n)
    key = "%s_n%d_nb%d_s%d" % (variant, n, nb, seed)
    np.testing.assert_array_equal(piv, golden[key + "_piv"])
    x = a[:, n].cpu().numpy()
    xr = golden[key + "_x"]
    xhp = golden["hp_n%d_s%d_x" % (n, seed)]
    d_ref = rel(xr, xhp)
    parity("lusolve %s n=%d nb=%d seed=%d" % (variant, n, nb, seed), rel(x, xr), x_bar(mode, d_ref),
           "fwd err gpu %.2e ref %.2e" % (rel(x, xhp), d_ref))
    if mode == PIVOT_PARTIAL:
        assert hpl(oracle.randomsetmat(n, seed), x, n) < 16


@pytest.mark.parametrize("n,nb,seed", DD_CASES)
@pytest.mark.parametrize("variant,mode", [("fixed", PIVOT_PARTIAL), ("shipped", PIVOT_REF)])
def test_lusolve_well_conditioned_matches_reference(ctx, golden, oracle, parity, n, nb, seed, variant, mode):
    """Diagonally dominant systems (the reference's matrix with a_ii replaced by
    the row's absolute sum): x within 1e-12 of the fixed reference."""
    import torch

    a, ld = dev_matrix(ctx, n, seed)
    diag = torch.tensor(golden["dd_diag_n%d_s%d" % (n, seed)], device="cuda")
    idx = torch.arange(n, device="cuda")
    a[idx, idx] = diag
    assert ctx.lusolve(a, n, ld, nb, 1, mode) == 0
    key = "%s_dd_n%d_nb%d_s%d" % (variant, n, nb, seed)
    np.testing.assert_array_equal(ctx.pivots(n), golden[key + "_piv"])
    x = a[:, n].cpu().numpy()
    xr = golden[key + "_x"]
    xhp = golden["dd_hp_n%d_s%d_x" % (n, seed)]
    d_ref = rel(xr, xhp)
    bar = XTOL_PARTIAL if mode == PIVOT_PARTIAL else x_bar(mode, d_ref)
    parity("lusolve diag-dominant %s n=%d nb=%d seed=%d" % (variant, n, nb, seed), rel(x, xr), bar,
           "fwd err gpu %.2e ref %.2e" % (rel(x, xhp), d_ref))


def test_lumcolumn_host_entry(oracle, golden, parity):
    n, nb, seed = 512, 64, 1
    a = oracle.randomsetmat(n, seed)
    b = np.zeros(n)
    pv = np.zeros(nb, dtype=np.int32)
    assert lumcolumn(a, b, nb, pv, PIVOT_PARTIAL) == 0
    ao = oracle.randomsetmat(n, seed)
    xo, po = oracle.lumcolumn(ao, n, nb, PIVOT_PARTIAL)
    np.testing.assert_array_equal(pv, po[n - nb:])
    xr = golden["fixed_n512_nb64_s1_x"]
    parity("lumcolumn (host) n=512 nb=64 seed=1 vs fixed reference", rel(b, xr),
           x_bar(PIVOT_PARTIAL, rel(xr, golden["hp_n512_s1_x"])), "vs oracle %.2e" % rel(b, xo))
    # the factors land in the caller's array in lu2's storage (unit U', y in column n)
    iu = np.triu_indices(n, 1)
    assert np.abs(a[:, :n][iu] - ao[:, :n][iu]).max() < 1e-9
    assert np.abs(a[:, n] - ao[:, n]).max() / np.abs(ao[:, n]).max() < 1e-10


@pytest.mark.parametrize("n,nb", [(1000, 256), (1500, 128), (37, 16)])
def test_lumcolumn_pinned_host_overlaps_copies(oracle, n, nb):
    """On pinned host buffers the finished factor blocks are copied back while
    the factorization runs; the result is the same, bit for bit, as the one
    copied back at the end for pageable buffers."""
    import torch

    a_pg = oracle.randomsetmat(n, 5)
    b_pg = np.zeros(n)
    pv_pg = np.zeros(nb, dtype=np.int32)
    assert lumcolumn(a_pg, b_pg, nb, pv_pg, PIVOT_PARTIAL) == 0
    a_t = torch.empty(a_pg.shape, dtype=torch.float64, pin_memory=True)
    b_t = torch.zeros(n, dtype=torch.float64, pin_memory=True)
    a_pin, b_pin = a_t.numpy(), b_t.numpy()
    a_pin[...] = np.nan  # every element the factorization owns must be written back
    a_pin[:, : n + 1] = oracle.randomsetmat(n, 5)[:, : n + 1]
    pv_pin = np.zeros(nb, dtype=np.int32)
    assert lumcolumn(a_pin, b_pin, nb, pv_pin, PIVOT_PARTIAL) == 0
    np.testing.assert_array_equal(a_pin[:, : n + 1], a_pg[:, : n + 1])
    np.testing.assert_array_equal(b_pin, b_pg)
    np.testing.assert_array_equal(pv_pin, pv_pg)


@pytest.mark.parametrize("n,nb,mode", [(2000, 128, PIVOT_PARTIAL), (1111, 64, PIVOT_PARTIAL), (3000, 256, PIVOT_REF),
                                       (2048, 512, PIVOT_PARTIAL), (12000, 256, PIVOT_PARTIAL)])
def test_lookahead_matches_serial_factorization(ctx, monkeypatch, n, nb, mode):
    """The lookahead schedule (the next panel factored on a high-priority
    stream while the rest of the update runs, its leaf on fewer CTAs once the
    rows need more than 64) gives the serial schedule's factors, right-hand
    side and pivots bit for bit."""
    out = []
    for env in ("0", "1"):
        monkeypatch.setenv("LU2GPU_LOOKAHEAD", env)
        a, ld = dev_matrix(ctx, n, 21)
        assert ctx.lusolve(a, n, ld, nb, 1, mode) == 0
        out.append((a.cpu().numpy()[:, : n + 1], ctx.pivots(n)))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("n,nb,left", [(1500, 128, 3), (1500, 128, 100), (1000, 48, 7), (300, 256, 2),
                                       (37, 16, 1)])
def test_lumcolumn_left_looking_start_is_bit_identical(oracle, monkeypatch, n, nb, left):
    """On pinned host buffers the matrix arrives in column chunks and the
    first panels are factored left-looking as they arrive (the columns right
    of them catch up afterwards); every element sees the same operations in
    the same order as in the right-looking schedule, so the result is the
    same bit for bit as the pageable path's.  `left` forces the number of
    left-looking panels (100: all of them)."""
    import torch

    a_pg = oracle.randomsetmat(n, 9)
    b_pg = np.zeros(n)
    pv_pg = np.zeros(nb, dtype=np.int32)
    assert lumcolumn(a_pg, b_pg, nb, pv_pg, PIVOT_PARTIAL) == 0
    monkeypatch.setenv("LU2GPU_LEFT_PANELS", str(left))
    a_t = torch.empty(a_pg.shape, dtype=torch.float64, pin_memory=True)
    b_t = torch.zeros(n, dtype=torch.float64, pin_memory=True)
    a_pin, b_pin = a_t.numpy(), b_t.numpy()
    a_pin[...] = np.nan
    a_pin[:, : n + 1] = oracle.randomsetmat(n, 9)[:, : n + 1]
    pv_pin = np.zeros(nb, dtype=np.int32)
    assert lumcolumn(a_pin, b_pin, nb, pv_pin, PIVOT_PARTIAL) == 0
    np.testing.assert_array_equal(a_pin[:, : n + 1], a_pg[:, : n + 1])
    np.testing.assert_array_equal(b_pin, b_pg)
    np.testing.assert_array_equal(pv_pin, pv_pg)


def _host_memory_type(arr) -> int:
    """cudaPointerAttributes.type of a host array (0: unregistered, 1: page-locked)."""
    import ctypes
    import glob

    rt = ctypes.CDLL(sorted(glob.glob("/usr/local/cuda/lib64/libcudart.so*"))[0])
    attr = (ctypes.c_int * 8)()
    rc = rt.cudaPointerGetAttributes(ctypes.byref(attr), ctypes.c_void_p(arr.ctypes.data))
    rt.cudaGetLastError()
    return int(attr[0]) if rc == 0 else 0


@pytest.mark.parametrize("n,nb", [(1500, 128), (700, 64)])
def test_lumcolumn_registers_pageable_matrix_for_the_call(oracle, monkeypatch, n, nb):
    """A pageable matrix page-locked by lumcolumn for the call (forced here
    with LU2GPU_HOST_REGISTER=1; by default only from 2 GB) takes the
    overlapped path and gives the pageable path's result bit for bit; the
    array is unregistered again when the call returns."""
    out = []
    for reg in ("0", "1"):
        monkeypatch.setenv("LU2GPU_HOST_REGISTER", reg)
        a = oracle.randomsetmat(n, 21)
        b = np.zeros(n)
        pv = np.zeros(nb, dtype=np.int32)
        assert _host_memory_type(a) == 0
        assert lumcolumn(a, b, nb, pv, PIVOT_PARTIAL) == 0
        assert _host_memory_type(a) == 0
        out.append((a[:, : n + 1].copy(), b.copy(), pv.copy()))
    for u, v in zip(out[0], out[1]):
        np.testing.assert_array_equal(u, v)


@pytest.mark.parametrize("n,nb", [(1, 16), (2, 16), (15, 16), (16, 16), (17, 16), (33, 16), (100, 32), (1000, 256),
                                  (777, 64)])
def test_ragged_sizes_vs_lapack(ctx, oracle, n, nb):
    import scipy.linalg as sl

    a, ld = dev_matrix(ctx, n, 11)
    a0 = a.cpu().numpy().copy()
    assert ctx.lusolve(a, n, ld, nb, 1, PIVOT_PARTIAL) == 0
    lu, lp = sl.lu_factor(a0[:, :n])
    np.testing.assert_array_equal(ctx.pivots(n), lp)
    xs = sl.lu_solve((lu, lp), a0[:, n])
    x = a[:, n].cpu().numpy()
    assert np.abs(x - xs).max() / np.abs(xs).max() < 1e-10
    assert hpl(a0, x, n) < 16


def test_many_rhs(ctx):
    import scipy.linalg as sl

    n, nb, nrhs = 384, 64, 11
    a, ld = dev_matrix(ctx, n, 5, nrhs)
    a0 = a.cpu().numpy().copy()
    assert ctx.lusolve(a, n, ld, nb, nrhs, PIVOT_PARTIAL) == 0
    xs = sl.solve(a0[:, :n], a0[:, n:n + nrhs])
    x = a[:, n:n + nrhs].cpu().numpy()
    assert np.abs(x - xs).max() / np.abs(xs).max() < 1e-11


def test_factor_then_separate_backsolve(ctx, oracle):
    import torch

    n, nb = 640, 128
    a, ld = dev_matrix(ctx, n, 21)
    a0 = a.cpu().numpy().copy()
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert ctx.factor(a, n, ld, nb, 1, PIVOT_PARTIAL, ipiv) == 0
    x = a[:, n].clone().reshape(n, 1).contiguous()
    ctx.backsolve(a, n, ld, x, 1, 1)
    assert hpl(a0, x.cpu().numpy()[:, 0], n) < 16
    np.testing.assert_array_equal(ipiv.cpu().numpy(), ctx.pivots(n))


@pytest.mark.parametrize("mode", [PIVOT_PARTIAL, PIVOT_REF])
def test_resolve_from_stored_factors(ctx, mode):
    """lu2gpu_solve: new right-hand sides against the stored factors (lu2's
    storage + the full pivot sequence), including one factored with nrhs = 0."""
    import scipy.linalg as sl
    import torch

    n, nb = 1000, 64
    a, ld = dev_matrix(ctx, n, 31)
    a0 = a.cpu().numpy().copy()
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert ctx.factor(a, n, ld, nb, 1, mode, ipiv) == 0
    x_aug = a[:, n].clone().reshape(n, 1).contiguous()
    ctx.backsolve(a, n, ld, x_aug, 1, 1)
    rng = np.random.default_rng(0)
    B = np.concatenate([a0[:, n:n + 1], rng.uniform(-0.5, 0.5, (n, 2))], axis=1)
    b = torch.tensor(B, device="cuda").contiguous()
    ctx.solve(a, n, ld, nb, ipiv, b, 3, 3)
    xs = sl.solve(a0[:, :n], B)
    xb = b.cpu().numpy()
    tol = 1e-10 if mode == PIVOT_PARTIAL else 1e-6
    assert np.abs(xb - xs).max() / np.abs(xs).max() < tol
    xa = x_aug.cpu().numpy()[:, 0]
    assert np.abs(xb[:, 0] - xa).max() / np.abs(xa).max() < 1e-13
    # factor without a riding right-hand side, then solve
    a2, _ = dev_matrix(ctx, n, 31)
    assert ctx.factor(a2, n, ld, nb, 0, mode, ipiv) == 0
    b2 = torch.tensor(B[:, :1], device="cuda").contiguous()
    ctx.solve(a2, n, ld, nb, ipiv, b2, 1, 1)
    assert np.abs(b2.cpu().numpy()[:, 0] - xa).max() / np.abs(xa).max() < 1e-13


def test_zero_pivot_reports_column(ctx):
    import torch

    n, nb = 96, 32
    a, ld = dev_matrix(ctx, n, 2)
    a[:, 40] = 0.0  # an exactly singular column
    info = ctx.lusolve(a, n, ld, nb, 1, PIVOT_PARTIAL)
    assert info == 41
    assert torch.isfinite(a[:, :40]).all()


def test_pivot_ties_go_to_lowest_row(ctx, oracle):
    n, nb = 64, 16
    a, ld = dev_matrix(ctx, n, 4)
    a[:, 0] = 0.1
    a[9, 0] = 0.5
    a[5, 0] = -0.5  # same |a| as row 9, lower index
    a0 = a.cpu().numpy().copy()
    assert ctx.lusolve(a, n, ld, nb, 1, PIVOT_PARTIAL) == 0
    assert ctx.pivots(n)[0] == 5
    ao = np.zeros((n, n + 16))
    ao[:, : n + 1] = a0[:, : n + 1]
    _, po = oracle.lumcolumn(ao, n, nb, PIVOT_PARTIAL)
    np.testing.assert_array_equal(ctx.pivots(n), po)


def hp_solution(a0, n):
    """The system's solution refined with long-double residuals (the yardstick
    of forward errors; the fixtures' hp_* vectors are made the same way)."""
    import scipy.linalg as sl

    A, b = a0[:, :n], a0[:, n]
    lu = sl.lu_factor(A)
    x = sl.lu_solve(lu, b).astype(np.longdouble)
    Al, bl = A.astype(np.longdouble), b.astype(np.longdouble)
    for _ in range(3):
        x = x + sl.lu_solve(lu, (bl - Al @ x).astype(np.float64)).astype(np.longdouble)
    return x.astype(np.float64)


@pytest.fixture(scope="module")
def n8192_case(oracle):
    a0 = oracle.randomsetmat(8192, 1)
    return a0, hp_solution(a0, 8192)


@pytest.mark.skipif(not RefLib.available("fixed"), reason="compiled reference not present")
@pytest.mark.parametrize("variant,mode", [("fixed", PIVOT_PARTIAL), ("shipped", PIVOT_REF)])
def test_n8192_against_compiled_reference(ctx, oracle, parity, n8192_case, variant, mode):
    """Cross-check at N=8192 (nb=256): the compiled reference CPU lu2 on identical inputs."""
    import os

    n, nb, seed = 8192, 256, 1
    a0, xhp = n8192_case
    ref = RefLib(variant)
    ref.set_threads(max(1, min(32, os.cpu_count() or 1)), 1)
    xr, pr, _ = ref.factor_solve(n, nb, seed)
    a, ld = dev_matrix(ctx, n, seed)
    assert ctx.lusolve(a, n, ld, nb, 1, mode) == 0
    piv = ctx.pivots(n)
    x = a[:, n].cpu().numpy()
    mism = int((piv != pr).sum())
    assert mism == 0, "%d pivot mismatches" % mism
    d_ref = rel(xr, xhp)
    parity("lusolve %s n=8192 nb=256 seed=1 (live reference)" % variant, rel(x, xr), x_bar(mode, d_ref),
           "fwd err gpu %.2e ref %.2e" % (rel(x, xhp), d_ref))
    if mode == PIVOT_PARTIAL:
        assert hpl(a0, x, n) < 16

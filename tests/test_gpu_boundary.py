"""lu2's per-panel entry points (lu2.c) and column-major slab API (lu2tlib.h)
on host arrays, through the C ABI.  lumcolumn's own loop (lu2.c:1122-1144) is
driven through them exactly as the reference's main would and compared with
the reference's golden pivots and solution."""
import ctypes

import numpy as np
import pytest

import lu2_b200 as L
from lu2_b200._lib import last_error

pytestmark = pytest.mark.gpu


def _p(x):
    return ctypes.c_void_p(x.ctypes.data)


@pytest.mark.parametrize("n,nb,seed,variant,mode",
                         [(512, 128, 12345, "fixed", L.PIVOT_PARTIAL),
                          (2048, 256, 1, "fixed", L.PIVOT_PARTIAL),
                          (256, 64, 12345, "shipped", L.PIVOT_REF)])
def test_lu2_panel_loop_through_boundary(oracle, golden, parity, n, nb, seed, variant, mode):
    """Bars as in test_gpu_lu.py: max(1e-12, 4 d_ref) against the fixed
    reference, 4 d_ref against the shipped one (d_ref = that reference's own
    forward error against the extended-precision solution)."""
    lib = L.load()
    old = lib.lu2gpu_set_pivot_mode(mode)
    try:
        a = oracle.randomsetmat(n, seed)
        pv = np.zeros(nb, dtype=np.int32)
        piv = np.zeros(n, dtype=np.int32)
        for i in range(0, n, nb):
            lib.column_decomposition_recursive(n, _p(a), nb, None, _p(pv), i)
            lib.process_right_part(n, _p(a), nb, None, _p(pv), i, n + 1)
            piv[i:i + nb] = pv
        b = np.zeros(n)
        lib.backward_sub(n, _p(a), _p(b))
    finally:
        lib.lu2gpu_set_pivot_mode(old)
    key = "%s_n%d_nb%d_s%d" % (variant, n, nb, seed)
    np.testing.assert_array_equal(piv, golden[key + "_piv"])
    xr = golden[key + "_x"]
    xhp = golden["hp_n%d_s%d_x" % (n, seed)]
    d_ref = np.abs(xr - xhp).max() / np.abs(xhp).max()
    bar = max(1e-12, 4 * d_ref) if mode == L.PIVOT_PARTIAL else 4 * d_ref
    parity("lu2 panel loop %s n=%d nb=%d seed=%d" % (variant, n, nb, seed), np.abs(b - xr).max() / np.abs(xr).max(),
           bar, "fwd err ref %.2e" % d_ref)


def _slab(oracle, n, i, cols, seed):
    """Columns i..i+cols-1 of lu2's matrix as lu2tlib's column-major slab a[j][r] (stride n)."""
    a = oracle.randomsetmat(n, seed)
    s = np.zeros((cols, n))
    s[:, i:] = a[i:, i:i + cols].T
    return s


def test_cm_recursive_equals_row_major_panel(oracle):
    lib = L.load()
    n, i, m = 700, 64, 16
    s = _slab(oracle, n, i, m, 3)
    pv = np.zeros(m, dtype=np.int32)
    lib.cm_column_decomposition_recursive(n, _p(s), m, _p(pv), i)
    a = oracle.randomsetmat(n, 3)
    pv2 = np.zeros(m, dtype=np.int32)
    lib.column_decomposition_recursive(n, _p(a), m, None, _p(pv2), i)
    np.testing.assert_array_equal(pv, pv2)
    assert np.abs(s[:, i:].T - a[i:, i:i + m]).max() < 1e-13


def test_cm_right_part_matches_numpy(oracle):
    lib = L.load()
    n, i, m, cols = 300, 32, 8, 16
    s0 = _slab(oracle, n, i, cols, 9)
    s = s0.copy()
    pv = np.zeros(m, dtype=np.int32)
    lib.cm_column_decomposition_recursive(n, _p(s), m, _p(pv), i)
    left = s[:m, i:].T.copy()                     # factored left block, rows i..n-1
    right = s0[m:cols, i:].T.copy()               # original right block
    for k in range(m):                            # exchanges with 1/pivot scaling
        p = pv[k] - i
        right[[k, p]] = right[[p, k]]
        right[k] /= left[k, k]
    T = np.tril(left[:m, :m], -1) + np.eye(m)     # unit lower, row-scaled entries
    right[:m] = np.linalg.solve(T, right[:m])
    right[m:] -= left[m:, :m] @ right[:m]
    lib.cm_process_right_part(n, _p(s), m, _p(pv), i, i + cols)
    assert np.abs(s[m:cols, i:].T - right).max() < 1e-12


def test_cm_column_decomposition_reference_mode_pivots_on_first_column(oracle):
    """lu2tlib.c:1052: called directly on a slab, every column's pivot search
    scans the slab's first column."""
    lib = L.load()
    n, i, m = 200, 16, 6
    s = _slab(oracle, n, i, m, 11)
    ref = s.copy()
    pr = np.zeros(m, dtype=np.int32)
    for ip in range(m):  # lu2tlib.c:1041-1066 as written (findpivot scans a[0])
        ii = i + ip
        p = ii + int(np.argmax(np.abs(ref[0, ii:n])))
        pr[ip] = p
        ref[:m, [ii, p]] = ref[:m, [p, ii]]
        ainv = 1.0 / ref[ip, ii]
        ref[:ip, ii] *= ainv
        ref[ip + 1:m, ii] *= ainv
        for k in range(ip + 1, m):
            ref[k, ii + 1:n] -= ref[ip, ii + 1:n] * ref[k, ii]
    pv = np.zeros(m, dtype=np.int32)
    old = lib.lu2gpu_set_pivot_mode(L.PIVOT_REF)
    try:
        lib.cm_column_decomposition(n, _p(s), m, _p(pv), i)
    finally:
        lib.lu2gpu_set_pivot_mode(old)
    np.testing.assert_array_equal(pv, pr)
    assert np.abs(s[:, i:] - ref[:, i:]).max() < 1e-12


def test_right_part_rejects_out_of_range_pivots(oracle):
    """Caller-supplied pivots outside [i + k, n) are refused before any kernel runs."""
    lib = L.load()
    n, nb = 128, 32
    a = oracle.randomsetmat(n, 1)
    a0 = a.copy()
    for bad in (n, 0, -5):
        pv = np.arange(32, 64, dtype=np.int32)
        pv[3] = bad
        lib.process_right_part(n, _p(a), nb, None, _p(pv), 32, n + 1)
        assert "pivot 3" in last_error()
        assert np.array_equal(a, a0)

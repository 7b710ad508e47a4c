"""The oracle (CPU restatement of lu2) pinned against the reference itself.

Golden vectors come from the reference compiled from its own sources
(tests/golden/make_golden.py); these tests need no GPU."""
import ctypes

import numpy as np
import pytest

from oracle.oracle import PIVOT_PARTIAL, PIVOT_REF, RefLib

CASES = [(128, 64, 1), (256, 64, 1), (256, 64, 12345), (512, 64, 1), (512, 128, 12345), (1024, 256, 1),
         (2048, 64, 1), (2048, 128, 12345), (2048, 256, 1)]


def test_drand48_stream_matches_libc(oracle):
    libc = ctypes.CDLL("libc.so.6")
    libc.drand48.restype = ctypes.c_double
    for seed in (1, 12345, 0, 2**31 - 1):
        n = 31
        a = oracle.randomsetmat(n, seed)
        libc.srand48(ctypes.c_long(seed))
        ref = np.array([libc.drand48() - 0.5 for _ in range(n * (n + 1))]).reshape(n, n + 1)
        assert np.array_equal(a[:, : n + 1], ref)


@pytest.mark.parametrize("n,nb,seed", CASES)
@pytest.mark.parametrize("variant,mode,xtol", [("shipped", PIVOT_REF, 2e-8), ("fixed", PIVOT_PARTIAL, 2e-11)])
def test_oracle_matches_reference_golden(oracle, golden, n, nb, seed, variant, mode, xtol):
    key = "%s_n%d_nb%d_s%d" % (variant, n, nb, seed)
    x, piv = oracle.solve(n, nb, seed, mode)
    np.testing.assert_array_equal(piv, golden[key + "_piv"])
    xr = golden[key + "_x"]
    assert np.abs(x - xr).max() / np.abs(xr).max() < xtol


@pytest.mark.parametrize("n,seed", [(128, 1), (512, 1), (1024, 1), (2048, 12345)])
def test_fixed_pivots_equal_lapack(golden, n, seed):
    nbs = [c[1] for c in CASES if c[0] == n and c[2] == seed]
    for nb in nbs:
        np.testing.assert_array_equal(golden["fixed_n%d_nb%d_s%d_piv" % (n, nb, seed)],
                                      golden["lapack_n%d_s%d_piv" % (n, seed)])


def test_oracle_partial_vs_scipy(oracle):
    import scipy.linalg as sl

    n, nb = 256, 64
    a0 = oracle.randomsetmat(n, 7)
    a = a0.copy()
    x, piv = oracle.lumcolumn(a, n, nb, PIVOT_PARTIAL)
    lu, lpiv = sl.lu_factor(a0[:, :n].copy())
    np.testing.assert_array_equal(piv, lpiv)
    xl = sl.lu_solve((lu, lpiv), a0[:, n].copy())
    assert np.abs(x - xl).max() / np.abs(xl).max() < 1e-12


def test_hpl_residuals_document_the_reference_bug(oracle, golden):
    """Shipped lu2 fails HPL < 16 at INSTALL's sample config; the fixed one passes."""
    n, nb, seed = 2048, 128, 12345
    a0 = oracle.randomsetmat(n, seed)
    r_ship = oracle.residual(a0, n, golden["shipped_n%d_nb%d_s%d_x" % (n, nb, seed)])
    r_fix = oracle.residual(a0, n, golden["fixed_n%d_nb%d_s%d_x" % (n, nb, seed)])
    assert r_ship["hpl"] > 16
    assert r_fix["hpl"] < 0.1
    assert abs(r_ship["rinf"] - float(golden["shipped_n%d_nb%d_s%d_emax" % (n, nb, seed)])) < 1e-12


def test_oracle_multiple_rhs(oracle):
    import scipy.linalg as sl

    n, nb, nrhs = 128, 64, 3
    a0 = oracle.randomsetmat(n, 5, nrhs=nrhs)
    a = a0.copy()
    x, _ = oracle.lumcolumn(a, n, nb, PIVOT_PARTIAL, nrhs=nrhs)
    xs = sl.solve(a0[:, :n], a0[:, n:n + nrhs])
    assert np.abs(x - xs).max() / np.abs(xs).max() < 1e-12


def test_oracle_rejects_unsupported_shapes(oracle):
    a = oracle.randomsetmat(96, 1)
    with pytest.raises(ValueError):
        oracle.lumcolumn(a, 96, 48)  # nb not a power of two (the reference halves m)


@pytest.mark.skipif(not RefLib.available("fixed"), reason="reference not compiled here")
def test_live_reference_equals_oracle(oracle):
    ref = RefLib("fixed")
    ref.set_threads(1, 1)
    xr, pr, _ = ref.factor_solve(256, 64, 99)
    x, p = oracle.solve(256, 64, 99, PIVOT_PARTIAL)
    np.testing.assert_array_equal(p, pr)
    assert np.abs(x - xr).max() / np.abs(xr).max() < 1e-12

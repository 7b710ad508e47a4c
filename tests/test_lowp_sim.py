"""The CPU simulation of the precision forms' factorization
(tests/lowp_lu_sim.py), and what it shows about the FP8 form on general
matrices.  No GPU needed; tests/test_gpu_fp8.py checks the GPU's factors
against the same simulation.

Findings pinned here (lu2's uniform [-0.5, 0.5) matrices, nb = 256):
* with E4M3 trailing updates the computed factors of a GENERAL matrix are the
  exact factors of A + E with ||E|| / ||A|| above 0.5 already at n = 512 and
  growing about linearly with n, and the pivots grow away from those of the
  FP32-update factorization as it proceeds; M = L U is then no preconditioner (||I - M^-1 A|| >> 1), and
  at the benchmark's n = 98304 the FP32 solves with these factors overflow;
* a two-term E4M3 split of each operand (hi + lo, three products) and BF16
  halve or keep that error but it still grows linearly with n (about 0.17 at
  n = 4096), so neither reaches a contracting preconditioner at n = 98304;
* on the diagonally dominant matrices of the BF16 configuration the same FP8
  factors are a strong preconditioner (||I - M^-1 A|| ~ 1e-4)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from lowp_lu_sim import (backward_error, e4m3, lowp_lu, lu2_factors_to_plu, precond_rho,  # noqa: E402
                         tile_exponent)


def matrix(oracle, n, kind):
    a = oracle.randomsetmat(n, 1)[:, :n].copy()
    if kind == "dd":
        a[np.arange(n), np.arange(n)] = np.abs(a).sum(1)
    return a


def test_e4m3_rounding_and_tile_scale():
    assert e4m3(np.array([448.0]))[0] == 448.0
    assert e4m3(np.array([1000.0]))[0] == 448.0          # saturates (satfinite)
    assert e4m3(np.array([1.0625]))[0] == 1.0            # halfway between 1 and 1.125: ties to even
    assert e4m3(np.array([1.1875]))[0] == 1.25
    assert e4m3(np.array([2.0**-9]))[0] == 2.0**-9       # the smallest subnormal
    assert e4m3(np.array([2.0**-10]))[0] == 0.0          # halfway to zero: ties to even
    assert e4m3(np.array([-3.3]))[0] == -3.25
    assert tile_exponent(448.0) == 0 and tile_exponent(1.0) == 8 and tile_exponent(300.0) == 0
    assert tile_exponent(0.0) == 0


def test_conversion_of_lu2_storage(oracle):
    """lu2's factor storage (the oracle's, FP64) to P A = L U, exactly."""
    n, nb = 512, 64
    a = oracle.randomsetmat(n, 3)
    a0 = a[:, :n].copy()
    _, piv = oracle.lumcolumn(a, n, nb, 1)
    lo, up, perm = lu2_factors_to_plu(a[:, :n], piv, nb)
    assert backward_error(a0, lo, up, perm) < 1e-14


def test_fp32_updates_control(oracle):
    a = matrix(oracle, 1024, "general")
    lo, up, perm = lowp_lu(a, 256, "fp32")
    assert backward_error(a, lo, up, perm) < 1e-4
    assert precond_rho(a, lo, up, perm, iters=10) < 0.1


def test_fp8_updates_precondition_diagonally_dominant_matrices(oracle):
    a = matrix(oracle, 1024, "dd")
    lo, up, perm = lowp_lu(a, 256, "fp8")
    assert backward_error(a, lo, up, perm) < 1e-3
    assert precond_rho(a, lo, up, perm, iters=10) < 1e-2


def test_fp8_updates_do_not_precondition_general_matrices(oracle):
    errs = {}
    for n in (512, 1024):
        a = matrix(oracle, n, "general")
        lo, up, perm = lowp_lu(a, 256, "fp8")
        errs[n] = backward_error(a, lo, up, perm)
        assert precond_rho(a, lo, up, perm, iters=10) > 10
    assert errs[512] > 0.5                 # the factors are those of a matrix far from A
    assert errs[1024] > 1.5 * errs[512]     # and the distance grows with n


def test_fp8_pivots_grow_away_from_the_fp32_ones(oracle):
    """The pivots of lu2's uniform matrices grow along the factorization in any
    precision; with E4M3 updates they grow faster: the first quarter's agree
    with the FP32-update factorization's, the last quarter's are half as large
    again at n = 2048 (twice at n = 4096)."""
    n = 2048
    a = matrix(oracle, n, "general")
    med = {}
    for upd in ("fp32", "fp8"):
        lo, _, _ = lowp_lu(a, 256, upd)
        piv = np.abs(np.diag(lo))
        med[upd] = (np.median(piv[:n // 4]), np.median(piv[-n // 4:]))
    assert med["fp8"][0] / med["fp32"][0] < 1.1
    assert med["fp8"][1] / med["fp32"][1] > 1.3


@pytest.mark.parametrize("upd", ["fp8x2", "bf16"])
def test_two_term_split_and_bf16_still_degrade_with_n(oracle, upd):
    errs = {}
    for n in (512, 1024):
        a = matrix(oracle, n, "general")
        lo, up, perm = lowp_lu(a, 256, upd)
        errs[n] = backward_error(a, lo, up, perm)
    assert 1e-3 < errs[512] < 0.2
    assert errs[1024] > 1.5 * errs[512]

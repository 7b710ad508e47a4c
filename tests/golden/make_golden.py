"""Generate tests/golden/lu2_ref_golden.npz from the reference itself.

The reference (telmin/lu2) ships no golden vectors for its factor+solve path
(INSTALL:83-93 quotes one Emax that the shipped code does not reproduce), so
the fixtures are produced by running the reference compiled from its own
sources (oracle/build_oracle.py -> oracle/_ref):

  * ``shipped``: the reference as shipped (pivot search of lu2tlib.c:1052);
  * ``fixed``:   the same with the one-token pivot fix;
  * ``lapack``:  scipy.linalg.lu_factor (LAPACK dgetrf) pivots for the same A.

For every (n, nb, seed) the file stores the full pivot sequence (0-based row
exchanged with row c at step c) and x, computed with one OpenBLAS thread and
one OpenMP thread so the bytes are reproducible, and ``hp_n*_s*_x``: the
solution of the same system refined with residuals in extended precision
(x87 long double), the yardstick for each solver's forward error.

``DD_CASES`` are well-conditioned systems: lu2's matrix with each diagonal
entry replaced by the sum of the absolute values of its row (``dd_diag``,
stored so every consumer builds the identical matrix).  Run from the
repository root:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.build_oracle import build_oracle, build_ref  # noqa: E402
from oracle.oracle import OracleLib, RefLib  # noqa: E402

CASES = [
    (128, 64, 1),
    (256, 64, 1),
    (256, 64, 12345),
    (512, 64, 1),
    (512, 128, 12345),
    (1024, 256, 1),
    (2048, 64, 1),
    (2048, 128, 12345),  # the sample run of INSTALL:83
    (2048, 256, 1),
]

# well-conditioned (diagonally dominant) systems
DD_CASES = [
    (1024, 64, 1),
    (2048, 256, 12345),
    (4096, 256, 1),
]

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lu2_ref_golden.npz")


def lapack_pivots(a0: np.ndarray, n: int) -> np.ndarray:
    import scipy.linalg as sl

    _, piv = sl.lu_factor(a0[:, :n].copy())
    return piv.astype(np.int32)


def hp_solution(A: np.ndarray, b: np.ndarray, steps: int = 4) -> np.ndarray:
    """x refined from LAPACK's solve with residuals b - A x in long double."""
    import scipy.linalg as sl

    lu = sl.lu_factor(A)
    x = sl.lu_solve(lu, b).astype(np.longdouble)
    Al, bl = A.astype(np.longdouble), b.astype(np.longdouble)
    for _ in range(steps):
        r = bl - Al @ x
        x = x + sl.lu_solve(lu, r.astype(np.float64)).astype(np.longdouble)
    return x.astype(np.float64)


def main() -> int:
    build_oracle()
    build_ref()
    orc = OracleLib()
    out = {"cases": np.array(CASES, dtype=np.int64)}
    for variant in ("shipped", "fixed"):
        ref = RefLib(variant)
        ref.set_threads(1, 1)
        for n, nb, seed in CASES:
            x, piv, _ = ref.factor_solve(n, nb, seed)
            key = "%s_n%d_nb%d_s%d" % (variant, n, nb, seed)
            out[key + "_piv"] = piv
            out[key + "_x"] = x
            a0 = orc.randomsetmat(n, seed)
            out[key + "_emax"] = np.array(orc.residual(a0, n, x)["rinf"])
    for n, nb, seed in CASES:
        a0 = orc.randomsetmat(n, seed)
        out["lapack_n%d_s%d_piv" % (n, seed)] = lapack_pivots(a0, n)
        out["hp_n%d_s%d_x" % (n, seed)] = hp_solution(a0[:, :n], a0[:, n])
    out["dd_cases"] = np.array(DD_CASES, dtype=np.int64)
    for n, nb, seed in DD_CASES:
        a0 = orc.randomsetmat(n, seed)
        diag = np.abs(a0[:, :n]).sum(axis=1)
        a0[np.arange(n), np.arange(n)] = diag
        out["dd_diag_n%d_s%d" % (n, seed)] = diag
        out["dd_hp_n%d_s%d_x" % (n, seed)] = hp_solution(a0[:, :n], a0[:, n])
        out["dd_lapack_n%d_s%d_piv" % (n, seed)] = lapack_pivots(a0, n)
        for variant in ("shipped", "fixed"):
            ref = RefLib(variant)
            ref.set_threads(1, 1)
            x, piv, _ = ref.factor_solve_diag(n, nb, seed, diag)
            key = "%s_dd_n%d_nb%d_s%d" % (variant, n, nb, seed)
            out[key + "_piv"] = piv
            out[key + "_x"] = x
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main())

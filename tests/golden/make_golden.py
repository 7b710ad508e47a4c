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
one OpenMP thread so the bytes are reproducible.  Run from the repository root:

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

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lu2_ref_golden.npz")


def lapack_pivots(a0: np.ndarray, n: int) -> np.ndarray:
    import scipy.linalg as sl

    _, piv = sl.lu_factor(a0[:, :n].copy())
    return piv.astype(np.int32)


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
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main())

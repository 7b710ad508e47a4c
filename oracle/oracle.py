"""ctypes access to the oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker.  The product library in lu2_b200/ never
loads anything from oracle/.

* ``OracleLib``: the C restatement (``lu2_oracle.c``) -- drand48 generator,
  lu2's recursive LU in both pivot modes, residuals.
* ``RefLib``: the compiled reference (``oracle/_ref``), present when it was
  built (see build_oracle.py).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PIVOT_REF = 0
PIVOT_PARTIAL = 1

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class OracleLib:
    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liblu2oracle.so")
        if not os.path.exists(path):
            from .build_oracle import build_oracle  # type: ignore

            build_oracle()
        self.lib = C.CDLL(path)
        L = self.lib
        L.orc_randomsetmat.argtypes = [C.c_int, C.c_int, C.c_long, _dp, C.c_long]
        L.orc_randomsetmat.restype = None
        L.orc_lumcolumn.argtypes = [C.c_int, C.c_int, _dp, C.c_long, C.c_int, C.c_int, _ip, _dp]
        L.orc_lumcolumn.restype = C.c_int
        L.orc_residual.argtypes = [C.c_int, _dp, C.c_long, _dp, _dp]
        L.orc_residual.restype = None

    def randomsetmat(self, n: int, seed: int, nrhs: int = 1, lda: int | None = None) -> np.ndarray:
        """lu2.c:70-85 stream: row-major (n, lda) with b in column n."""
        lda = lda or n + 16
        a = np.zeros((n, lda), dtype=np.float64)
        self.lib.orc_randomsetmat(n, nrhs, seed, a, lda)
        return a

    def lumcolumn(self, a: np.ndarray, n: int, nb: int, mode: int = PIVOT_PARTIAL, nrhs: int = 1):
        """In-place lu2 factor+solve of the augmented matrix ``a``; returns (x, ipiv)."""
        ipiv = np.zeros(n, dtype=np.int32)
        x = np.zeros(n * nrhs, dtype=np.float64)
        rc = self.lib.orc_lumcolumn(n, nrhs, a, a.shape[1], nb, mode, ipiv, x)
        if rc != 0:
            raise ValueError("orc_lumcolumn rejected n=%d nb=%d" % (n, nb))
        return (x if nrhs == 1 else x.reshape(n, nrhs)), ipiv

    def solve(self, n: int, nb: int, seed: int, mode: int = PIVOT_PARTIAL):
        a = self.randomsetmat(n, seed)
        return self.lumcolumn(a, n, nb, mode)

    def residual(self, a0: np.ndarray, n: int, x: np.ndarray) -> dict:
        """HPL residuals of x against the original augmented matrix a0."""
        out = np.zeros(10, dtype=np.float64)
        self.lib.orc_residual(n, np.ascontiguousarray(a0), a0.shape[1], np.ascontiguousarray(x, dtype=np.float64), out)
        keys = ["rinf", "ainf", "xinf", "binf", "a1", "x1", "hpl", "ref_r1", "ref_r2", "ref_r3"]
        return dict(zip(keys, out.tolist()))


class RefLib:
    """The reference itself, compiled from its sources into oracle/_ref."""

    def __init__(self, variant: str = "shipped"):
        path = os.path.join(HERE, "_ref", "libref_lu2_%s.so" % variant)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        L.ref_set_threads.argtypes = [C.c_int, C.c_int]
        L.ref_lu2_factor_solve.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _ip, C.POINTER(C.c_double)]
        L.ref_lu2_factor_solve.restype = C.c_int
        L.ref_lu2_lumcolumn.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.POINTER(C.c_double)]
        L.ref_lu2_lumcolumn.restype = C.c_int
        L.ref_lu2_factor_solve_diag.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _ip, C.POINTER(C.c_double)]
        L.ref_lu2_factor_solve_diag.restype = C.c_int

    @staticmethod
    def available(variant: str = "shipped") -> bool:
        return os.path.exists(os.path.join(HERE, "_ref", "libref_lu2_%s.so" % variant))

    def set_threads(self, blas: int, omp: int = 1) -> None:
        self.lib.ref_set_threads(blas, omp)

    def factor_solve(self, n: int, nb: int, seed: int):
        x = np.zeros(n, dtype=np.float64)
        piv = np.zeros(n, dtype=np.int32)
        t = C.c_double(0)
        rc = self.lib.ref_lu2_factor_solve(n, nb, seed, x, piv, C.byref(t))
        if rc != 0:
            raise RuntimeError("reference run failed rc=%d" % rc)
        return x, piv, t.value

    def factor_solve_diag(self, n: int, nb: int, seed: int, diag: np.ndarray):
        """factor_solve on randomsetmat's matrix with its diagonal replaced by ``diag``."""
        x = np.zeros(n, dtype=np.float64)
        piv = np.zeros(n, dtype=np.int32)
        t = C.c_double(0)
        rc = self.lib.ref_lu2_factor_solve_diag(n, nb, seed, np.ascontiguousarray(diag, dtype=np.float64), x, piv,
                                                C.byref(t))
        if rc != 0:
            raise RuntimeError("reference run failed rc=%d" % rc)
        return x, piv, t.value

    def lumcolumn(self, n: int, nb: int, seed: int):
        x = np.zeros(n, dtype=np.float64)
        t = C.c_double(0)
        rc = self.lib.ref_lu2_lumcolumn(n, nb, seed, x, C.byref(t))
        if rc != 0:
            raise RuntimeError("reference run failed rc=%d" % rc)
        return x, t.value

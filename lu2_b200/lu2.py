"""Host-side mirror of lu2's interface over liblu2gpu.so.

Names follow the reference (telmin/lu2): ``lumcolumn`` (lu2.c:1122),
``mydgemm`` (lu2lib.c:2079), ``gdr_dgemm_`` / ``gdrblas_dgemm`` /
``mygdrdgemm`` (gdrdgemm.c), ``randomsetmat`` (lu2.c:70).  Host arrays are
numpy; device arrays are anything with a ``data_ptr()`` (torch CUDA tensors)
or raw integer addresses.

Every call goes through the C ABI; there is no CPU path.  Failures raise
``Lu2GpuError`` carrying ``lu2gpu_last_error()``.
"""
from __future__ import annotations

import atexit
import ctypes as C
import sys
import weakref

import numpy as np

from . import _lib

# Contexts and batches still open when the interpreter exits are closed by an
# exit hook (batches first: a batch uses its context), while the CUDA runtime
# is still up; a finalizer that runs later does nothing.
_LIVE_BATCHES: "weakref.WeakSet" = weakref.WeakSet()
_LIVE_CONTEXTS: "weakref.WeakSet" = weakref.WeakSet()


def _close_live() -> None:
    for group in (_LIVE_BATCHES, _LIVE_CONTEXTS):
        for obj in list(group):
            try:
                obj.close()
            except Exception:
                pass


atexit.register(_close_live)

PIVOT_REF = 0
PIVOT_PARTIAL = 1
UPDATE_BF16 = 0
UPDATE_FP8 = 1
BATCH_FP64 = 0
BATCH_FP32_IR = 1
CBLAS_ROWMAJOR, CBLAS_COLMAJOR, CBLAS_NOTRANS, CBLAS_TRANS = 101, 102, 111, 112
TIMER_NAMES = ["col dec t", "swaprows", "solve tri", "DGEMMrest", "backward_sub", "panel update"]


class Lu2GpuError(RuntimeError):
    def __init__(self, where: str, rc: int):
        super().__init__("%s failed (status %d): %s" % (where, rc, _lib.last_error()))
        self.rc = rc


class SingularMatrix(Lu2GpuError):
    """The factorization met an exact zero pivot (status = column + 1)."""


def _check(where: str, rc: int) -> int:
    if rc < 0:
        raise Lu2GpuError(where, rc)
    return rc


def _ptr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return int(x.data_ptr())


def lib():
    return _lib.load()


def rdim(n: int) -> int:
    """Row stride of lu2's augmented matrix (RDIM, lu2.c:28)."""
    return n + 16


# ---------------------------------------------------------------------------
# reference entry points on host arrays


def lumcolumn(a: np.ndarray, b: np.ndarray, nb: int, pv: np.ndarray | None = None,
              pivot_mode: int = PIVOT_PARTIAL) -> int:
    """lu2.c:1122-1144 on host memory: ``a`` is (n, n+16) row-major float64 with
    b in column n; on return ``b`` holds x, ``a`` the factors.  Returns 0 or the
    zero-pivot status (column + 1)."""
    n = a.shape[0]
    if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape[1] != rdim(n):
        raise ValueError("a must be a C-contiguous float64 (n, n+16) array")
    if b.dtype != np.float64 or b.shape[0] < n or not b.flags.c_contiguous:
        raise ValueError("b must be a contiguous float64 vector of length n")
    if pv is None:
        pv = np.zeros(nb, dtype=np.int32)
    rc = lib().lu2gpu_lumcolumn(n, _ptr(a), _ptr(b), nb, _ptr(pv), pivot_mode)
    return _check("lumcolumn", rc)


def mydgemm(m, n, k, alpha, a, na, b, nb, beta, c, nc) -> None:
    """Row-major C = alpha*A*B + beta*C on host arrays (lu2lib.c:2079)."""
    lib().mydgemm(m, n, k, alpha, _ptr(a), na, _ptr(b), nb, beta, _ptr(c), nc)
    err = _lib.last_error()
    if err and "mydgemm" in err:
        raise Lu2GpuError("mydgemm", -2)


def gdr_dgemm_(nota, notb, m, n, k, alpha, beta, lda, ldb, ldc, a, b, c) -> int:
    """The board library's Fortran-style column-major DGEMM; returns doneflag."""
    I = C.c_int
    D = C.c_double
    done = I(0)
    lib().gdr_dgemm_(C.byref(I(nota)), C.byref(I(notb)), C.byref(I(m)), C.byref(I(n)), C.byref(I(k)),
                     C.byref(D(alpha)), C.byref(D(beta)), C.byref(I(lda)), C.byref(I(ldb)), C.byref(I(ldc)),
                     _ptr(a), _ptr(b), _ptr(c), C.byref(done))
    return done.value


def gdrblas_dgemm(order, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, Cm, ldc) -> None:
    lib().gdrblas_dgemm(order, transa, transb, M, N, K, alpha, _ptr(A), lda, _ptr(B), ldb, beta, _ptr(Cm), ldc)


def mygdrdgemm(m, n, k, alpha, a, na, b, nb, beta, c, nc) -> None:
    lib().mygdrdgemm(m, n, k, alpha, _ptr(a), na, _ptr(b), nb, beta, _ptr(c), nc)


def set_pivot_mode(mode: int) -> int:
    return _check("lu2gpu_set_pivot_mode", lib().lu2gpu_set_pivot_mode(mode))


# ---------------------------------------------------------------------------
# device-resident API


class Context:
    """One lu2gpu context (a device, its stream and workspaces)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        _check("lu2gpu_create", lib().lu2gpu_create(C.byref(self._h), device))
        self.device = device
        _LIVE_CONTEXTS.add(self)

    def close(self) -> None:
        if self._h:
            lib().lu2gpu_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        if sys.is_finalizing():
            return
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream) -> None:
        """Run on an external cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream)."""
        _check("lu2gpu_set_stream", lib().lu2gpu_set_stream(self._h, int(stream)))

    def generate(self, a, n: int, lda: int, seed: int, nrhs: int = 1, kind: int = 0) -> None:
        """randomsetmat on the device (kind 1: diagonally dominant)."""
        _check("lu2gpu_generate", lib().lu2gpu_generate(self._h, n, nrhs, seed, kind, _ptr(a), lda))

    def factor(self, a, n: int, lda: int, nb: int, nrhs: int = 1, pivot_mode: int = PIVOT_PARTIAL,
               ipiv=None) -> int:
        return _check("lu2gpu_factor",
                      lib().lu2gpu_factor(self._h, n, nrhs, _ptr(a), lda, nb, pivot_mode, _ptr(ipiv)))

    def backsolve(self, a, n: int, lda: int, x, ldx: int, nrhs: int = 1) -> None:
        _check("lu2gpu_backsolve", lib().lu2gpu_backsolve(self._h, n, nrhs, _ptr(a), lda, _ptr(x), ldx))

    def lusolve(self, a, n: int, lda: int, nb: int, nrhs: int = 1, pivot_mode: int = PIVOT_PARTIAL,
                ipiv=None) -> int:
        """Factor + solve in place (x in columns n..n+nrhs-1)."""
        return _check("lu2gpu_lusolve",
                      lib().lu2gpu_lusolve(self._h, n, nrhs, _ptr(a), lda, nb, pivot_mode, _ptr(ipiv)))

    def solve(self, a, n: int, lda: int, nb: int, ipiv, b, ldb: int, nrhs: int = 1) -> None:
        """Re-solve from stored factors (device a, ipiv) into b (overwritten by x)."""
        _check("lu2gpu_solve", lib().lu2gpu_solve(self._h, n, _ptr(a), lda, nb, _ptr(ipiv), _ptr(b), ldb, nrhs))

    def mixed_solve(self, a, n: int, lda: int, b, x, nb: int = 256, pivot_mode: int = PIVOT_PARTIAL,
                    max_iter: int = 30) -> dict:
        """Precision form: FP32/BF16 LU + FP64 iterative refinement (device a, b, x)."""
        out = np.zeros(4, dtype=np.float64)
        rc = lib().lu2gpu_mixed_solve(self._h, n, _ptr(a), lda, _ptr(b), _ptr(x), nb, pivot_mode, max_iter, _ptr(out))
        res = {"status": rc, "iterations": int(out[0]), "hpl": float(out[1]), "factor_s": float(out[2]),
               "refine_s": float(out[3])}
        if rc < 0 and rc != -6:
            raise Lu2GpuError("lu2gpu_mixed_solve", rc)
        return res

    def gmres_solve(self, a, n: int, lda: int, b, x, nb: int = 256, update: int = UPDATE_FP8, restart: int = 30,
                    inner_tol: float = 1e-6, max_iter: int = 300) -> dict:
        """GMRES-IR: FP32 panel + BF16/FP8 trailing updates, FP64 refinement with
        GMRES(restart) on the correction equations (device a, b, x)."""
        out = np.zeros(6, dtype=np.float64)
        rc = lib().lu2gpu_gmres_solve(self._h, n, _ptr(a), lda, _ptr(b), _ptr(x), nb, update, restart, inner_tol,
                                      max_iter, _ptr(out))
        res = {"status": rc, "refinements": int(out[0]), "gmres_iterations": int(out[1]), "hpl": float(out[2]),
               "factor_s": float(out[3]), "refine_s": float(out[4]), "finite_factors": bool(out[5])}  # finite_factors: the preconditioner's FP32 solve stayed finite
        if rc < 0 and rc != -6:
            raise Lu2GpuError("lu2gpu_gmres_solve", rc)
        return res

    def lowp_factor(self, a, n: int, lda: int, nb: int, update: int, f, ldf: int, ipiv=None) -> int:
        """The precision forms' factorization (FP32 panels, BF16 or E4M3 trailing
        updates) of the FP64 device matrix a into the FP32 device array f."""
        return _check("lu2gpu_lowp_factor", lib().lu2gpu_lowp_factor(self._h, n, _ptr(a), lda, nb, update, _ptr(f), ldf,
                                                                       _ptr(ipiv)))

    def fp8_update(self, M, N, K, a32, lda, bt32, ldb, c32, ldc, a_deq=None, bt_deq=None) -> None:
        """c -= q(a) q(bt)^T with per-128x128-tile E4M3 quantization (FP32 device arrays)."""
        _check("lu2gpu_fp8_update_dev",
               lib().lu2gpu_fp8_update_dev(self._h, M, N, K, _ptr(a32), lda, _ptr(bt32), ldb, _ptr(c32), ldc,
                                           _ptr(a_deq) if a_deq is not None else None,
                                           _ptr(bt_deq) if bt_deq is not None else None))

    def bf16_update(self, M, N, K, a16, lda, bt16, ldb, c32, ldc, scale=1.0) -> None:
        _check("lu2gpu_bf16_update_dev", lib().lu2gpu_bf16_update_dev(self._h, M, N, K, _ptr(a16), lda, _ptr(bt16),
                                                                       ldb, _ptr(c32), ldc, scale))

    def dgemm(self, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> None:
        _check("lu2gpu_dgemm_dev",
               lib().lu2gpu_dgemm_dev(self._h, m, n, k, alpha, _ptr(a), lda, _ptr(b), ldb, beta, _ptr(c), ldc))

    def swaprows(self, a, n: int, lda: int, k0: int, k1: int, ipiv, dinv, cs: int, ce: int) -> None:
        """lu2's row exchanges of a panel (rows k <-> ipiv[k], k = k0..k1-1, then
        row k *= dinv[k]) on columns cs..ce-1 of the device matrix a."""
        _check("lu2gpu_swaprows_dev", lib().lu2gpu_swaprows_dev(self._h, n, _ptr(a), lda, k0, k1, _ptr(ipiv),
                                                                 _ptr(dinv) if dinv is not None else None, cs, ce))

    def solve_triangle(self, K: int, t, ldt: int, x, ldx: int, ncols: int, bt=None) -> None:
        """x := T^{-1} x with T the unit lower triangle of the K x K block t;
        bt (optional) receives -x^T (lu2.c:485-521 on device memory)."""
        _check("lu2gpu_solve_triangle_dev", lib().lu2gpu_solve_triangle_dev(self._h, K, _ptr(t), ldt, _ptr(x), ldx,
                                                                             ncols, _ptr(bt) if bt is not None else None))

    def test_leaf_withhold(self, cta: int, wait_ms: float) -> None:
        """Fault-path test hook: leaf waits give up after wait_ms; CTA `cta` skips its publications."""
        _check("lu2gpu_test_leaf_withhold", lib().lu2gpu_test_leaf_withhold(self._h, cta, wait_ms))

    def pivots(self, n: int) -> np.ndarray:
        out = np.zeros(n, dtype=np.int32)
        _check("lu2gpu_copy_pivots", lib().lu2gpu_copy_pivots(self._h, _ptr(out), n))
        return out

    def set_timing(self, on: bool) -> None:
        lib().lu2gpu_set_timing(self._h, 1 if on else 0)

    def timers(self, reset: bool = True) -> dict:
        ms = np.zeros(8, dtype=np.float64)
        cnt = np.zeros(8, dtype=np.int64)
        k = lib().lu2gpu_get_timers(self._h, _ptr(ms), _ptr(cnt), 8, 1 if reset else 0)
        return {TIMER_NAMES[i]: (float(ms[i]), int(cnt[i])) for i in range(k)}


def batch_sizes(count: int, seed: int, nmin: int = 16, nmax: int = 512, frac_multi: float = 0.1,
                nrhs_multi: int = 8):
    """Orders log-uniform in [nmin, nmax]; a fraction frac_multi get nrhs_multi right-hand sides."""
    n = np.zeros(count, dtype=np.int32)
    r = np.zeros(count, dtype=np.int32)
    _check("lu2gpu_batch_sizes", lib().lu2gpu_batch_sizes(count, seed, nmin, nmax, frac_multi, nrhs_multi,
                                                          _ptr(n), _ptr(r)))
    return n, r


def batch_shard(n, nrhs, world: int, rank: int) -> np.ndarray:
    """Indices of the systems that rank `rank` of `world` solves.

    The batching form shards without any exchange: the systems are
    independent, so each GPU takes a share balanced by cost (2/3 n^3 + 2 n^2
    nrhs FLOPs), assigned largest first to the least-loaded rank (ties to the
    lowest rank).  Every rank computes the same split from the same sizes."""
    import heapq

    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    nf = np.asarray(n, dtype=np.float64)
    rf = np.asarray(nrhs, dtype=np.float64)
    cost = 2.0 / 3.0 * nf**3 + 2.0 * nf**2 * rf
    owner = np.empty(len(nf), dtype=np.int64)
    heap = [(0.0, k) for k in range(world)]
    for i in np.argsort(-cost, kind="stable"):
        load, k = heapq.heappop(heap)
        owner[i] = k
        heapq.heappush(heap, (load + cost[i], k))
    return np.nonzero(owner == rank)[0]


class Batch:
    """A batch of independent systems solved by one persistent launch."""

    def __init__(self, ctx: Context, n, nrhs=None):
        self.n = np.ascontiguousarray(n, dtype=np.int32)
        self.nrhs = np.ascontiguousarray(nrhs if nrhs is not None else np.ones_like(self.n), dtype=np.int32)
        self.count = len(self.n)
        self._ctx = ctx  # the batch's device memory and streams belong to this context
        self._h = C.c_void_p()
        _check("lu2gpu_batch_create", lib().lu2gpu_batch_create(ctx.handle, self.count, _ptr(self.n),
                                                                _ptr(self.nrhs), C.byref(self._h)))
        _LIVE_BATCHES.add(self)

    def close(self) -> None:
        if self._h:
            if self._ctx.handle:
                lib().lu2gpu_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        if sys.is_finalizing():
            return
        try:
            self.close()
        except Exception:
            pass

    def system(self, i: int):
        """(device pointer, row stride) of system i's augmented matrix."""
        p = C.c_void_p()
        ld = C.c_long()
        _check("lu2gpu_batch_system", lib().lu2gpu_batch_system(self._h, i, C.byref(p), C.byref(ld)))
        return p.value, ld.value

    def generate(self, seed: int) -> None:
        _check("lu2gpu_batch_generate", lib().lu2gpu_batch_generate(self._h, seed))

    def generate_seeds(self, seeds) -> None:
        """System i := lu2's stream with seed seeds[i]."""
        s = np.ascontiguousarray(seeds, dtype=np.int64)
        if s.shape != (self.count,):
            raise ValueError("need one seed per system")
        _check("lu2gpu_batch_generate_seeds", lib().lu2gpu_batch_generate_seeds(self._h, _ptr(s)))

    def snapshot(self) -> None:
        _check("lu2gpu_batch_snapshot", lib().lu2gpu_batch_snapshot(self._h))

    def restore(self) -> None:
        _check("lu2gpu_batch_restore", lib().lu2gpu_batch_restore(self._h))

    def set_config(self, threads: int, pw: int, ctas_per_sm: int) -> None:
        _check("lu2gpu_batch_set_config", lib().lu2gpu_batch_set_config(self._h, threads, pw, ctas_per_sm))

    def set_mode(self, mode: int, max_iter: int = 10) -> None:
        """BATCH_FP64 or BATCH_FP32_IR (FP32 factors, FP64 refinement to HPL < 16)."""
        _check("lu2gpu_batch_set_mode", lib().lu2gpu_batch_set_mode(self._h, mode, max_iter))

    def iterations(self) -> np.ndarray:
        out = np.zeros(self.count, dtype=np.int32)
        _check("lu2gpu_batch_iterations", lib().lu2gpu_batch_iterations(self._h, _ptr(out)))
        return out

    def autotune(self) -> dict:
        out = np.zeros(4, dtype=np.int32)
        _check("lu2gpu_batch_autotune", lib().lu2gpu_batch_autotune(self._h, _ptr(out)))
        return {"threads": int(out[0]), "pw": int(out[1]), "ctas_per_sm": int(out[2]), "us": int(out[3]),
                "bucket_pw": self.bucket_pw()}

    def bucket_pw(self) -> dict:
        """Autotuned panel width per size bucket {smallest n: width}, width 0 = the launch's."""
        out = np.zeros(8, dtype=np.int32)
        _check("lu2gpu_batch_bucket_pw", lib().lu2gpu_batch_bucket_pw(self._h, _ptr(out)))
        return {int(out[2 * k]): int(out[2 * k + 1]) for k in range(4)}

    def solve(self) -> np.ndarray:
        info = np.zeros(self.count, dtype=np.int32)
        _check("lu2gpu_batch_solve", lib().lu2gpu_batch_solve(self._h, _ptr(info)))
        return info

    def residuals(self) -> np.ndarray:
        out = np.zeros(self.count, dtype=np.float64)
        _check("lu2gpu_batch_residuals", lib().lu2gpu_batch_residuals(self._h, _ptr(out)))
        return out


def device_ld(n: int, nrhs: int = 1) -> int:
    """A row stride for device matrices: >= n + nrhs, even, 128-byte rows."""
    return ((n + nrhs + 15) // 16) * 16

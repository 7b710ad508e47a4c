"""CPU simulation of the precision forms' factorization (test
infrastructure): lu2's blocked LU of an FP32 copy of A whose top-level
trailing updates C -= L21 U12 take their operands rounded to E4M3 with one
power-of-two scale per 128 x 128 tile (the FP8 form) or to BF16 with one
power-of-two scale per operand block (the BF16 form), products accumulated
in FP32 -- the arithmetic of lu2gpu_lowp_factor (kernels_fp8.cu's tile
scale: the largest 2^k with max|tile| 2^k <= 448; CUDA's E4M3 conversion
rounds to nearest even and saturates).  The panels are factored exactly in
FP32, with lu2's pivot-row scaling (lu2tlib.c:1057-1059: the U rows carry
1/pivot, the L columns the unscaled eliminated values).

Also: the conversion of lu2's factor storage (lu2.c:1088-1144: pivot rows of
a panel scaled by 1/pivot across the panel, earlier panels' L columns not
swapped by later panels) to P A = L U, the backward error, and
rho = ||I - M^-1 A||_2 (power iteration) of the preconditioner M = L U that
GMRES-IR uses: GMRES(30)-IR contracts reliably only for rho well below 1."""
from __future__ import annotations

import numpy as np


def e4m3(x: np.ndarray) -> np.ndarray:
    """Round to the nearest E4M3 value (ties to even), saturating at +-448."""
    x = np.asarray(x, dtype=np.float64)
    ax = np.abs(x)
    e = np.floor(np.log2(np.where(ax > 0, ax, 1.0)))
    e = np.clip(e, -6, 8)                 # subnormals below 2^-6 share the 2^-9 quantum
    q = np.exp2(e - 3)
    r = np.minimum(np.round(ax / q) * q, 448.0)
    return np.where(ax > 0, np.sign(x) * r, 0.0)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (nearest, ties to even)."""
    b = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def tile_exponent(amax: float) -> int:
    """k of kernels_fp8.cu: the largest power of two with amax 2^k <= 448."""
    if not amax > 0:
        return 0
    mant, e = np.frexp(amax)
    k = 8 - (e - 1) if 2 * mant <= 1.75 else 7 - (e - 1)
    return int(min(126, max(-126, k)))


def quant_fp8_tiles(x: np.ndarray) -> np.ndarray:
    """x (rows x cols, cols a multiple of 128) quantized per 128 x 128 tile and dequantized."""
    out = np.empty(x.shape, dtype=np.float32)
    rows, cols = x.shape
    for r0 in range(0, rows, 128):
        for c0 in range(0, cols, 128):
            t = x[r0:r0 + 128, c0:c0 + 128].astype(np.float32)
            k = tile_exponent(float(np.abs(t).max()))
            out[r0:r0 + 128, c0:c0 + 128] = (e4m3(t.astype(np.float64) * 2.0**k) * 2.0**-k).astype(np.float32)
    return out


def quant_bf16_block(x: np.ndarray) -> np.ndarray:
    """BF16 with one power-of-two scale for the whole block (the rounding is
    scale-invariant for powers of two, so only the rounding itself matters)."""
    return bf16(x).astype(np.float32)


def lowp_lu(a: np.ndarray, nb: int, update: str = "fp8"):
    """Factor the n x n matrix a (any float type) as lu2's precision forms do.
    Returns (L, U, perm) with a[perm] ~ L U, L lower with the pivots on its
    diagonal (lu2's unscaled columns), U unit upper; update in {"fp8",
    "fp8x2" (a two-term E4M3 split of each operand), "bf16", "fp32"}."""
    n = a.shape[0]
    w_ = a.astype(np.float32).copy()
    perm = np.arange(n)
    for i in range(0, n, nb):
        w = min(nb, n - i)
        for c in range(i, i + w):  # the panel, exactly in FP32
            p = c + int(np.argmax(np.abs(w_[c:, c])))
            if p != c:
                w_[[c, p]] = w_[[p, c]]
                perm[[c, p]] = perm[[p, c]]
            d = w_[c, c]
            inv = np.float32(1.0) / d if d != 0 else np.float32(1.0)
            w_[c, c + 1:i + w] *= inv
            w_[c + 1:, c + 1:i + w] -= np.outer(w_[c + 1:, c], w_[c, c + 1:i + w])
        if i + w >= n:
            break
        # block row: U12 = L11^-1 X (L11 unit lower: the unscaled column values
        # over their pivots), then lu2's 1/pivot on each row
        dg = np.diag(w_[i:i + w, i:i + w]).astype(np.float64)
        dg = np.where(dg == 0, 1.0, dg)
        l11 = np.tril(w_[i:i + w, i:i + w], -1).astype(np.float64) / dg[None, :] + np.eye(w)
        x = w_[i:i + w, i + w:].astype(np.float64)
        u12 = (np.linalg.solve(l11, x) / dg[:, None]).astype(np.float32)
        w_[i:i + w, i + w:] = u12
        l21 = w_[i + w:, i:i + w]
        if update == "fp8":
            lq, uq = quant_fp8_tiles(l21), quant_fp8_tiles(u12.T).T
        elif update == "fp8x2":  # two-term split hi + lo, products hi*hi + hi*lo + lo*hi
            lh, uh = quant_fp8_tiles(l21), quant_fp8_tiles(u12.T).T
            ll, ul = quant_fp8_tiles(l21 - lh), quant_fp8_tiles((u12 - uh).T).T
            w_[i + w:, i + w:] -= lh @ uh + lh @ ul + ll @ uh
            continue
        elif update == "bf16":
            lq, uq = quant_bf16_block(l21), quant_bf16_block(u12)
        else:
            lq, uq = l21, u12
        w_[i + w:, i + w:] -= lq @ uq
    lo = np.tril(w_).astype(np.float64)
    up = np.triu(w_, 1).astype(np.float64) + np.eye(n)
    return lo, up, perm


def lu2_factors_to_plu(f: np.ndarray, ipiv: np.ndarray, nb: int):
    """lu2's storage (f: n x n factors, ipiv: 0-based LAPACK-order pivots,
    panels of nb columns) to (L, U, perm) with a[perm] = L U, L lower with the
    pivots on its diagonal, U unit upper."""
    n = f.shape[0]
    g = f.astype(np.float64).copy()
    perm = np.arange(n)
    for k in range(n):
        p = int(ipiv[k])
        perm[[k, p]] = perm[[p, k]]
        c0 = (k // nb) * nb  # later panels never swapped the L columns of earlier ones
        if p != k and c0 > 0:
            g[[k, p], :c0] = g[[p, k], :c0]
    for r in range(n):  # a panel's pivot rows carry 1/pivot left of the diagonal too
        c0 = (r // nb) * nb
        g[r, c0:r] *= g[r, r]
    return np.tril(g), np.triu(g, 1) + np.eye(n), perm


def backward_error(a: np.ndarray, lo: np.ndarray, up: np.ndarray, perm: np.ndarray) -> float:
    """||a[perm] - L U||_inf / ||a||_inf"""
    return float(np.abs(a[perm] - lo @ up).sum(1).max() / np.abs(a).sum(1).max())


def precond_rho(a: np.ndarray, lo: np.ndarray, up: np.ndarray, perm: np.ndarray, iters: int = 30,
                seed: int = 0) -> float:
    """Power-iteration estimate of ||I - M^-1 a||_2 with M = P^T L U."""
    import scipy.linalg as sl

    n = a.shape[0]
    inv = np.empty(n, dtype=int)
    inv[perm] = np.arange(n)
    v = np.random.default_rng(seed).standard_normal(n)
    v /= np.linalg.norm(v)

    def op(x):
        y = a @ x
        z = sl.solve_triangular(lo, y[perm], lower=True)
        z = sl.solve_triangular(up, z, lower=False, unit_diagonal=True)
        return x - z

    def opt(x):  # the transpose of op
        z = sl.solve_triangular(up, x, lower=False, unit_diagonal=True, trans=1)
        z = sl.solve_triangular(lo, z, lower=True, trans=1)
        y = np.empty(n)
        y[perm] = z
        return x - a.T @ y

    s = 0.0
    for _ in range(iters):
        w = opt(op(v))
        s = np.linalg.norm(w)
        if not np.isfinite(s) or s == 0:
            return float(s)
        v = w / s
    return float(np.sqrt(s))

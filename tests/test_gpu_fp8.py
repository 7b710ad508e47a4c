"""FP8 form on the GPU: the tcgen05 E4M3 trailing update (per-128x128-tile
power-of-two scales, FP32 accumulation) against a float64 product of the
dequantized operands, the quantizer against the E4M3 format's bounds, and
GMRES-IR (FP64 refinement, GMRES(30) preconditioned by the low-precision
factors) on diagonally dominant and general systems."""
import numpy as np
import pytest

import lu2_b200 as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(300, 200, 256), (128, 128, 128), (1000, 129, 256), (4097, 515, 128)])
def test_fp8_update_matches_dequantized_product(ctx, M, N, K):
    import torch

    g = torch.Generator(device="cuda").manual_seed(M * 7 + N + K)
    a = (torch.rand((M, K), device="cuda", generator=g) - 0.5) * 3.0
    a[: min(M, 128), :128] *= 1e-3  # tiles of very different magnitude get their own scales
    bt = torch.rand((N, K), device="cuda", generator=g) - 0.5
    ldc = ((N + 3) // 4) * 4 + 4
    c = torch.rand((M, ldc), device="cuda", generator=g, dtype=torch.float32) - 0.5
    c0 = c.clone()
    ad = torch.zeros((M, K), device="cuda")
    bd = torch.zeros((N, K), device="cuda")
    ctx.fp8_update(M, N, K, a, K, bt, K, c, ldc, ad, bd)
    torch.cuda.synchronize()
    # quantization: E4M3 keeps 4 significant bits (relative error <= 2^-4) for
    # values within the tile scale's normal range
    for x, xd in ((a, ad), (bt, bd)):
        rel = ((x - xd).abs() / x.abs().clamp_min(1e-30))
        big = x.abs() > x.abs().max() * 2.0**-6  # inside E4M3's normal range for any tile
        assert float(rel[big].max()) <= 2.0**-4 + 1e-6
    ref = c0.double()
    ref[:, :N] -= ad.double() @ bd.double().T
    # products of E4M3 values are exact in FP32; the bound allows for the
    # tensor cores' FP32 accumulation order (and reduced-precision internal
    # accumulation), far below the quantization error itself (2^-4)
    bound = 1e-6 * K * (ad.double().abs() @ bd.double().abs().T) + 1e-6
    err = (c.double()[:, :N] - ref[:, :N]).abs()
    assert bool((err <= bound).all()), float(err.max())
    assert torch.equal(c[:, N:], c0[:, N:])  # padding columns untouched


def test_fp8_update_rejects_bad_k(ctx):
    import torch

    a = torch.zeros((128, 192), device="cuda")
    with pytest.raises(L.Lu2GpuError):
        ctx.fp8_update(128, 128, 192, a, 192, a, 192, a, 192)


def _system(ctx, n, seed, kind):
    import torch

    ld = L.device_ld(n, 1)
    a = torch.zeros((n, ld), dtype=torch.float64, device="cuda")
    ctx.generate(a, n, ld, seed, 1, kind=kind)
    b = a[:, n].clone()
    return a, ld, b


@pytest.mark.parametrize("n,nb,update", [(2048, 256, L.UPDATE_FP8), (1500, 128, L.UPDATE_FP8),
                                         (2048, 256, L.UPDATE_BF16)])
def test_gmres_ir_diagonally_dominant(ctx, n, nb, update):
    import scipy.linalg as sl
    import torch

    a, ld, b = _system(ctx, n, 23, kind=1)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    res = ctx.gmres_solve(a, n, ld, b, x, nb, update=update, restart=30, max_iter=100)
    assert res["status"] == 0, res
    assert res["hpl"] < 16 and res["gmres_iterations"] <= 20
    a0 = a.cpu().numpy()
    xs = sl.solve(a0[:, :n], a0[:, n])
    assert np.abs(x.cpu().numpy() - xs).max() / np.abs(xs).max() < 1e-10


def test_gmres_ir_bf16_general_matrix(ctx):
    """A general (not diagonally dominant) lu2 matrix: BF16 trailing updates
    leave a preconditioner that GMRES(30) still converges with at n = 1024."""
    import scipy.linalg as sl
    import torch

    n = 1024
    a, ld, b = _system(ctx, n, 1, kind=0)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    res = ctx.gmres_solve(a, n, ld, b, x, 256, update=L.UPDATE_BF16, restart=30, max_iter=400)
    assert res["status"] == 0, res
    a0 = a.cpu().numpy()
    xs = sl.solve(a0[:, :n], a0[:, n])
    assert np.abs(x.cpu().numpy() - xs).max() / np.abs(xs).max() < 1e-9


def test_gmres_ir_fp8_general_matrix_reports_no_convergence(ctx):
    """With E4M3 trailing updates (3 mantissa bits) the factors of a general
    uniform matrix are too far from A for GMRES(30) to converge (the
    perturbation times cond(A) is far above 1); the solver stops at its
    iteration budget and says so instead of returning a wrong x silently."""
    import torch

    n = 1024
    a, ld, b = _system(ctx, n, 1, kind=0)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    res = ctx.gmres_solve(a, n, ld, b, x, 256, update=L.UPDATE_FP8, restart=30, max_iter=60)
    assert res["status"] == -6 and res["hpl"] >= 16 and res["gmres_iterations"] == 60


def test_gmres_ir_rejects_bad_arguments(ctx):
    import torch

    n = 256
    a, ld, b = _system(ctx, n, 1, kind=1)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    for kw in ({"nb": 64, "update": L.UPDATE_FP8}, {"nb": 256, "update": 7}, {"nb": 256, "restart": 40}):
        args = {"nb": 256, "update": L.UPDATE_FP8, "restart": 30}
        args.update(kw)
        with pytest.raises(L.Lu2GpuError):
            ctx.gmres_solve(a, n, ld, b, x, args["nb"], update=args["update"], restart=args["restart"])


@pytest.mark.parametrize("kind,update,upd", [("general", L.UPDATE_FP8, "fp8"), ("dd", L.UPDATE_FP8, "fp8"),
                                             ("general", L.UPDATE_BF16, "bf16")])
def test_lowp_factors_match_the_cpu_simulation(ctx, oracle, kind, update, upd):
    """The GPU's precision-form factors (lu2gpu_lowp_factor) against the CPU
    simulation of the same arithmetic (tests/lowp_lu_sim.py) at n = 2048:
    backward error ||P A - L U|| / ||A|| within a factor 2 of the
    simulation's (the two differ only in FP32 rounding order, which moves
    single E4M3 roundings), and the same verdict on the preconditioner: for a
    general matrix with E4M3 updates ||I - M^-1 A|| >> 1 (the divergence the
    FP8 form reports), for a diagonally dominant one << 1."""
    import os
    import sys

    import torch

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from lowp_lu_sim import backward_error, lowp_lu, lu2_factors_to_plu, precond_rho

    n, nb = 2048, 256
    a, ld, _ = _system(ctx, n, 1, kind=1 if kind == "dd" else 0)
    f = torch.empty((n, n), dtype=torch.float32, device="cuda")
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert ctx.lowp_factor(a, n, ld, nb, update, f, n, ipiv) == 0
    a0 = a.cpu().numpy()[:, :n]
    lo, up, perm = lu2_factors_to_plu(f.cpu().numpy(), ipiv.cpu().numpy(), nb)
    be_gpu = backward_error(a0, lo, up, perm)
    rho_gpu = precond_rho(a0, lo, up, perm, iters=10)
    slo, sup, sperm = lowp_lu(a0, nb, upd)
    be_sim = backward_error(a0, slo, sup, sperm)
    print("lowp %s %s n=%d: backward error gpu %.3e sim %.3e, ||I - M^-1 A|| gpu %.3g" % (upd, kind, n, be_gpu, be_sim,
                                                                                        rho_gpu))
    assert be_sim / 2 < be_gpu < 2 * be_sim
    if kind == "dd":
        assert rho_gpu < 1e-2
    else:
        assert rho_gpu > 10

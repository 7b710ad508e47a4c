"""Batching form on the GPU: many uneven systems in one persistent launch
(replayed from a CUDA graph), each checked by its HPL scaled residual and
against an FP64 LAPACK solve; the generator against the oracle's lu2 stream."""
import ctypes

import numpy as np
import pytest

import lu2_b200 as L

pytestmark = pytest.mark.gpu


_CUDART = None


def _cudart():
    """The CUDA runtime (the process's CUDA context is torch's / the library's primary context)."""
    global _CUDART
    if _CUDART is None:
        import glob

        _CUDART = ctypes.CDLL(sorted(glob.glob("/usr/local/cuda/lib64/libcudart.so*"))[0])
    return _CUDART


def _memcpy_d2h(dst: np.ndarray, src_ptr: int) -> None:
    # the batch's copies run on the context's own stream; wait for them first
    assert _cudart().cudaDeviceSynchronize() == 0
    rc = _cudart().cudaMemcpy(ctypes.c_void_p(dst.ctypes.data), ctypes.c_void_p(src_ptr), ctypes.c_size_t(dst.nbytes),
                              2)
    assert rc == 0


def fetch(batch, i):
    """System i (n x (n+nrhs)) copied to the host."""
    ptr, ld = batch.system(i)
    n, r = int(batch.n[i]), int(batch.nrhs[i])
    host = np.zeros((n, ld), dtype=np.float64)
    _memcpy_d2h(host, ptr)
    return host[:, : n + r]


@pytest.fixture(scope="module")
def small_batch(ctx):
    n, r = L.batch_sizes(300, 7, 16, 512, 0.1, 8)
    b = L.Batch(ctx, n, r)
    b.generate(1000)
    b.snapshot()
    yield b
    b.close()


def test_batch_generator_is_lu2_stream(ctx, oracle, small_batch):
    for i in (0, 1, 17, 299):
        n, r = int(small_batch.n[i]), int(small_batch.nrhs[i])
        host = fetch(small_batch, i)
        ref = oracle.randomsetmat(n, 1000 + i, nrhs=r)
        assert np.array_equal(host, ref[:, : n + r])


def test_batch_solve_residuals_and_lapack(ctx, small_batch):
    import scipy.linalg as sl

    small_batch.restore()
    info = small_batch.solve()
    assert (info == 0).all()
    res = small_batch.residuals()
    assert (res < 16).all(), res.max()
    orig = {}
    for i in (0, 5, 123, 299):
        n, r = int(small_batch.n[i]), int(small_batch.nrhs[i])
        x = fetch(small_batch, i)[:, n:n + r]
        small_batch.restore()
        a0 = fetch(small_batch, i)
        orig[i] = (a0, x)
        xs = sl.solve(a0[:, :n], a0[:, n:n + r])
        assert np.abs(x - xs).max() / np.abs(xs).max() < 1e-10
        small_batch.solve()


@pytest.mark.parametrize("threads,pw,ctas", [(128, 16, 1), (256, 32, 1), (512, 32, 1), (256, 16, 2)])
def test_batch_launch_shapes(ctx, small_batch, threads, pw, ctas):
    small_batch.set_config(threads, pw, ctas)
    small_batch.restore()
    assert (small_batch.solve() == 0).all()
    assert (small_batch.residuals() < 16).all()


def test_batch_bucket_widths_reset_by_set_config(ctx, small_batch):
    """A per-bucket panel width from the autotuner is dropped by set_config
    (one width for every system again); the solve stays correct."""
    small_batch.autotune()
    small_batch.set_config(256, 16, 2)
    assert all(w == 0 for w in small_batch.bucket_pw().values())
    small_batch.restore()
    assert (small_batch.solve() == 0).all()
    assert (small_batch.residuals() < 16).all()


def test_batch_panel_too_wide_is_rejected(ctx, small_batch):
    """n = 510 with a 64-column panel needs more than 220 KB of shared memory."""
    with pytest.raises(L.Lu2GpuError):
        small_batch.set_config(512, 64, 1)


def test_batch_wide_panel_blocked_path(ctx):
    """Systems up to n = 300 with 64-column panels; the larger ones take the
    blocked path, several right-hand sides exercise the blocked back substitution."""
    n = np.array([300, 257, 200, 150, 64, 16], dtype=np.int32)
    r = np.array([1, 8, 3, 1, 64, 2], dtype=np.int32)
    b = L.Batch(ctx, n, r)
    b.generate(77)
    b.snapshot()
    b.set_config(512, 64, 1)
    assert (b.solve() == 0).all()
    assert (b.residuals() < 16).all()
    b.close()


def test_batch_autotune_then_graph_replay(ctx, small_batch):
    cfg = small_batch.autotune()
    assert cfg["threads"] in (128, 256, 512) and cfg["pw"] in (16, 32, 64)
    assert sorted(cfg["bucket_pw"]) == [1, 64, 128, 256]
    assert all(w in (0, 16, 32, 64) for w in cfg["bucket_pw"].values())
    for _ in range(2):  # second call replays the captured graph
        small_batch.restore()
        assert (small_batch.solve() == 0).all()
        assert (small_batch.residuals() < 16).all()


def test_batch_zero_pivot_reported(ctx):
    import torch

    b = L.Batch(ctx, np.array([40, 33], dtype=np.int32))
    b.generate(5)
    ptr, ld = b.system(1)
    # zero column 7 of system 1 through a device tensor view
    host = np.zeros((33, ld))
    _memcpy_d2h(host, ptr)
    host[:, 7] = 0.0
    cudart = _cudart()
    assert cudart.cudaMemcpy(ctypes.c_void_p(ptr), ctypes.c_void_p(host.ctypes.data), ctypes.c_size_t(host.nbytes),
                             1) == 0
    torch.cuda.synchronize()
    info = b.solve()
    assert info[0] == 0 and info[1] == 8
    b.close()


def test_batch_on_legacy_default_stream():
    """A context on the legacy default stream (as torch's current stream is by
    default): the graph is captured on the batch's own stream and launched there."""
    c = L.Context(0)
    c.set_stream(0)
    n, r = L.batch_sizes(64, 3, 16, 200, 0.2, 4)
    b = L.Batch(c, n, r)
    b.generate(9)
    b.snapshot()
    for _ in range(2):
        b.restore()
        assert (b.solve() == 0).all()
        assert (b.residuals() < 16).all()
    b.close()
    c.close()


@pytest.fixture(scope="module")
def ir_batch(ctx):
    n, r = L.batch_sizes(300, 11, 16, 512, 0.1, 8)
    b = L.Batch(ctx, n, r)
    b.generate(2000)
    b.snapshot()
    b.set_mode(L.BATCH_FP32_IR, 10)
    yield b
    b.close()


def test_batch_fp32_ir_reaches_fp64_residual(ctx, ir_batch):
    """FP32 factors + FP64 refinement: every system (blocked and in-shared-
    memory paths, 1 and 8 right-hand sides) reaches HPL < 16 and matches an
    FP64 LAPACK solve."""
    import scipy.linalg as sl

    ir_batch.restore()
    info = ir_batch.solve()
    assert (info == 0).all()
    res = ir_batch.residuals()
    assert (res < 16).all(), res.max()
    its = ir_batch.iterations()
    assert its.min() >= 1 and its.max() <= 6, (its.min(), its.max())
    for i in (0, 3, 150, 299):
        n, r = int(ir_batch.n[i]), int(ir_batch.nrhs[i])
        x = fetch(ir_batch, i)[:, n:n + r]
        ir_batch.restore()
        a0 = fetch(ir_batch, i)
        xs = sl.solve(a0[:, :n], a0[:, n:n + r])
        assert np.abs(x - xs).max() / np.abs(xs).max() < 1e-9
        ir_batch.solve()


@pytest.mark.parametrize("threads,pw,ctas", [(128, 16, 1), (512, 32, 1), (256, 16, 2)])
def test_batch_fp32_ir_launch_shapes(ctx, ir_batch, threads, pw, ctas):
    ir_batch.set_config(threads, pw, ctas)
    ir_batch.restore()
    assert (ir_batch.solve() == 0).all()
    assert (ir_batch.residuals() < 16).all()


def test_batch_fp32_ir_autotune_and_replay(ctx, ir_batch):
    cfg = ir_batch.autotune()
    assert cfg["threads"] in (128, 256, 512)
    for _ in range(2):
        ir_batch.restore()
        assert (ir_batch.solve() == 0).all()
        assert (ir_batch.residuals() < 16).all()


def test_batch_fp32_ir_rejects_many_rhs(ctx):
    b = L.Batch(ctx, np.array([32, 40], dtype=np.int32), np.array([1, 9], dtype=np.int32))
    with pytest.raises(L.Lu2GpuError):
        b.set_mode(L.BATCH_FP32_IR, 10)
    b.close()


def test_objects_left_open_at_exit_are_closed_in_order():
    """A script that leaves a context and a batch open (module globals) exits
    cleanly: the binding closes batches before contexts while the CUDA
    runtime is still up, and a batch keeps its context alive."""
    import os
    import subprocess
    import sys

    code = ("import numpy as np, lu2_b200 as L\n"
            "ctx = L.Context(0)\n"
            "b = L.Batch(ctx, np.array([40, 300], dtype=np.int32))\n"
            "b.generate(1)\n"
            "assert (b.solve() == 0).all()\n"
            "ctx2 = L.Context(0)\n"
            "b2 = L.Batch(ctx2, np.array([17], dtype=np.int32))\n"
            "del ctx2\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stderr[-2000:])

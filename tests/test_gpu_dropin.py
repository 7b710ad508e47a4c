"""The reference's own programs on the GPU (see tests/test_dropin.py for how
they are linked): lu2's main with the library's lumcolumn, lu2's GDR build
with the library as its board, and the GDR build's panel loop through the
harness compared with the all-CPU reference on the same input."""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle.oracle import RefLib

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def run_program(name, args, env_extra=None, timeout=600):
    path = os.path.join(REF, name)
    if not os.path.exists(path):
        pytest.fail("%s not built" % path)
    env = dict(os.environ, LU2GPU_REPORT="1", **(env_extra or {}))
    r = subprocess.run(["bash", "-c", "ulimit -s unlimited; exec %s %s" % (path, args)], capture_output=True,
                       text=True, timeout=timeout, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    emax = float(re.search(r"Emax=\s*(\S+)", r.stdout).group(1))
    launches = int(re.search(r"lu2gpu: (\d+) kernel launches", r.stderr).group(1))
    gflops = float(re.search(r"([0-9.eE+-]+) Gflops", r.stdout).group(1))
    return emax, launches, gflops, r


def cpu_emax(variant, n, nb, seed, oracle):
    ref = RefLib(variant)
    ref.set_threads(os.cpu_count() or 1, 1)
    x, piv, _ = ref.factor_solve(n, nb, seed)
    return oracle.residual(oracle.randomsetmat(n, seed), n, x)["rinf"], x, piv


def test_lu2_main_runs_the_library_lumcolumn(oracle):
    """lu2.c's main, unchanged, at its default block size (nb = 2048): the
    factorization and solve run on the GPU (partial pivoting), Emax as small
    as the pivot-fixed CPU reference's."""
    n, nb = 4096, 2048
    emax, launches, gflops, r = run_program("lu2_gpu", "-n %d -b %d -s 1" % (n, nb))
    e_fixed, _, _ = cpu_emax("fixed", n, nb, 1, oracle)
    print("lu2_gpu n=%d nb=%d: Emax %.3e (fixed CPU reference %.3e), %d launches, %.1f GFLOP/s"
          % (n, nb, emax, e_fixed, launches, gflops))
    assert launches > 1000
    assert emax < 10 * e_fixed


def test_lu2_main_reference_pivoting_through_the_environment(oracle):
    """LU2GPU_PIVOT=ref reaches the library through lu2's unchanged main: the
    bug-compatible pivots (lu2tlib.c:1052) raise Emax far above the
    partial-pivoting run's, and it stays below the shipped CPU build's own
    (same pivots; that build also inverts L11 explicitly, lu2.c:370-483,
    which amplifies the large multipliers those pivots produce)."""
    n, nb = 4096, 2048
    emax, launches, _, _ = run_program("lu2_gpu", "-n %d -b %d -s 1" % (n, nb), {"LU2GPU_PIVOT": "ref"})
    e_partial, _, _, _ = run_program("lu2_gpu", "-n %d -b %d -s 1" % (n, nb))
    e_shipped, _, _ = cpu_emax("shipped", n, nb, 1, oracle)
    print("lu2_gpu LU2GPU_PIVOT=ref: Emax %.3e (partial pivoting %.3e, shipped CPU reference %.3e)"
          % (emax, e_partial, e_shipped))
    assert launches > 1000
    assert 10 * e_partial < emax < 10 * e_shipped


def test_lu2_gdr_build_with_the_gpu_as_its_board(oracle):
    """lu2's GDR build (GDR mode needs nb >= 2048, lu2lib.c:2142-2145): its
    self-test (gdr_check_and_restart) passes on the GPU, every product with
    k > 512 goes through gdr_dgemm_ (no fallback message), and Emax matches
    the all-CPU build's."""
    n, nb = 4096, 2048
    emax, launches, _, r = run_program("lu2_gdr", "-n %d -b %d -s 1" % (n, nb))
    assert "gdr_check_and_restart passed 0" in r.stderr
    assert "failed" not in r.stderr
    e_shipped, _, _ = cpu_emax("shipped", n, nb, 1, oracle)
    print("lu2_gdr n=%d nb=%d: Emax %.3e (all-CPU shipped reference %.3e), %d launches"
          % (n, nb, emax, e_shipped, launches))
    assert launches > 0
    assert e_shipped / 10 < emax < 10 * e_shipped


def test_gdr_build_panel_loop_matches_cpu_build(oracle, parity):
    """The GDR build's per-panel loop through the harness (its DGEMMs with
    k > 512 on the GPU board, the rest on the CPU) against the all-CPU
    build on the same input: pivots index for index, x within 4 d_ref of it
    (the shipped algorithm's own forward error, as in tests/test_gpu_lu.py)."""
    import lu2_b200 as L
    import scipy.linalg as sl

    n, nb, seed = 4096, 2048, 1
    lib = L.load()
    k0 = lib.lu2gpu_kernel_launches()
    gdr = RefLib("gdr")
    gdr.set_threads(os.cpu_count() or 1, 1)
    xg, pg, _ = gdr.factor_solve(n, nb, seed)
    assert lib.lu2gpu_kernel_launches() > k0, "no GPU kernel ran"
    _, xc, pc = cpu_emax("shipped", n, nb, seed, oracle)
    mism = int((pg != pc).sum())
    a0 = oracle.randomsetmat(n, seed)
    A, b = a0[:, :n], a0[:, n]
    lu = sl.lu_factor(A)
    xhp = sl.lu_solve(lu, b).astype(np.longdouble)
    for _ in range(3):
        xhp = xhp + sl.lu_solve(lu, (b.astype(np.longdouble) - A.astype(np.longdouble) @ xhp).astype(np.float64))
    xhp = xhp.astype(np.float64)
    d_ref = np.abs(xc - xhp).max() / np.abs(xhp).max()
    assert mism == 0, "%d pivot mismatches" % mism
    parity("lu2_gdr panel loop vs all-CPU shipped n=%d nb=%d" % (n, nb), np.abs(xg - xc).max() / np.abs(xc).max(),
           4 * d_ref, "fwd err ref %.2e" % d_ref)

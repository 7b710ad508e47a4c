"""The reference's own programs linked against liblu2gpu.so without editing
any reference source (oracle/build_oracle.py:build_dropin):

* lu2_gdr: lu2's GDR build (Makefile.common:69-70, 87-88) with the library
  in place of the GRAPE-DR board library;
* lu2_gpu: lu2.c's main whose lumcolumn call binds to the library's.

Here (no GPU needed) the binding is checked: which objects define which
symbols, and that lu2_gpu's main really calls into the library (without a
GPU the library's lumcolumn reports the missing device and exits, as the
reference's MP_error does)."""
import os
import subprocess

import pytest

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")
LU2_GDR = os.path.join(REF, "lu2_gdr")
LU2_GPU = os.path.join(REF, "lu2_gpu")
needs = pytest.mark.skipif(not (os.path.exists(LU2_GDR) and os.path.exists(LU2_GPU)),
                           reason="drop-in binaries not built (reference checkout absent at build time)")


def symbols(path):
    out = subprocess.run(["nm", path], capture_output=True, text=True, check=True).stdout
    table = {}
    for line in out.splitlines():
        parts = line.split()
        table[parts[-1]] = parts[-2]
    return table


@needs
def test_gdr_build_keeps_its_own_gdrdgemm_and_takes_the_board_from_the_library():
    """gdrdgemm.c's definitions (gdrblas_dgemm, mygdrdgemm,
    gdr_check_and_restart) are the program's own; only the board symbols come
    from liblu2gpu.so.  The library is linked -Bsymbolic, so its own calls
    never bind to the program's same-named functions."""
    t = symbols(LU2_GDR)
    for own in ("gdrblas_dgemm", "mygdrdgemm", "gdr_check_and_restart", "mydgemm", "lumcolumn"):
        assert t.get(own) == "T", own
    for board in ("gdr_dgemm_", "gdr_init", "gdr_free", "gdrdgemm_set_procname"):
        assert t.get(board) == "U", board


@needs
def test_lu2_main_binds_lumcolumn_to_the_library():
    t = symbols(LU2_GPU)
    assert t.get("lumcolumn") == "U"      # from liblu2gpu.so
    assert t.get("lumcolumn_cpu") == "T"  # the forwarding definition, not lu2.c's weakened one


@needs
def test_lu2_main_without_gpu_reaches_the_library():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present: tests/test_gpu_dropin.py runs the program")
    r = subprocess.run(["bash", "-c", "ulimit -s unlimited; exec %s -n 128 -b 64" % LU2_GPU], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 255, r.stderr
    assert "lu2gpu: lumcolumn failed" in r.stderr

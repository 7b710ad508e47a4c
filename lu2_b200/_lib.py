"""Loader for the in-tree liblu2gpu.so (the CUDA library behind the C ABI in
include/lu2gpu.h).  There is no fallback: if the library is missing the import
of the binding fails loudly."""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "liblu2gpu.so")
HEADER = os.path.join(ROOT, "include", "lu2gpu.h")

_lib = None

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)
vp = C.c_void_p

# argtypes of every exported function (names as in include/lu2gpu.h)
SIGNATURES = {
    "lumcolumn": (None, [C.c_int, vp, vp, C.c_int, vp, vp, C.c_int]),
    "column_decomposition_recursive": (None, [C.c_int, vp, C.c_int, vp, vp, C.c_int]),
    "process_right_part": (None, [C.c_int, vp, C.c_int, vp, vp, C.c_int, C.c_int]),
    "backward_sub": (None, [C.c_int, vp, vp]),
    "cm_column_decomposition_recursive": (None, [C.c_int, vp, C.c_int, vp, C.c_int]),
    "cm_column_decomposition": (None, [C.c_int, vp, C.c_int, vp, C.c_int]),
    "cm_process_right_part": (None, [C.c_int, vp, C.c_int, vp, C.c_int, C.c_int]),
    "mydgemm": (None, [C.c_int, C.c_int, C.c_int, C.c_double, vp, C.c_int, vp, C.c_int, C.c_double, vp, C.c_int]),
    "matmul_for_small_nk": (None, [C.c_int, vp, C.c_int, vp, C.c_int, vp, C.c_int, C.c_int, C.c_int]),
    "reset_gdr": (None, [C.c_int, vp, C.c_int, vp, C.c_int]),
    "gdrsetboardid": (None, [C.c_int]),
    "gdrsetnboards": (None, [C.c_int]),
    "gdrsetforceswapab": (None, []),
    "gdrresetforceswapab": (None, []),
    "gdrsetskipsendjmat": (None, []),
    "gdrresetskipsendjmat": (None, []),
    "set_matmul_msg_level": (None, [C.c_int]),
    "gdrdgemm_set_stress_factor": (None, [C.c_int]),
    "gdr_dgemm_": (None, [ip, ip, ip, ip, ip, dp, dp, ip, ip, ip, vp, vp, vp, ip]),
    "gdr_init": (None, []),
    "gdr_free": (None, []),
    "gdrdgemm_set_procname": (None, [C.c_int]),
    "gdrblas_dgemm": (None, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, vp, C.c_int, vp,
                             C.c_int, C.c_double, vp, C.c_int]),
    "mygdrdgemm": (None, [C.c_int, C.c_int, C.c_int, C.c_double, vp, C.c_int, vp, C.c_int, C.c_double, vp, C.c_int]),
    "gdr_check_and_restart": (None, [vp, vp, vp]),
    "lu2gpu_create": (C.c_int, [C.POINTER(vp), C.c_int]),
    "lu2gpu_destroy": (C.c_int, [vp]),
    "lu2gpu_set_stream": (C.c_int, [vp, vp]),
    "lu2gpu_factor": (C.c_int, [vp, C.c_int, C.c_int, vp, C.c_long, C.c_int, C.c_int, vp]),
    "lu2gpu_backsolve": (C.c_int, [vp, C.c_int, C.c_int, vp, C.c_long, vp, C.c_long]),
    "lu2gpu_lusolve": (C.c_int, [vp, C.c_int, C.c_int, vp, C.c_long, C.c_int, C.c_int, vp]),
    "lu2gpu_solve": (C.c_int, [vp, C.c_int, vp, C.c_long, C.c_int, vp, vp, C.c_long, C.c_int]),
    "lu2gpu_mixed_solve": (C.c_int, [vp, C.c_int, vp, C.c_long, vp, vp, C.c_int, C.c_int, C.c_int, vp]),
    "lu2gpu_bf16_update_dev": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, C.c_long, vp, C.c_long, vp, C.c_long,
                                         C.c_float]),
    "lu2gpu_gmres_solve": (C.c_int, [vp, C.c_int, vp, C.c_long, vp, vp, C.c_int, C.c_int, C.c_int, C.c_double,
                                     C.c_int, vp]),
    "lu2gpu_fp8_update_dev": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, C.c_long, vp, C.c_long, vp, C.c_long,
                                        vp, vp]),
    "lu2gpu_batch_create": (C.c_int, [vp, C.c_int, vp, vp, C.POINTER(vp)]),
    "lu2gpu_batch_destroy": (C.c_int, [vp]),
    "lu2gpu_batch_system": (C.c_int, [vp, C.c_int, C.POINTER(vp), C.POINTER(C.c_long)]),
    "lu2gpu_batch_generate": (C.c_int, [vp, C.c_long]),
    "lu2gpu_batch_generate_seeds": (C.c_int, [vp, vp]),
    "lu2gpu_batch_snapshot": (C.c_int, [vp]),
    "lu2gpu_batch_restore": (C.c_int, [vp]),
    "lu2gpu_batch_set_config": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
    "lu2gpu_batch_set_mode": (C.c_int, [vp, C.c_int, C.c_int]),
    "lu2gpu_batch_iterations": (C.c_int, [vp, vp]),
    "lu2gpu_batch_autotune": (C.c_int, [vp, vp]),
    "lu2gpu_batch_bucket_pw": (C.c_int, [vp, vp]),
    "lu2gpu_batch_solve": (C.c_int, [vp, vp]),
    "lu2gpu_batch_residuals": (C.c_int, [vp, vp]),
    "lu2gpu_batch_sizes": (C.c_int, [C.c_int, C.c_long, C.c_int, C.c_int, C.c_double, C.c_int, vp, vp]),
    "lu2gpu_generate": (C.c_int, [vp, C.c_int, C.c_int, C.c_long, C.c_int, vp, C.c_long]),
    "lu2gpu_dgemm_dev": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_double, vp, C.c_long, vp, C.c_long,
                                   C.c_double, vp, C.c_long]),
    "lu2gpu_copy_pivots": (C.c_int, [vp, vp, C.c_int]),
    "lu2gpu_lumcolumn": (C.c_int, [C.c_int, vp, vp, C.c_int, vp, C.c_int]),
    "lu2gpu_default_context": (vp, []),
    "lu2gpu_release": (C.c_int, []),
    "lu2gpu_set_pivot_mode": (C.c_int, [C.c_int]),
    "lu2gpu_set_abort_on_error": (C.c_int, [C.c_int]),
    "lu2gpu_last_error": (C.c_char_p, []),
    "lu2gpu_set_timing": (C.c_int, [vp, C.c_int]),
    "lu2gpu_get_timers": (C.c_int, [vp, vp, vp, C.c_int, C.c_int]),
    "lu2gpu_timer_name": (C.c_char_p, [C.c_int]),
    "lu2gpu_kernel_launches": (C.c_long, []),
    "lu2gpu_lusolve_noalloc": (C.c_int, [C.c_int, C.c_int, vp, C.c_long, C.c_int, C.c_int, vp, vp]),
    "lu2gpu_test_leaf_withhold": (C.c_int, [vp, C.c_int, C.c_double]),
    "lu2gpu_swaprows_dev": (C.c_int, [vp, C.c_int, vp, C.c_long, C.c_int, C.c_int, vp, vp, C.c_int, C.c_int]),
    "lu2gpu_solve_triangle_dev": (C.c_int, [vp, C.c_int, vp, C.c_long, vp, C.c_long, C.c_int, vp]),
    "lu2gpu_lowp_factor": (C.c_int, [vp, C.c_int, vp, C.c_long, C.c_int, C.c_int, vp, C.c_long, vp]),
}


def header_functions(path: str = HEADER) -> list[str]:
    """Function names declared in include/lu2gpu.h."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-zA-Z_][a-zA-Z0-9_ ]*?\**\s*\**([a-zA-Z_][a-zA-Z0-9_]*)\s*\(", text, re.M)
    return [n for n in names if n not in ("if", "defined")]


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load liblu2gpu.so and declare its signatures.  Raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError("liblu2gpu.so not built (%s); run `python lu2_b200/build.py`" % path)
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    lib.lu2gpu_set_abort_on_error(0)
    _lib = lib
    return lib


def last_error() -> str:
    return (load().lu2gpu_last_error() or b"").decode()

"""The C-ABI library loads and exports every symbol include/lu2gpu.h declares
(no compute calls: this suite runs without a GPU)."""
import ctypes
import os
import subprocess

import pytest

from lu2_b200 import _lib


def test_library_built_for_sm100a():
    from lu2_b200 import build

    assert os.path.exists(_lib.LIB_PATH), "run lu2_b200/build.py"
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert not build._stale(), "liblu2gpu.so is older than its sources"


def test_exports_every_header_function(lib):
    names = _lib.header_functions()
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    names = set(_lib.header_functions())
    assert names == set(_lib.SIGNATURES), names ^ set(_lib.SIGNATURES)


def test_no_libcuda_link_dependency():
    out = subprocess.run(["readelf", "-d", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "libcuda.so" not in out
    assert "libtorch" not in out


def test_create_without_gpu_reports_nodev(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = lib.lu2gpu_create(ctypes.byref(h), 0)
    assert rc == -5
    assert "device" in _lib.last_error()


def test_header_status_codes_match_binding():
    text = open(_lib.HEADER).read()
    for name, val in [("LU2GPU_ERR_ARG", "(-1)"), ("LU2GPU_ERR_NODEV", "(-5)"), ("LU2GPU_PIVOT_REF", "0"),
                      ("LU2GPU_PIVOT_PARTIAL", "1")]:
        assert "#define %s %s" % (name, val) in text


def test_exit_hook_closes_batches_before_contexts(monkeypatch):
    """The binding's exit hook closes every batch still open before any
    context (a batch's memory and streams belong to its context).  Run on
    private registries, so that no real context of the session is touched."""
    import weakref

    from lu2_b200 import lu2

    order = []

    class Fake:
        def __init__(self, name):
            self.name = name

        def close(self):
            order.append(self.name)

    monkeypatch.setattr(lu2, "_LIVE_CONTEXTS", weakref.WeakSet())
    monkeypatch.setattr(lu2, "_LIVE_BATCHES", weakref.WeakSet())
    ctx, batch = Fake("context"), Fake("batch")
    lu2._LIVE_CONTEXTS.add(ctx)
    lu2._LIVE_BATCHES.add(batch)
    lu2._close_live()
    assert order == ["batch", "context"]

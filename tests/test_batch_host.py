"""Host-side logic of the batching form (no GPU needed): the size
distribution of the benchmark batch and argument checks."""
import ctypes

import numpy as np

import lu2_b200 as L


def test_batch_sizes_distribution():
    n, r = L.batch_sizes(20000, 1, 16, 512, 0.1, 8)
    assert n.min() >= 16 and n.max() <= 512
    assert abs(np.log(n).mean() - (np.log(16) + np.log(513)) / 2) < 0.05
    assert abs((r == 8).mean() - 0.1) < 0.01 and set(np.unique(r)) == {1, 8}


def test_batch_sizes_deterministic_and_seeded():
    a = L.batch_sizes(1000, 3)
    b = L.batch_sizes(1000, 3)
    c = L.batch_sizes(1000, 4)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])


def test_batch_sizes_rejects_bad_ranges():
    lib = L.load()
    n = np.zeros(4, dtype=np.int32)
    r = np.zeros(4, dtype=np.int32)
    p = lambda x: ctypes.c_void_p(x.ctypes.data)  # noqa: E731
    assert lib.lu2gpu_batch_sizes(4, 1, 0, 10, 0.1, 8, p(n), p(r)) == -1
    assert lib.lu2gpu_batch_sizes(4, 1, 20, 10, 0.1, 8, p(n), p(r)) == -1
    assert lib.lu2gpu_batch_sizes(0, 1, 16, 512, 0.1, 8, p(n), p(r)) == -1


def test_batch_create_rejects_without_context():
    lib = L.load()
    n = np.array([16, 32], dtype=np.int32)
    out = ctypes.c_void_p()
    assert lib.lu2gpu_batch_create(None, 2, ctypes.c_void_p(n.ctypes.data), None, ctypes.byref(out)) == -1
    assert not out.value

"""lu2_b200: B200-native (sm_100a) dense LU with partial pivoting and solve,
behind telmin/lu2's C entry points.  The compute path is liblu2gpu.so
(lu2_b200/csrc); this package is its host-side binding."""
from .lu2 import (  # noqa: F401
    CBLAS_COLMAJOR,
    CBLAS_NOTRANS,
    CBLAS_ROWMAJOR,
    CBLAS_TRANS,
    PIVOT_PARTIAL,
    PIVOT_REF,
    UPDATE_BF16,
    UPDATE_FP8,
    BATCH_FP64,
    BATCH_FP32_IR,
    Batch,
    Context,
    Lu2GpuError,
    batch_shard,
    batch_sizes,
    device_ld,
    gdr_dgemm_,
    gdrblas_dgemm,
    lumcolumn,
    mydgemm,
    mygdrdgemm,
    rdim,
    set_pivot_mode,
)
from ._lib import LIB_PATH, load  # noqa: F401

"""B200-native fast matrix multiplication (Strassen-like recursive algorithms).

The engine is libfmm.so (CUDA for sm_100a behind the C ABI in include/fmm.h);
this package builds it and exposes the reference's operator surface to
Python.  See api.py.
"""

from ._lib import FmmError, lib  # noqa: F401
from .api import (  # noqa: F401
    AUTO,
    CLASSICAL,
    INSIDE,
    INSIDE_OUTSIDE,
    OUTSIDE,
    OUTSIDE_INSIDE,
    Handle,
    Plan,
    Server,
    autotune,
    autotune_choice,
    autotune_load,
    autotune_table,
    autotune_tile,
    fast_matmul_batched,
    algorithm_index,
    algorithm_info,
    algorithm_names,
    colmajor_empty,
    default_handle,
    diagonal_scaling,
    fast_matmul,
    fast_matmul_host,
    fast_matmul_host_async,
    host_sync,
    matmul,
    matmul_split_bf16,
    matmul_split_int8,
    max_relative_diff,
    num_algorithms,
    random_matrix,
    scaling_postprocess,
    synchronize,
    workspace_bytes,
)

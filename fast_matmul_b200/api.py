"""Python surface of the engine, mirroring the reference's operator API.

The reference's user-facing calls are, per algorithm namespace,
``<ns>::FastMatmul(A, B, C, num_steps, x, alpha, beta)``
(algorithms/strassen.hpp:661-722), the classical ``MatMul(A, B, C, beta)``
(linalg/linalg.hpp:261-269), ``RandomMatrix`` (linalg/linalg.hpp:422-433) and
``MaxRelativeDiff`` (linalg/linalg.hpp:280-295).  The same names are exposed
here over column-major FP64 matrices held in CUDA memory as torch tensors
(``A.stride(0) == 1``, leading dimension ``A.stride(1)``); PyTorch only
provides the memory and the stream -- all arithmetic runs in libfmm.so.
"""

from __future__ import annotations

import ctypes
import threading
from typing import Dict, Optional, Tuple

from . import _lib
from ._lib import Options, check, lib


def _torch():
    import torch

    return torch


# ---------------------------------------------------------------------------
# algorithm registry


def num_algorithms() -> int:
    return lib().fmm_num_algorithms()


def algorithm_names():
    L = lib()
    return [L.fmm_algorithm_name(i).decode() for i in range(L.fmm_num_algorithms())]


def algorithm_index(name) -> int:
    """Index of an algorithm by namespace (``grey424_26_206``), header
    (``fast424_26_206.hpp``) or header stem (``fast424_26_206``)."""
    if isinstance(name, int):
        if not 0 <= name < num_algorithms():
            raise _lib.FmmError(2, "unknown algorithm index %d" % name)
        return name
    idx = lib().fmm_algorithm_lookup(name.encode())
    if idx < 0:
        raise _lib.FmmError(2, "unknown algorithm %r" % name)
    return idx


def algorithm_info(name) -> Dict[str, int]:
    idx = algorithm_index(name)
    vals = [ctypes.c_int() for _ in range(5)]
    check(lib().fmm_algorithm_info(idx, *[ctypes.byref(v) for v in vals]))
    m0, k0, n0, rank, approx = [v.value for v in vals]
    return {"index": idx, "name": lib().fmm_algorithm_name(idx).decode(), "m0": m0, "k0": k0, "n0": n0,
            "rank": rank, "approximate": bool(approx)}


# ---------------------------------------------------------------------------
# handles


class Handle:
    """An engine handle on one device (fmm_handle_create / fmm_handle_destroy)."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        check(lib().fmm_handle_create(ctypes.byref(self._h), device))
        self.device = device

    @property
    def ptr(self):
        return self._h

    def close(self):
        if self._h:
            lib().fmm_handle_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream_ptr: int):
        check(lib().fmm_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def bind_current_stream(self):
        torch = _torch()
        self.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def set_workspace_limit(self, nbytes: int):
        check(lib().fmm_set_workspace_limit(self._h, nbytes))

    def release_workspace(self):
        """Frees the handle's workspace and staging buffers (fmm_release_workspace)."""
        check(lib().fmm_release_workspace(self._h))

    def debug_fill_workspace(self, nbytes: int, pattern: int = 0xFF):
        """Grows the workspace to nbytes and fills it with a byte pattern (test support)."""
        check(lib().fmm_debug_fill_workspace(self._h, nbytes, pattern))

    def launches(self) -> int:
        return int(lib().fmm_kernel_launch_count(self._h))

    def synchronize(self):
        check(lib().fmm_synchronize(self._h))

    def profile(self, enable: bool = True):
        """Bracket every launch with CUDA events (per-phase timing)."""
        check(lib().fmm_profile_enable(self._h, 1 if enable else 0))

    def profile_reset(self):
        check(lib().fmm_profile_reset(self._h))

    def profile_read(self) -> dict:
        p = _lib.Profile()
        check(lib().fmm_profile_read(self._h, ctypes.byref(p)))
        return p.as_dict()


_tls = threading.local()


def default_handle(device: Optional[int] = None) -> Handle:
    """The calling thread's handle for `device`, bound to torch's current stream."""
    torch = _torch()
    if device is None:
        device = torch.cuda.current_device()
    handles = getattr(_tls, "handles", None)
    if handles is None:
        handles = _tls.handles = {}
    h = handles.get(device)
    if h is None:
        h = handles[device] = Handle(device)
    h.bind_current_stream()
    return h


# ---------------------------------------------------------------------------
# matrices


def colmajor_empty(m: int, n: int, device="cuda"):
    """Uninitialised column-major m x n FP64 matrix (leading dimension m)."""
    torch = _torch()
    return torch.empty((n, m), dtype=torch.float64, device=device).t()


F32_DEFAULT_SLICES = 5  # FMM_F32_DEFAULT_SLICES of include/fmm.h (split-INT8 slices)


def _mat(t, rows: int, cols: int, name: str, dtype=None) -> Tuple[int, int]:
    torch = _torch()
    want = torch.float64 if dtype is None else dtype
    if t.dtype != want:
        raise TypeError("%s must be %s" % (name, str(want).replace("torch.", "")))
    if tuple(t.shape) != (rows, cols):
        raise ValueError("%s has shape %s, expected %s" % (name, tuple(t.shape), (rows, cols)))
    if rows > 1 and cols > 1 and t.stride(0) != 1:
        raise ValueError("%s must be column-major (stride(0) == 1)" % name)
    ld = t.stride(1) if cols > 1 else max(rows, 1)
    return t.data_ptr(), max(ld, rows, 1)


def _options(schedule="auto", dfs_levels=-1, workspace_limit=0, precision="fp64", split_slices=0,
             gemm_tile="auto") -> Options:
    o = Options()
    lib().fmm_options_init(ctypes.byref(o))
    o.schedule = _lib.SCHEDULES[schedule]
    o.precision = _lib.PRECISIONS[precision]
    o.split_slices = split_slices
    o.dfs_levels = dfs_levels
    o.workspace_limit = workspace_limit
    o.gemm_tile = _lib.GEMM_TILES[gemm_tile]
    return o


def fast_matmul(alg, A, B, C, num_steps: int, x: float = 1e-8, alpha: float = 1.0, beta: float = 0.0,
                schedule: str = "auto", dfs_levels: int = -1, workspace_limit: int = 0,
                precision: Optional[str] = None, split_slices: int = 0, handle: Optional[Handle] = None,
                gemm_tile: str = "auto") -> None:
    """C := alpha * A * B + beta * C with `num_steps` levels of algorithm
    `alg` -- <alg>::FastMatmul(A, B, C, num_steps, x, alpha, beta).
    precision "split_bf16" runs the leaf products on the BF16 tensor cores
    over `split_slices` slices (0 = 5), "split_int8" on the INT8 tensor cores
    over 7-bit slices (0 = 6).  gemm_tile ("auto", "large" 128 x 64, "small"
    64 x 64) is the FP64 GEMM's tile configuration (speed only; the result
    does not depend on it).  Queued on torch's current stream.

    float32 operands (all three) select FastMatmul<float>
    (fmm_fast_matmul_f32): computed on FP64 copies and rounded to FP32 once;
    precision None there means split-INT8 leaves with 5 slices."""
    torch = _torch()
    idx = algorithm_index(alg)
    m, k = A.shape
    k2, n = B.shape
    if k2 != k:
        raise ValueError("inner dimensions differ")
    h = handle or default_handle(C.device.index)
    if A.dtype == torch.float32:
        pa, lda = _mat(A, m, k, "A", torch.float32)
        pb, ldb = _mat(B, k, n, "B", torch.float32)
        pc, ldc = _mat(C, m, n, "C", torch.float32)
        if precision is None:  # the FP32 default: split-INT8 leaves, FMM_F32_DEFAULT_SLICES slices
            o = _options(schedule, dfs_levels, workspace_limit, "split_int8", split_slices or F32_DEFAULT_SLICES)
        else:
            o = _options(schedule, dfs_levels, workspace_limit, precision, split_slices)
        check(lib().fmm_fast_matmul_f32(h.ptr, idx, pa, lda, pb, ldb, pc, ldc, m, k, n, num_steps, x, alpha, beta,
                                        ctypes.byref(o)))
        return
    pa, lda = _mat(A, m, k, "A")
    pb, ldb = _mat(B, k, n, "B")
    pc, ldc = _mat(C, m, n, "C")
    o = _options(schedule, dfs_levels, workspace_limit, precision or "fp64", split_slices, gemm_tile)
    check(lib().fmm_fast_matmul(h.ptr, idx, pa, lda, pb, ldb, pc, ldc, m, k, n, num_steps, x, alpha, beta,
                                ctypes.byref(o)))


def workspace_bytes(alg, m: int, k: int, n: int, num_steps: int, schedule: str = "auto", dfs_levels: int = -1,
                    workspace_limit: int = 0, precision: str = "fp64", split_slices: int = 0,
                    handle: Optional[Handle] = None) -> int:
    h = handle or default_handle()
    o = _options(schedule, dfs_levels, workspace_limit, precision, split_slices)
    out = ctypes.c_size_t()
    check(lib().fmm_workspace_query(h.ptr, algorithm_index(alg), m, k, n, num_steps, ctypes.byref(o),
                                    ctypes.byref(out)))
    return out.value


def _host_mat(a, rows, cols, name):
    """(pointer, leading dimension) of a column-major float64 host matrix."""
    import numpy as np

    if hasattr(a, "data_ptr"):
        if a.device.type != "cpu":
            raise ValueError("%s must be in host memory" % name)
        ld = a.stride(1) if cols > 1 else max(rows, 1)
        if rows > 1 and cols > 1 and a.stride(0) != 1:
            raise ValueError("%s must be column-major" % name)
        return a.data_ptr(), max(ld, rows, 1)
    arr = a
    if arr.dtype != np.float64 or (rows > 1 and cols > 1 and not arr.flags.f_contiguous):
        raise ValueError("%s must be a Fortran-ordered float64 array" % name)
    return arr.ctypes.data, max(rows, 1)


def fast_matmul_host_async(alg, A, B, C, num_steps: int, x: float = 1e-8, alpha: float = 1.0, beta: float = 0.0,
                           schedule: str = "auto", handle: Optional[Handle] = None) -> None:
    """Pipelined host-memory call (fmm_fast_matmul_host_async): queues the
    copies in, the product and the copy of C out, and returns at once; the
    host buffers must stay alive and unchanged until host_sync().  Pinned
    buffers let consecutive calls overlap their copies with each other's
    products."""
    m, k = A.shape
    n = B.shape[1]
    pa, lda = _host_mat(A, m, k, "A")
    pb, ldb = _host_mat(B, k, n, "B")
    pc, ldc = _host_mat(C, m, n, "C")
    h = handle or default_handle()
    o = _options(schedule)
    check(lib().fmm_fast_matmul_host_async(h.ptr, algorithm_index(alg), pa, lda, pb, ldb, pc, ldc, m, k, n,
                                           num_steps, x, alpha, beta, ctypes.byref(o)))


def host_sync(handle: Optional[Handle] = None) -> None:
    """Waits for every queued fast_matmul_host_async call (fmm_host_sync)."""
    h = handle or default_handle()
    check(lib().fmm_host_sync(h.ptr))


def fast_matmul_host(alg, A, B, C, num_steps: int, x: float = 1e-8, alpha: float = 1.0, beta: float = 0.0,
                     schedule: str = "auto", handle: Optional[Handle] = None) -> float:
    """Host-memory variant (fmm_fast_matmul_host): A, B, C are column-major
    float64 host arrays (numpy, Fortran order) or CPU torch tensors; returns
    the call's wall time in ms, copies included."""
    m, k = A.shape
    n = B.shape[1]
    pa, lda = _host_mat(A, m, k, "A")
    pb, ldb = _host_mat(B, k, n, "B")
    pc, ldc = _host_mat(C, m, n, "C")
    h = handle or default_handle()
    o = _options(schedule)
    ms = ctypes.c_double()
    check(lib().fmm_fast_matmul_host(h.ptr, algorithm_index(alg), pa, lda, pb, ldb, pc, ldc, m, k, n, num_steps,
                                     x, alpha, beta, ctypes.byref(o), ctypes.byref(ms)))
    return ms.value


def matmul(A, B, C, alpha: float = 1.0, beta: float = 0.0, handle: Optional[Handle] = None) -> None:
    """Classical C := alpha * A * B + beta * C on the engine's FP64 GEMM
    (MatMul with C's multiplier as alpha).  float32 operands: MatMul<float>
    (fmm_sgemm: FP64 copies, split-INT8 with 5 slices, rounded to FP32)."""
    torch = _torch()
    m, k = A.shape
    n = B.shape[1]
    if A.dtype == torch.float32:
        pa, lda = _mat(A, m, k, "A", torch.float32)
        pb, ldb = _mat(B, k, n, "B", torch.float32)
        pc, ldc = _mat(C, m, n, "C", torch.float32)
        h = handle or default_handle(C.device.index)
        check(lib().fmm_sgemm(h.ptr, pa, lda, pb, ldb, pc, ldc, m, k, n, alpha, beta, None))
        return
    pa, lda = _mat(A, m, k, "A")
    pb, ldb = _mat(B, k, n, "B")
    pc, ldc = _mat(C, m, n, "C")
    h = handle or default_handle(C.device.index)
    check(lib().fmm_dgemm(h.ptr, pa, lda, pb, ldb, pc, ldc, m, k, n, alpha, beta))


def matmul_split_bf16(A, B, C, alpha: float = 1.0, beta: float = 0.0, slices: int = 0,
                      handle: Optional[Handle] = None) -> None:
    """Classical C := alpha * A * B + beta * C with split-BF16 tensor-core
    products (fmm_dgemm_split_bf16; `slices` 0 = 5)."""
    m, k = A.shape
    n = B.shape[1]
    pa, lda = _mat(A, m, k, "A")
    pb, ldb = _mat(B, k, n, "B")
    pc, ldc = _mat(C, m, n, "C")
    h = handle or default_handle(C.device.index)
    check(lib().fmm_dgemm_split_bf16(h.ptr, pa, lda, pb, ldb, pc, ldc, m, k, n, alpha, beta, slices))


def matmul_split_int8(A, B, C, alpha: float = 1.0, beta: float = 0.0, slices: int = 0,
                      handle: Optional[Handle] = None) -> None:
    """Classical C := alpha * A * B + beta * C with split-INT8 tensor-core
    products (fmm_dgemm_split_int8; `slices` 0 = 6)."""
    m, k = A.shape
    n = B.shape[1]
    pa, lda = _mat(A, m, k, "A")
    pb, ldb = _mat(B, k, n, "B")
    pc, ldc = _mat(C, m, n, "C")
    h = handle or default_handle(C.device.index)
    check(lib().fmm_dgemm_split_int8(h.ptr, pa, lda, pb, ldb, pc, ldc, m, k, n, alpha, beta, slices))


def synchronize(handle: Optional[Handle] = None) -> None:
    """Waits for the handle's stream; raises if a split-BF16 kernel reported
    a bounded wait that gave up."""
    h = handle or default_handle()
    check(lib().fmm_synchronize(h.ptr))


def random_matrix(m: int, n: int, seed: int, stream: int = 0, lo: float = 0.0, hi: float = 1.0, device=None,
                  handle: Optional[Handle] = None):
    """Seeded column-major m x n matrix, entries lo + (hi - lo) * U[0, 1)."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    out = colmajor_empty(m, n, dev)
    h = handle or default_handle(dev.index)
    check(lib().fmm_fill_uniform(h.ptr, out.data_ptr(), m, n, max(m, 1), seed, stream, lo, hi))
    return out


def max_relative_diff(A, B, handle: Optional[Handle] = None) -> Tuple[float, float]:
    """(max_ij |a-b|/|a|, max_ij |a-b|) -- MaxRelativeDiff and MaxAbsDiff."""
    m, n = A.shape
    pa, lda = _mat(A, m, n, "A")
    pb, ldb = _mat(B, m, n, "B")
    h = handle or default_handle(A.device.index)
    rel = ctypes.c_double()
    ab = ctypes.c_double()
    check(lib().fmm_max_relative_diff(h.ptr, pa, lda, pb, ldb, m, n, ctypes.byref(rel), ctypes.byref(ab)))
    return rel.value, ab.value


# ---------------------------------------------------------------------------
# diagonal scaling (scaling/scaling.hpp)

OUTSIDE_INSIDE, INSIDE_OUTSIDE, INSIDE, OUTSIDE = 0, 1, 2, 3
_SCALING_TYPES = {"outside_inside": OUTSIDE_INSIDE, "inside_outside": INSIDE_OUTSIDE, "inside": INSIDE,
                  "outside": OUTSIDE}


def diagonal_scaling(A, B, num_steps: int, scaling_type=OUTSIDE_INSIDE, r_vals=None, s_vals=None,
                     handle: Optional[Handle] = None):
    """Scaling(A, B, num_steps, r_vals, s_vals, scaling_type)
    (scaling/scaling.hpp:153-196): scales the device matrices A and B in
    place and returns the factors (r_vals, s_vals) as device tensors, for
    scaling_postprocess.  scaling_type is 0..3 or its name.  Given r_vals /
    s_vals (float64 device vectors of length m / n) are updated in place and
    returned, as the reference multiplies into vectors that arrive sized;
    otherwise fresh vectors of ones are used."""
    torch = _torch()
    m, k = A.shape
    n = B.shape[1]
    kind = _SCALING_TYPES.get(scaling_type, scaling_type) if isinstance(scaling_type, str) else scaling_type
    if isinstance(kind, str):
        raise ValueError("Unknown iteration type.")
    dt = A.dtype if A.dtype == torch.float32 else torch.float64  # float32: Scaling<float>
    pa, lda = _mat(A, m, k, "A", dt)
    pb, ldb = _mat(B, k, n, "B", dt)
    r = torch.ones(m, dtype=dt, device=A.device) if r_vals is None else r_vals
    s = torch.ones(n, dtype=dt, device=A.device) if s_vals is None else s_vals
    for v, size, name in ((r, m, "r_vals"), (s, n, "s_vals")):
        if v.dtype != dt or tuple(v.shape) != (size,) or (size > 1 and v.stride(0) != 1):
            raise ValueError("%s must be a contiguous %s vector of length %d" % (name, dt, size))
    h = handle or default_handle(A.device.index)
    fn = lib().fmm_diagonal_scaling_f32 if dt == torch.float32 else lib().fmm_diagonal_scaling
    check(fn(h.ptr, pa, lda, pb, ldb, m, k, n, num_steps, int(kind), r.data_ptr(), s.data_ptr()))
    return r, s


def scaling_postprocess(C, r_vals, s_vals, handle: Optional[Handle] = None) -> None:
    """PostProcessScaling(C, r_vals, s_vals) (scaling/scaling.hpp:143-148):
    C(i, j) := (C(i, j) * r_vals[i]) * s_vals[j] on the device."""
    torch = _torch()
    m, n = C.shape
    dt = C.dtype if C.dtype == torch.float32 else torch.float64
    pc, ldc = _mat(C, m, n, "C", dt)
    for v, size, name in ((r_vals, m, "r_vals"), (s_vals, n, "s_vals")):
        if v.dtype != dt or tuple(v.shape) != (size,) or (size > 1 and v.stride(0) != 1):
            raise ValueError("%s must be a contiguous %s vector of length %d" % (name, dt, size))
    h = handle or default_handle(C.device.index)
    fn = lib().fmm_scaling_postprocess_f32 if dt == torch.float32 else lib().fmm_scaling_postprocess
    check(fn(h.ptr, pc, ldc, m, n, r_vals.data_ptr(), s_vals.data_ptr()))


# ---------------------------------------------------------------------------
# batches, autotuning and CUDA-graph plans (no counterpart in the reference)

CLASSICAL = _lib.FMM_ALG_CLASSICAL
AUTO = _lib.FMM_ALG_AUTO


def _batch_items(problems):
    """problems: iterable of dicts with A, B, C (column-major CUDA tensors) and
    optional alg (name, index, AUTO or CLASSICAL), num_steps, x, alpha, beta,
    precision, split_slices, gemm_tile ("auto", "large", "small")."""
    problems = list(problems)
    arr = (_lib.BatchItem * len(problems))()
    for i, p in enumerate(problems):
        A, B, C = p["A"], p["B"], p["C"]
        m, k = A.shape
        n = B.shape[1]
        pa, lda = _mat(A, m, k, "A")
        pb, ldb = _mat(B, k, n, "B")
        pc, ldc = _mat(C, m, n, "C")
        alg = p.get("alg", AUTO)
        if not (isinstance(alg, int) and alg < 0):
            alg = algorithm_index(alg)
        it = arr[i]
        it.alg = alg
        it.num_steps = int(p.get("num_steps", 1))
        it.A, it.lda, it.B, it.ldb, it.C, it.ldc = pa, lda, pb, ldb, pc, ldc
        it.m, it.k, it.n = m, k, n
        it.x = float(p.get("x", 1e-8))
        it.alpha = float(p.get("alpha", 1.0))
        it.beta = float(p.get("beta", 0.0))
        it.precision = _lib.PRECISIONS[p.get("precision", "fp64")]
        it.split_slices = int(p.get("split_slices", 0))
        it.gemm_tile = _lib.GEMM_TILES[p.get("gemm_tile", "auto")]
    return arr


def fast_matmul_batched(problems, handle: Optional[Handle] = None) -> None:
    """Independent products in one program (fmm_fast_matmul_batched)."""
    arr = _batch_items(problems)
    h = handle or default_handle()
    check(lib().fmm_fast_matmul_batched(h.ptr, arr, len(arr)))


def autotune(shapes, candidates=None, max_steps: int = 2, handle: Optional[Handle] = None) -> None:
    flat = [int(v) for s in shapes for v in s]
    sh = (ctypes.c_int64 * len(flat))(*flat)
    h = handle or default_handle()
    if candidates:
        idx = [algorithm_index(c) for c in candidates]
        ca = (ctypes.c_int * len(idx))(*idx)
        check(lib().fmm_autotune(h.ptr, sh, len(shapes), ca, len(idx), max_steps))
    else:
        check(lib().fmm_autotune(h.ptr, sh, len(shapes), None, 0, max_steps))


def autotune_choice(m: int, k: int, n: int, handle: Optional[Handle] = None):
    h = handle or default_handle()
    a = ctypes.c_int()
    s = ctypes.c_int()
    check(lib().fmm_autotune_choice(h.ptr, m, k, n, ctypes.byref(a), ctypes.byref(s)))
    return a.value, s.value


def autotune_tile(m: int, k: int, n: int, handle: Optional[Handle] = None) -> str:
    """The FP64 GEMM tile configuration tuned for the shape's bucket
    ("large", "small", or "auto" where the bucket was not measured)."""
    h = handle or default_handle()
    t = ctypes.c_int()
    check(lib().fmm_autotune_tile(h.ptr, m, k, n, ctypes.byref(t)))
    return {v: name for name, v in _lib.GEMM_TILES.items()}[t.value]


def autotune_table(handle: Optional[Handle] = None) -> str:
    h = handle or default_handle()
    n = ctypes.c_size_t()
    check(lib().fmm_autotune_export(h.ptr, None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value)
    check(lib().fmm_autotune_export(h.ptr, buf, n.value, ctypes.byref(n)))
    return buf.value.decode()


def autotune_load(text: str, handle: Optional[Handle] = None) -> None:
    h = handle or default_handle()
    check(lib().fmm_autotune_import(h.ptr, text.encode()))


class Plan:
    """A product or batch captured once as a CUDA graph (fmm_plan_*)."""

    def __init__(self, ptr, handle):
        self._p = ptr
        self.handle = handle

    @classmethod
    def for_product(cls, alg, A, B, C, num_steps, x=1e-8, alpha=1.0, beta=0.0, schedule="auto",
                    precision: str = "fp64", split_slices: int = 0, handle: Optional[Handle] = None):
        m, k = A.shape
        n = B.shape[1]
        pa, lda = _mat(A, m, k, "A")
        pb, ldb = _mat(B, k, n, "B")
        pc, ldc = _mat(C, m, n, "C")
        h = handle or default_handle(C.device.index)
        out = ctypes.c_void_p()
        o = _options(schedule, precision=precision, split_slices=split_slices)
        check(lib().fmm_plan_create(h.ptr, algorithm_index(alg), pa, lda, pb, ldb, pc, ldc, m, k, n, num_steps, x,
                                    alpha, beta, ctypes.byref(o), ctypes.byref(out)))
        return cls(out, h)

    @classmethod
    def for_batch(cls, problems, handle: Optional[Handle] = None):
        arr = _batch_items(problems)
        h = handle or default_handle()
        out = ctypes.c_void_p()
        check(lib().fmm_plan_create_batched(h.ptr, arr, len(arr), ctypes.byref(out)))
        return cls(out, h)

    def execute(self):
        self.handle.bind_current_stream()
        check(lib().fmm_plan_execute(self._p))

    @property
    def kernels(self) -> int:
        return int(lib().fmm_plan_kernel_count(self._p))

    def close(self):
        if self._p:
            lib().fmm_plan_destroy(self._p)
            self._p = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# serving: continuous-batching request loop (fmm_server_*)


class Server:
    """Requests are admitted in arrival order as launch slots and workspace
    free up; results are written into each request's C in place."""

    def __init__(self, device: int = 0, workspace_bytes: int = 0, max_inflight: int = 4, max_batch: int = 64):
        cfg = _lib.ServerConfig(device, workspace_bytes, max_inflight, max_batch)
        self._s = ctypes.c_void_p()
        check(lib().fmm_server_create(ctypes.byref(cfg), ctypes.byref(self._s)))
        self._keep = {}

    def submit(self, A, B, C, alg=AUTO, num_steps: int = 1, precision: str = "fp64", x: float = 1e-8,
               alpha: float = 1.0, beta: float = 0.0, split_slices: int = 0) -> int:
        m, k = A.shape
        n = B.shape[1]
        pa, lda = _mat(A, m, k, "A")
        pb, ldb = _mat(B, k, n, "B")
        pc, ldc = _mat(C, m, n, "C")
        if not (isinstance(alg, int) and alg < 0):
            alg = algorithm_index(alg)
        r = _lib.Request(alg, num_steps, _lib.PRECISIONS[precision], pa, lda, pb, ldb, pc, ldc, m, k, n, x, alpha,
                         beta, split_slices)
        t = ctypes.c_uint64()
        check(lib().fmm_server_submit(self._s, ctypes.byref(r), ctypes.byref(t)))
        self._keep[t.value] = (A, B, C)  # operands stay alive until the request is done
        return t.value

    def wait(self, ticket: int, timeout_ms: float = -1.0) -> dict:
        inf = _lib.RequestInfo()
        check(lib().fmm_server_wait(self._s, ticket, timeout_ms, ctypes.byref(inf)))
        self._keep.pop(ticket, None)
        return {"done": bool(inf.done), "status": inf.status, "submit_ms": inf.submit_ms,
                "launch_ms": inf.launch_ms, "done_ms": inf.done_ms}

    def drain(self, timeout_ms: float = -1.0) -> None:
        check(lib().fmm_server_drain(self._s, timeout_ms))

    def stats(self) -> dict:
        st = _lib.ServerStats()
        check(lib().fmm_server_get_stats(self._s, ctypes.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def close(self):
        if self._s:
            lib().fmm_server_destroy(self._s)
            self._s = ctypes.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""TEST INFRASTRUCTURE ONLY -- Python access to the CPU oracle.

Only tests/, the smoke check and the benchmark's CPU-baseline leg may import
this module, and only as the checker (or, for the baseline, as the timed
reference CPU path).  Nothing in the product imports it.

  liboracle.so        plain-C restatement of the reference recursion
                      (oracle/fmm_oracle.c); always buildable with gcc.
  _ref/libfmm_ref.so  the reference's own headers compiled unchanged
                      (oracle/ref_shim.cpp); built where the reference tree
                      is available, shipped with the repository snapshot.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libfmm_ref.so")

_P = ctypes.POINTER(ctypes.c_double)
_D = ctypes.c_double
_I = ctypes.c_int
_L = ctypes.c_long

_oracle = None
_ref = None


def reference_tree() -> Optional[str]:
    """The reference checkout: $FMM_REFERENCE, else the tree _ref/ was built
    from (recorded by the Makefile); None where neither exists."""
    cands = [os.environ.get("FMM_REFERENCE")]
    rec = os.path.join(HERE, "_ref", "REFERENCE_TREE")
    if os.path.exists(rec):
        with open(rec) as fh:
            cands.append(fh.read().strip())
    for c in cands:
        if c and os.path.isdir(os.path.join(c, "algorithms")):
            return c
    return None


def build(ref: bool = True) -> None:
    """Builds liboracle.so and, when a reference tree is known, _ref/libfmm_ref.so."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    tree = reference_tree() if ref else None
    if tree:
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + tree], check=True)


def oracle_lib() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            build(ref=False)
        L = ctypes.CDLL(ORACLE_LIB)
        L.oracle_fast_matmul.argtypes = [_I, _P, _L, _P, _L, _P, _L, _I, _I, _I, _I, _D, _D, _D]
        L.oracle_fast_matmul.restype = _I
        L.oracle_matmul.argtypes = [_P, _L, _P, _L, _P, _L, _I, _I, _I, _D, _D]
        L.oracle_matmul.restype = None
        L.oracle_max_relative_diff.argtypes = [_P, _L, _P, _L, _I, _I]
        L.oracle_max_relative_diff.restype = _D
        L.oracle_algorithm_name.argtypes = [_I]
        L.oracle_algorithm_name.restype = ctypes.c_char_p
        L.oracle_algorithm_index.argtypes = [ctypes.c_char_p]
        L.oracle_algorithm_index.restype = _I
        L.oracle_fill_uniform.argtypes = [_P, _L, ctypes.c_uint64, ctypes.c_uint64, _D, _D]
        L.oracle_quad_errors.argtypes = [_P, _P, _L, _L, _P, ctypes.POINTER(_D), ctypes.POINTER(_D)]
        L.oracle_quad_errors.restype = None
        L.oracle_scaling.argtypes = [_P, _L, _P, _L, _I, _I, _I, _I, _I, _P, _P]
        L.oracle_scaling.restype = _I
        L.oracle_scaling_postprocess.argtypes = [_P, _L, _I, _I, _P, _P]
        L.oracle_scaling_postprocess.restype = None
        L.oracle_fill_uniform.restype = None
        L.oracle_set_leaf_gemm.argtypes = [ctypes.c_void_p]
        L.oracle_set_leaf_gemm.restype = None
        _oracle = L
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _pin_blas_kernels() -> None:
    """The reference build's BLAS (OpenBLAS with run-time kernel dispatch)
    picks its DGEMM kernels by CPU model, and kernels for different models
    sum in different orders.  The committed reference digests were made with
    its SkylakeX (AVX-512) kernels; on a CPU with AVX-512 the same kernels
    are selected here, before the library loads, so the leaf products of the
    reference build give the same bits on every such host.  (Without
    AVX-512 those kernels cannot run; the default choice stays and
    bit-for-bit pins against the digests may then differ.)"""
    if "OPENBLAS_CORETYPE" in os.environ:
        return
    try:
        with open("/proc/cpuinfo") as fh:
            flags = fh.read()
    except OSError:
        return
    if " avx512f" in flags and " avx512dq" in flags and " avx512vl" in flags:
        os.environ["OPENBLAS_CORETYPE"] = "SkylakeX"


def ref_lib() -> Optional[ctypes.CDLL]:
    global _ref
    if _ref is None:
        if not ref_available():
            return None
        _pin_blas_kernels()
        L = ctypes.CDLL(REF_LIB)
        L.fmmref_fast_matmul.argtypes = [ctypes.c_char_p, _P, _I, _P, _I, _P, _I, _I, _I, _I, _I, _D, _D, _D]
        L.fmmref_fast_matmul.restype = _D
        L.fmmref_matmul.argtypes = [_P, _I, _P, _I, _P, _I, _I, _I, _I, _D, _D]
        L.fmmref_matmul.restype = None
        _F = ctypes.c_float
        _PF = ctypes.POINTER(ctypes.c_float)
        L.fmmref_fast_matmul_f32.argtypes = [ctypes.c_char_p, _PF, _I, _PF, _I, _PF, _I, _I, _I, _I, _I, _D, _F, _F]
        L.fmmref_fast_matmul_f32.restype = _D
        L.fmmref_matmul_f32.argtypes = [_PF, _I, _PF, _I, _PF, _I, _I, _I, _I, _F, _F]
        L.fmmref_matmul_f32.restype = None
        L.fmmref_scaling_f32.argtypes = [_PF, _I, _PF, _I, _I, _I, _I, _I, _I, _PF, _PF]
        L.fmmref_scaling_f32.restype = None
        L.fmmref_scaling_postprocess_f32.argtypes = [_PF, _I, _I, _I, _PF, _PF]
        L.fmmref_scaling_postprocess_f32.restype = None
        L.fmmref_set_threads.argtypes = [_I]
        L.fmmref_scaling.argtypes = [_P, _I, _P, _I, _I, _I, _I, _I, _I, _P, _P]
        L.fmmref_scaling.restype = None
        L.fmmref_scaling_postprocess.argtypes = [_P, _I, _I, _I, _P, _P]
        L.fmmref_scaling_postprocess.restype = None
        L.fmmref_set_threads.restype = None
        L.fmmref_num_algorithms.restype = _I
        L.fmmref_algorithm_name.argtypes = [_I]
        L.fmmref_algorithm_name.restype = ctypes.c_char_p
        _ref = L
    return _ref


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.f_contiguous
    return a.ctypes.data_as(_P)


# --------------------------------------------------------------------------
# seeded inputs: counter-based splitmix64, identical to fmm_fill_uniform


_GOLD = np.uint64(0x9E3779B97F4A7C15)


def uniform(rows: int, cols: int, seed: int, stream: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
    """Column-major rows x cols matrix; element e = i + j * rows."""
    with np.errstate(over="ignore"):
        key = np.uint64(seed) * np.uint64(0xD1B54A32D192ED03) + np.uint64(stream) * np.uint64(0x8CB92BA72F3D8DD7)
        e = np.arange(1, rows * cols + 1, dtype=np.uint64)
        z = key + e * _GOLD
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    vals = lo + (hi - lo) * u
    return np.asfortranarray(vals.reshape(cols, rows).T)


# --------------------------------------------------------------------------
# calls


def fast_matmul(alg: str, A: np.ndarray, B: np.ndarray, C: np.ndarray, num_steps: int, x: float = 1e-8,
                alpha: float = 1.0, beta: float = 0.0) -> None:
    """The C restatement of <alg>::FastMatmul on Fortran-ordered arrays (C in place)."""
    L = oracle_lib()
    idx = L.oracle_algorithm_index(alg.encode())
    if idx < 0:
        raise KeyError(alg)
    m, k = A.shape
    n = B.shape[1]
    rc = L.oracle_fast_matmul(idx, _p(A), max(m, 1), _p(B), max(k, 1), _p(C), max(m, 1), m, k, n, num_steps, x,
                              alpha, beta)
    if rc != 0:
        raise RuntimeError("oracle failed")


def matmul(A: np.ndarray, B: np.ndarray, C: np.ndarray, alpha: float = 1.0, beta: float = 0.0) -> None:
    L = oracle_lib()
    m, k = A.shape
    n = B.shape[1]
    L.oracle_matmul(_p(A), max(m, 1), _p(B), max(k, 1), _p(C), max(m, 1), m, k, n, alpha, beta)


def ref_fast_matmul(alg: str, A: np.ndarray, B: np.ndarray, C: np.ndarray, num_steps: int, x: float = 1e-8,
                    alpha: float = 1.0, beta: float = 0.0) -> float:
    """The reference itself (compiled headers + host BLAS); returns its ms."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference build oracle/_ref is not available")
    m, k = A.shape
    n = B.shape[1]
    ms = L.fmmref_fast_matmul(alg.encode(), _p(A), max(m, 1), _p(B), max(k, 1), _p(C), max(m, 1), m, k, n,
                              num_steps, x, alpha, beta)
    if ms < 0:
        raise KeyError(alg)
    return ms


def ref_matmul(A, B, C, alpha=1.0, beta=0.0) -> None:
    L = ref_lib()
    m, k = A.shape
    n = B.shape[1]
    L.fmmref_matmul(_p(A), max(m, 1), _p(B), max(k, 1), _p(C), max(m, 1), m, k, n, alpha, beta)


def _pf(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.f_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def ref_fast_matmul_f32(alg: str, A: np.ndarray, B: np.ndarray, C: np.ndarray, num_steps: int, x: float = 1e-8,
                        alpha: float = 1.0, beta: float = 0.0) -> float:
    """The reference's <alg>::FastMatmul<float> (sgemm leaves) on
    Fortran-ordered float32 arrays, C in place; returns its ms."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference build oracle/_ref is not available")
    m, k = A.shape
    n = B.shape[1]
    ms = L.fmmref_fast_matmul_f32(alg.encode(), _pf(A), max(m, 1), _pf(B), max(k, 1), _pf(C), max(m, 1), m, k, n,
                                  num_steps, x, alpha, beta)
    if ms < 0:
        raise KeyError(alg)
    return ms


def ref_matmul_f32(A, B, C, alpha=1.0, beta=0.0) -> None:
    """The reference's MatMul<float> (sgemm) on float32 arrays, C in place."""
    L = ref_lib()
    m, k = A.shape
    n = B.shape[1]
    L.fmmref_matmul_f32(_pf(A), max(m, 1), _pf(B), max(k, 1), _pf(C), max(m, 1), m, k, n, alpha, beta)


def ref_scaling_f32(A: np.ndarray, B: np.ndarray, num_steps: int, kind: int, r=None, s=None):
    """The reference's Scaling<float> on Fortran-ordered float32 A, B in
    place; returns (r, s) as float32 (fresh vectors of ones by default)."""
    L = ref_lib()
    m, k = A.shape
    n = B.shape[1]
    r = np.ones(m, dtype=np.float32) if r is None else np.array(r, dtype=np.float32)
    s = np.ones(n, dtype=np.float32) if s is None else np.array(s, dtype=np.float32)
    pf = ctypes.POINTER(ctypes.c_float)
    L.fmmref_scaling_f32(_pf(A), max(m, 1), _pf(B), max(k, 1), m, k, n, num_steps, kind, r.ctypes.data_as(pf),
                         s.ctypes.data_as(pf))
    return r, s


def ref_scaling_postprocess_f32(C: np.ndarray, r: np.ndarray, s: np.ndarray) -> None:
    """The reference's PostProcessScaling on Fortran-ordered float32 C in place."""
    m, n = C.shape
    pf = ctypes.POINTER(ctypes.c_float)
    r = np.ascontiguousarray(r, dtype=np.float32)
    s = np.ascontiguousarray(s, dtype=np.float32)
    ref_lib().fmmref_scaling_postprocess_f32(_pf(C), max(m, 1), m, n, r.ctypes.data_as(pf), s.ctypes.data_as(pf))


def use_reference_leaf(enabled: bool) -> None:
    """Route the restatement's leaf products through the reference's BLAS."""
    L = oracle_lib()
    if enabled:
        R = ref_lib()
        L.oracle_set_leaf_gemm(ctypes.cast(R.fmmref_matmul, ctypes.c_void_p))
    else:
        L.oracle_set_leaf_gemm(None)


def quad_errors(A: np.ndarray, B: np.ndarray, rows, cols, values) -> tuple:
    """Errors of computed entries values[s] = C[rows[s], cols[s]] against the
    quad-precision product (oracle_quad_errors, after linalg/quadmatmul.hpp):
    (max |v - q| / |q|, max |v - q| / (|A| |B|)_ij)."""
    L = oracle_lib()
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    ar = np.ascontiguousarray(A[rows, :], dtype=np.float64)
    bc = np.ascontiguousarray(B[:, cols].T, dtype=np.float64)
    v = np.ascontiguousarray(values, dtype=np.float64)
    mr = ctypes.c_double()
    ms = ctypes.c_double()
    L.oracle_quad_errors(ar.ctypes.data_as(_P), bc.ctypes.data_as(_P), A.shape[1], len(rows), v.ctypes.data_as(_P),
                         ctypes.byref(mr), ctypes.byref(ms))
    return mr.value, ms.value


def scaling(A: np.ndarray, B: np.ndarray, num_steps: int, kind: int, ref: bool = False, r=None, s=None):
    """Scaling<double>(A, B, num_steps, r, s, kind) (scaling/scaling.hpp) on
    Fortran-ordered A, B in place; returns (r, s), which start as the given
    vectors (fresh vectors of ones by default).  ref=True runs the
    reference's own header through the reference build."""
    m, k = A.shape
    n = B.shape[1]
    r = np.ones(m) if r is None else np.array(r, dtype=np.float64)
    s = np.ones(n) if s is None else np.array(s, dtype=np.float64)
    if ref:
        ref_lib().fmmref_scaling(_p(A), max(m, 1), _p(B), max(k, 1), m, k, n, num_steps, kind,
                                 r.ctypes.data_as(_P), s.ctypes.data_as(_P))
    else:
        rc = oracle_lib().oracle_scaling(_p(A), max(m, 1), _p(B), max(k, 1), m, k, n, num_steps, kind,
                                         r.ctypes.data_as(_P), s.ctypes.data_as(_P))
        if rc != 0:
            raise ValueError("unknown scaling type %d" % kind)
    return r, s


def scaling_postprocess(C: np.ndarray, r: np.ndarray, s: np.ndarray, ref: bool = False) -> None:
    """PostProcessScaling(C, r, s) (scaling/scaling.hpp) on Fortran-ordered C in place."""
    m, n = C.shape
    r = np.ascontiguousarray(r, dtype=np.float64)
    s = np.ascontiguousarray(s, dtype=np.float64)
    if ref:
        ref_lib().fmmref_scaling_postprocess(_p(C), max(m, 1), m, n, r.ctypes.data_as(_P), s.ctypes.data_as(_P))
    else:
        oracle_lib().oracle_scaling_postprocess(_p(C), max(m, 1), m, n, r.ctypes.data_as(_P), s.ctypes.data_as(_P))


def max_relative_diff(a: np.ndarray, b: np.ndarray) -> float:
    """max_ij |a_ij - b_ij| / |a_ij| (linalg/linalg.hpp:280-295), NaN terms skipped."""
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.abs(a - b) / np.abs(a)
    r = r[~np.isnan(r)]
    return float(r.max()) if r.size else 0.0

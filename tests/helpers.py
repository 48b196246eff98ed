"""Shared test helpers: golden fixtures, planner emulator, GPU checks."""

import base64
import ctypes
import json
import os
import subprocess
import zlib

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden", "reference_cases.json")
CSRC = os.path.join(REPO, "fast_matmul_b200", "csrc")
EMU_SRC = os.path.join(REPO, "tests", "native", "plan_emulator.cpp")
EMU_LIB = os.path.join(REPO, "tests", "native", "_build", "libplan_emu.so")

# lambda per step count chosen by the reference's RunAlgorithm
# (algorithms/all_algorithms.hpp:102-141)
def default_x(alg, steps):
    if alg == "bini322_10_52_approx":
        return {2: 1e-4, 3: 1e-2, 4: 1e-1}.get(steps, 1e-8)
    if alg == "schonhage333_21_117_approx":
        return {1: 1e-4, 2: 1e-2, 3: 1e-1, 4: 1e-1}.get(steps, 1e-4)
    return 1e-8


def load_golden():
    with open(GOLDEN) as fh:
        return json.load(fh)


def decode_matrix(s, m, n):
    raw = np.frombuffer(zlib.decompress(base64.b64decode(s)), dtype=np.float64)
    return np.asfortranarray(raw.reshape(n, m).T)


def emulator():
    """The planner interpreter (tests/native/plan_emulator.cpp), built on demand."""
    srcs = [EMU_SRC, os.path.join(CSRC, "plan.cpp"), os.path.join(CSRC, "split_plan.cpp")]
    deps = srcs + [os.path.join(CSRC, f) for f in ("plan.h", "fmm_internal.h")] + \
        [os.path.join(CSRC, "generated", f) for f in os.listdir(os.path.join(CSRC, "generated"))]
    if not os.path.exists(EMU_LIB) or os.path.getmtime(EMU_LIB) < max(os.path.getmtime(d) for d in deps):
        os.makedirs(os.path.dirname(EMU_LIB), exist_ok=True)
        cuda_inc = "/usr/local/cuda/include"
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-w",
                        "-I" + CSRC, "-I" + os.path.join(REPO, "include"), "-I" + cuda_inc] + srcs +
                       ["-o", EMU_LIB], check=True)
    L = ctypes.CDLL(EMU_LIB)
    P = ctypes.POINTER(ctypes.c_double)
    i64 = ctypes.c_int64
    I = ctypes.c_int
    D = ctypes.c_double
    L.emu_fast_matmul.argtypes = [I, P, i64, P, i64, P, i64, I, I, I, I, D, D, D, I, ctypes.POINTER(i64)]
    L.emu_fast_matmul.restype = I
    L.emu_workspace_bytes.argtypes = [I, i64, i64, i64, I, I]
    L.emu_workspace_bytes.restype = ctypes.c_size_t
    IP = ctypes.POINTER(ctypes.c_int)
    LP = ctypes.POINTER(i64)
    L.emu_fast_matmul_batch.argtypes = [I, IP, IP, LP, P, LP, P, LP, P, LP, D, D, D, LP]
    L.emu_fast_matmul_batch.restype = I
    L.emu_fast_matmul_split.argtypes = [I, P, i64, P, i64, P, i64, I, I, I, I, D, D, D, I, I, ctypes.POINTER(i64)]
    L.emu_fast_matmul_split.restype = I
    L.emu_workspace_bytes_split.argtypes = [I, i64, i64, i64, I, I, I]
    L.emu_workspace_bytes_split.restype = ctypes.c_size_t
    L.emu_split_gemm.argtypes = [I, I, I, P, i64, P, i64, P, i64, D, D, I]
    L.emu_split_gemm.restype = None
    L.emu_fast_matmul_batch_split.argtypes = [I, IP, IP, LP, P, LP, P, LP, P, LP, D, D, D, IP, LP]
    L.emu_fast_matmul_batch_split.restype = I
    return L


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def to_device(a):
    """Fortran-ordered numpy -> column-major torch CUDA tensor."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    return t.t()


def to_host(t):
    return np.asfortranarray(t.t().contiguous().cpu().numpy().T)


def colmajor_copy(t):
    """A new column-major tensor with t's values (never an alias of t)."""
    import torch
    out = torch.empty((t.shape[1], t.shape[0]), dtype=t.dtype, device=t.device).t()
    out.copy_(t)
    return out

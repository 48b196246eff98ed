"""The C-ABI library loads and exports every entry point include/fmm.h declares.

No compute call is made here (these tests run without a GPU); handle
creation must fail with a status, never crash.
"""

import ctypes
import os
import re

import pytest

from helpers import REPO, gpu_available

import fast_matmul_b200 as fmm
from fast_matmul_b200 import _lib


def declared_functions(header):
    text = open(os.path.join(REPO, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fmm_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    L = _lib.lib()
    names = declared_functions("fmm.h")
    assert len(names) >= 18
    for name in names:
        assert hasattr(L, name), name
        assert name in _lib.SIGNATURES, name


def test_registry_without_gpu():
    assert fmm.num_algorithms() == 42
    names = fmm.algorithm_names()
    assert "strassen" in names and "grey424_26_206" in names and "bini322_10_52_approx" in names
    info = fmm.algorithm_info("fast424_26_206")  # header stem resolves to the namespace
    assert (info["name"], info["m0"], info["k0"], info["n0"], info["rank"]) == ("grey424_26_206", 4, 2, 4, 26)
    assert fmm.algorithm_info("fast333_23_125.hpp")["name"] == "grey333_23_125"
    assert fmm.algorithm_info("bini322_10_52_approx")["approximate"]
    with pytest.raises(fmm.FmmError):
        fmm.algorithm_index("smirnov333_23_125")  # not generated by the reference either


def test_options_defaults():
    o = _lib.Options()
    _lib.lib().fmm_options_init(ctypes.byref(o))
    assert (o.schedule, o.precision, o.dfs_levels, o.workspace_limit, o.gemm_tile) == (0, 0, -1, 0, 0)


CHECKED = os.path.join(REPO, "fast_matmul_b200", "libfmm_checked.so")


@pytest.mark.skipif(not os.path.exists(CHECKED), reason="libfmm_checked.so not built")
def test_checked_library_exports_every_symbol():
    L = ctypes.CDLL(CHECKED)
    for name in declared_functions("fmm.h"):
        assert hasattr(L, name), name


def test_regular_library_has_no_device_checks():
    flags = ctypes.c_uint(7)
    assert _lib.lib().fmm_debug_check_flags(ctypes.byref(flags)) == 5  # FMM_ERR_NOT_SUPPORTED
    assert flags.value == 0


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_handle_create_without_gpu_reports_status():
    h = ctypes.c_void_p()
    st = _lib.lib().fmm_handle_create(ctypes.byref(h), 0)
    assert st == 4  # FMM_ERR_CUDA
    assert _lib.lib().fmm_last_error()


def test_null_arguments_are_rejected():
    L = _lib.lib()
    assert L.fmm_fast_matmul(None, 0, None, 1, None, 1, None, 1, 1, 1, 1, 1, 1e-8, 1.0, 0.0, None) == 1
    assert b"null" in L.fmm_last_error()
    assert L.fmm_dgemm(None, None, 1, None, 1, None, 1, 1, 1, 1, 1.0, 0.0) == 1

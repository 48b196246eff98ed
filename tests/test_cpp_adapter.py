"""The C++ drop-in surface (include/fmm/*.hpp): a driver written against the
reference's API compiles against the adapter and libfmm.so (CPU), and its
checks pass on the GPU."""

import os
import subprocess

import pytest

from helpers import REPO

DRIVER = os.path.join(REPO, "tests", "cpp", "adapter_driver.cpp")
LIBDIR = os.path.join(REPO, "fast_matmul_b200")
OUT = os.path.join(REPO, "tests", "native", "_build", "adapter_driver")


def build_driver():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.run(["g++", "-std=c++11", "-O2", "-Wall", "-Werror", "-I" + os.path.join(REPO, "include"), DRIVER,
                    "-o", OUT, "-L" + LIBDIR, "-lfmm", "-Wl,-rpath," + LIBDIR], check=True,
                   capture_output=True, text=True)
    return OUT


def test_adapter_driver_builds_against_the_c_abi():
    assert os.path.exists(build_driver())


@pytest.mark.gpu
def test_adapter_driver_passes_on_gpu():
    exe = build_driver()
    res = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "PASSED" in res.stdout

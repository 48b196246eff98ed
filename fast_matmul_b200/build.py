"""Builds libfmm.so (the engine) in-tree for sm_100a.

    python -m fast_matmul_b200.build [--force] [--jobs N] [--checked]

Every translation unit under csrc/ is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo`` into _build/, then
linked into fast_matmul_b200/libfmm.so (CUDA runtime linked statically).
Host code is compiled with -ffp-contract=off so coefficient and multiplier
products round exactly like the reference's.

--checked builds the same sources with -DFMM_DEVICE_CHECKS into
_build_checked/ and fast_matmul_b200/libfmm_checked.so: the debug library
whose kernels check their descriptor walks (fmm_debug_check_flags).
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libfmm.so")
BUILD_CHECKED = os.path.join(PKG, "_build_checked")
LIB_CHECKED = os.path.join(PKG, "libfmm_checked.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def common_flags(checked: bool = False):
    return ARCH + (["-DFMM_DEVICE_CHECKS"] if checked else []) + [
        "-O3", "-lineinfo", "-std=c++17",
        "-Xcompiler", "-fPIC,-ffp-contract=off",
        "-I" + os.path.join(REPO, "include"),
        "-I" + CSRC,
    ]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(CSRC, "generated", "*")) + glob.glob(os.path.join(REPO, "include", "*.h")))


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def _compile(src: str, force: bool, build_dir: str = BUILD, checked: bool = False) -> str:
    obj = os.path.join(build_dir, os.path.basename(src) + ".o")
    newest_dep = max([_mtime(src)] + [_mtime(h) for h in headers()])
    if not force and _mtime(obj) > newest_dep:
        return obj
    cmd = [nvcc_path()] + common_flags(checked) + ["-c", src, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), res.stderr[-8000:]))
    return obj


def build(force: bool = False, jobs: int = 0, verbose: bool = True, checked: bool = False) -> str:
    build_dir = BUILD_CHECKED if checked else BUILD
    lib = LIB_CHECKED if checked else LIB
    os.makedirs(build_dir, exist_ok=True)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, build_dir, checked), srcs))
    if force or not os.path.exists(lib) or max(_mtime(o) for o in objs) > _mtime(lib):
        cmd = [nvcc_path()] + ARCH + ["-shared", "-o", lib] + objs + ["-cudart", "static"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), res.stderr[-8000:]))
        if verbose:
            print("built", os.path.relpath(lib, REPO))
    return lib


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--checked", action="store_true", help="build libfmm_checked.so (-DFMM_DEVICE_CHECKS)")
    a = ap.parse_args(argv)
    build(force=a.force, jobs=a.jobs, checked=a.checked)
    return 0


if __name__ == "__main__":
    sys.exit(main())

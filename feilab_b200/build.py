"""Build recipe of the native library: nvcc for sm_100a, in-tree output.

    python -m feilab_b200.build          # builds feilab_b200/libicon_b200.so
                                         # and feilab_b200/icon-gpu (CLI)

The library is built in place (next to this file) so it travels with the
repository; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libicon_b200.so")
CLI = os.path.join(HERE, "icon-gpu")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]

# (source, extra flags, object): the batched FFT kernels are built once per
# slice-group size B, in parallel.
LIB_UNITS = [("icon_api.cu", [], "icon_api.o"), ("icon_noalloc.cu", [], "icon_noalloc.o"),
             ("ws_api.cu", [], "ws_api.o"), ("ws_net.cu", [], "ws_net.o"),
             ("tools.cu", [], "tools.o"), ("mask.cu", [], "mask.o"),
             ("frc.cu", [], "frc.o"), ("loo.cu", [], "loo.o"), ("icon_batch.cu", [], "icon_batch.o"),
             ("icon_warm.cu", [], "icon_warm.o")] + [
    ("icon_kern_b.cu", ["-DICON_KB=%d" % b], "icon_kern_b%d.o" % b) for b in (1, 2, 4, 8)]
LIB_DEPS = ["icon_api.cu", "icon_noalloc.cu", "icon_kern_b.cu", "icon_launch.h", "icon_kernels.cuh", "icon_device.cuh",
            "ws_api.cu", "ws_conv.cuh", "ws_tc.cuh", "ws_net.cu", "ws_kernels.cuh", "tools.cu", "mask.cu", "frc.cu", "loo.cu",
            "icon_batch.cu", "icon_internal.h", "icon_warm.cu"]
BUILD_DIR = os.path.join(HERE, "_build")
# Command-line tools: executable -> sources (host C++ over the C ABI).
TOOLS = {"icon-gpu": ["icon_cli.cpp", "mrc_io.cpp"], "icon-preprocess": ["preprocess_cli.cpp", "mrc_io.cpp"],
         "icon-mask": ["mask_cli.cpp", "mrc_io.cpp"]}


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def build_lib(force=False, verbose=False):
    deps = [os.path.join(CSRC, f) for f in LIB_DEPS] + [os.path.join(ROOT, "include", h)
                                                        for h in ("icon_b200.h", "icon_warmstart.h", "icon_tools.h",
                                                                  "icon_batch.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    cmds = [[_nvcc(), *ARCH, *NVFLAGS, *extra, "-c", "-o", os.path.join(BUILD_DIR, obj), os.path.join(CSRC, src)]
            for src, extra, obj in LIB_UNITS]
    if verbose:
        for c in cmds:
            print(" ".join(c))
    procs = [subprocess.Popen(c) for c in cmds]
    rcs = [p.wait() for p in procs]
    if any(rcs):
        raise subprocess.CalledProcessError(max(rcs), "nvcc")
    link = [_nvcc(), *ARCH, "-shared", "-o", LIB] + [os.path.join(BUILD_DIR, obj) for _, _, obj in LIB_UNITS]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    return LIB


def build_cli(force=False, verbose=False):
    """The command-line tools (TOOLS), linked against the library."""
    built = []
    for exe, sources in TOOLS.items():
        srcs = [os.path.join(CSRC, f) for f in sources]
        if not all(os.path.exists(s) for s in srcs):
            continue
        target = os.path.join(HERE, exe)
        deps = srcs + [LIB, os.path.join(CSRC, "mrc_io.h")] + [os.path.join(ROOT, "include", h) for h in
                                                              ("icon_b200.h", "icon_tools.h")]
        if force or _stale(target, deps):
            cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-o", target, *srcs,
                   "-L" + HERE, "-licon_b200", "-Wl,-rpath,$ORIGIN", "-lpthread"]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        built.append(target)
    return built


def build(force=False, verbose=False):
    build_lib(force, verbose)
    build_cli(force, verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

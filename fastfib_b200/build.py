"""Builds libfastfib_b200.so in-tree: the CUDA units for sm_100a with nvcc, the
host C surface with gcc, linked into one shared library next to this file.

    python -m fastfib_b200.build        (or fastfib_b200.build.build())

Objects go to fastfib_b200/_build/; the command line fastfib_b200/fastfib
links against the library.  Only files whose sources changed are
recompiled (header changes rebuild everything).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libfastfib_b200.so")
CLI = os.path.join(PKG, "fastfib")

NVCC = os.environ.get("NVCC", "nvcc")
CC = os.environ.get("CC", "gcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
           f"-I{INC}", f"-I{CSRC}"]
CFLAGS = ["-O2", "-std=gnu17", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter", f"-I{INC}",
          f"-I{os.path.join(CSRC, 'host')}"]


def _newer(src: list[str], dst: str) -> bool:
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in src)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {' '.join(cmd[:3])} ...")


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(CSRC, "host", "*.h")) + glob.glob(os.path.join(INC, "*.h"))
    objs = []
    for cu in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(cu) + ".o")
        if _newer([cu, *headers], obj):
            if verbose:
                print("nvcc", os.path.basename(cu))
            _run([NVCC, *ARCH, *NVFLAGS, "-c", cu, "-o", obj])
        objs.append(obj)
    for c in sorted(glob.glob(os.path.join(CSRC, "host", "*.c"))):
        obj = os.path.join(BUILD, "host_" + os.path.basename(c) + ".o")
        if _newer([c, *headers], obj):
            if verbose:
                print("gcc", os.path.basename(c))
            _run([CC, *CFLAGS, "-c", c, "-o", obj])
        objs.append(obj)
    if _newer(objs, LIB):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs])
    # the command line (fastfib [n] [--print]) over the library's Big surface
    cli_src = os.path.join(CSRC, "cli", "fastfib_cli.c")
    if _newer([cli_src, LIB, *headers], CLI):
        if verbose:
            print("gcc", os.path.basename(cli_src))
        _run([CC, *CFLAGS, cli_src, "-o", CLI, f"-L{PKG}", "-lfastfib_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))

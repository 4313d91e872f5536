"""Builds the in-tree CUDA library patchtable_b200/libpatchtable_b200.so for sm_100a.

Each .cu/.cpp under csrc/ is compiled to an object in csrc/_build/ (rebuilt when the source or
any header is newer), then linked into one shared library with a plain C ABI
(include/patchtable_b200.h).  Usage:  python -m patchtable_b200.build
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(CSRC, "_build")
LIB = os.path.join(HERE, "libpatchtable_b200.so")
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    headers = (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
               glob.glob(os.path.join(ROOT, "include", "*.h")))
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", os.path.join(ROOT, "include")]
    cmds, objs = [], []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if not _newer(o, [s] + headers):
            continue
        if s.endswith(".cu"):
            cmd = [nvcc, ARCH, "-lineinfo", "--expt-relaxed-constexpr", "-c", s, "-o", o] + common
        else:
            cmd = [nvcc, ARCH, "-x", "c++", "-c", s, "-o", o] + common
        cmds.append(cmd)
    procs = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= jobs:
            _wait(procs.pop(0))
    for pr in procs:
        _wait(pr)
    if cmds or _newer(LIB, objs):
        cmd = [nvcc, ARCH, "-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
        if r.returncode:
            raise RuntimeError("link failed:\n" + r.stdout.decode())
    return LIB


def _wait(pr):
    cmd, p = pr
    out, _ = p.communicate()
    if p.returncode:
        raise RuntimeError("compile failed: %s\n%s" % (" ".join(cmd), out.decode()))
    txt = out.decode().strip()
    if txt:
        print(txt)


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

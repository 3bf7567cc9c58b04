"""Build libpyspectral_b200.so in-tree with nvcc for sm_100a.

    python -m pyspectral_b200.build [--force] [--debug]

Objects go to ``_build/`` (git-ignored); the shared library lands next to
this file so that it travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libpyspectral_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                "-Xcompiler", "-Wno-deprecated-declarations"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(target, inputs):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in inputs)


def build(force: bool = False, extra_flags=None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nv = nvcc()
    flags = FLAGS + list(extra_flags or [])
    deps = _deps()
    jobs = []
    objs = []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + deps):
            jobs.append([nv] + flags + ["-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose:
            sys.stdout.write(r.stdout + r.stderr)
        return cmd[-1]

    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or _stale(LIB, objs):
        cmd = [nv] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, extra_flags=["-G"] if "--debug" in sys.argv else None, verbose=True)
    print(LIB)

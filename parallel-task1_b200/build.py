"""Build the traversal library for sm_100a: ``parallel-task1_b200/libtrav_b200.so``.

Compiles every ``csrc/*.cu`` / ``csrc/*.cpp`` with nvcc
(``-gencode arch=compute_100a,code=sm_100a -lineinfo``) in parallel and links
one shared library in the package directory, so it travels with the working
tree.  Also builds the sample programs (``sample/sssp``, ``sample/bfs``).
Rebuilds only what changed (source or header newer than its object).

    python parallel-task1_b200/build.py [--force] [--verbose-ptxas]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libtrav_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
          "--expt-relaxed-constexpr"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, obj, verbose_ptxas):
    cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
    if verbose_ptxas and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stdout + r.stderr


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdrs = _headers()
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if force or verbose_ptxas or _stale(o, [s] + hdrs):
            jobs.append((s, o))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for src, rc, out in ex.map(lambda j: _compile(j[0], j[1], verbose_ptxas), jobs):
                if out.strip() and (rc != 0 or verbose_ptxas):
                    sys.stderr.write(out)
                if rc != 0:
                    raise RuntimeError(f"nvcc failed on {src}")
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libtrav_b200.so failed")
        os.replace(LIB + ".tmp", LIB)
    _build_samples(force)
    return LIB


def _build_samples(force: bool):
    sdir = os.path.join(PKG, "sample")
    for src in sorted(glob.glob(os.path.join(sdir, "*.cpp"))):
        exe = src[:-4]
        deps = [src, LIB] + glob.glob(os.path.join(PKG, "host", "*.hpp")) + _headers()
        if not force and not _stale(exe, deps):
            continue
        cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-I", os.path.join(ROOT, "include"), "-I", PKG, src, "-o", exe,
               "-L", PKG, "-ltrav_b200", "-Wl,-rpath,$ORIGIN/..", "-Wl,-rpath," + PKG]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"g++ failed on {src}")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    args = ap.parse_args()
    print(build(args.force, args.verbose_ptxas))

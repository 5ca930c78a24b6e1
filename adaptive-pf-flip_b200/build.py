"""Build libpfgpu.so (the sm_100a kernels and the C ABI) in-tree with nvcc.

    python adaptive-pf-flip_b200/build.py [--force] [-j N]

Objects go to ``adaptive-pf-flip_b200/_build/``, the library to
``adaptive-pf-flip_b200/lib/libpfgpu.so``.  Every translation unit is compiled
for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "lib", "libpfgpu.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
                "-Xcompiler", "-ffp-contract=off",
                "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]

SOURCES = ["pf_pool.cu", "pf_transfer.cu", "pf_project.cu", "pf_pcg.cu", "pf_timing.cu", "pf_noalloc.cu",
           "pf_coarse.cu", "pf_flex.cu", "pf_outer.cu", "pf_learned.cu", "pf_adapt.cu", "pf_diag.cu", "pf_render.cu", "pf_scene.cu", "pf_mr.cu", "pf_secondary.cu",
           "pf_capi.cu"]


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
        [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]


def _stale(target, inputs):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(i) > t for i in inputs)


def _compile(src, verbose):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    cmd = [NVCC] + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{out.stdout}\n{out.stderr}")
    return obj, out.stderr


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    """Compile stale objects and relink; returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    deps = _deps()
    todo = [s for s in SOURCES
            if force or _stale(os.path.join(BUILD, os.path.splitext(s)[0] + ".o"), [os.path.join(CSRC, s)] + deps)]
    logs = []
    if todo:
        jobs = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for obj, log in ex.map(lambda s: _compile(s, verbose), todo):
                logs.append(log)
    objs = [os.path.join(BUILD, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    if todo or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError(f"link failed:\n{out.stdout}\n{out.stderr}")
    if verbose:
        for log in logs:
            sys.stderr.write(log)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=0)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.verbose))

"""Build the native library and the command-line driver in-tree.

    python -m morphoshell_b200.build [--force]

Outputs (git-ignored, shipped with the source tree):
    morphoshell_b200/lib/libmorphoshell.so   host set-up + sm_100a kernels + C ABI
    morphoshell_b200/lib/morphoshell_gpu     command-line drop-in for the reference's executable

CUDA sources are compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
there is no other device target and no CPU fallback.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
OBJ_DIR = os.path.join(LIB_DIR, "obj")
LIB = os.path.join(LIB_DIR, "libmorphoshell.so")
EXE = os.path.join(LIB_DIR, "morphoshell_gpu")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function"]
NVCCFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
             "-Xptxas", "-O3"] + GENCODE

HOST_SOURCES = ["host/settings.cpp", "host/vtk_io.cpp", "host/mesh_setup.cpp", "host/host_capi.cpp"]
CUDA_SOURCES = ["cuda/kernels.cu", "cuda/cluster.cu", "cuda/capi.cu", "cuda/noalloc.cu", "cuda/batch.cu",
                "cuda/learned.cu", "cuda/tri_tiles.cu", "cuda/node_tiles.cu", "cuda/node_tile_plan.cu",
                "cuda/node_pipe.cu", "cuda/setup.cu"]
# Per-file nvcc flags: the device set-up rounds every operation as the host
# set-up does (no contraction into fused multiply-adds).
CUDA_FILE_FLAGS = {"cuda/setup.cu": ["-fmad=false"]}
HEADERS = ["host/host.hpp", "host/small_linalg.hpp", "cuda/internal.cuh", "cuda/tri_physics.cuh", "cuda/step_common.cuh",
           "cuda/tri_contrib.cuh", "cuda/tc_gemm.cuh", "cuda/tile_copy.cuh", "cuda/node_tile_walk.cuh",
           "host/patch_fit.hpp",
           "../../include/morphoshell_gpu.h", "../../include/morphoshell_host.h"]


def _newest_header() -> float:
    return max(os.path.getmtime(os.path.join(CSRC, h)) for h in HEADERS)


def _stale(out: str, src: str) -> bool:
    if not os.path.exists(out):
        return True
    return os.path.getmtime(out) < max(os.path.getmtime(src), _newest_header())


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def _compile(src_rel: str, force: bool, extra: list[str]) -> str:
    src = os.path.join(CSRC, src_rel)
    obj = os.path.join(OBJ_DIR, src_rel.replace("/", "_") + ".o")
    if force or _stale(obj, src):
        if src.endswith(".cu"):
            _run([NVCC] + NVCCFLAGS + extra + ["-c", src, "-o", obj])
        else:
            _run(["g++"] + CXXFLAGS + extra + ["-c", src, "-o", obj])
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    extra_cu = ["-Xptxas", "-v"] if verbose_ptxas else []
    jobs = [(s, []) for s in HOST_SOURCES] + [(s, extra_cu + CUDA_FILE_FLAGS.get(s, [])) for s in CUDA_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda j: _compile(j[0], force, j[1]), jobs))
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        _run([NVCC] + GENCODE + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    main_obj = _compile("host/main.cpp", force, [])
    if force or not os.path.exists(EXE) or os.path.getmtime(EXE) < os.path.getmtime(LIB):
        _run(["g++", "-o", EXE, main_obj, "-L" + LIB_DIR, "-lmorphoshell", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register / spill usage")
    a = ap.parse_args()
    print(build(force=a.force, verbose_ptxas=a.ptxas))

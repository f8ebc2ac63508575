"""Build recipe of the sm_100a library: nvcc -> dim2d_finite_volume_b200/lib/libdim2d.so.

Run as `python -m dim2d_finite_volume_b200.build` (or through
__graft_entry__.build()).  nvcc cross-compiles for sm_100a without a GPU.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libdim2d.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = [
    "dim2d_capi.cu",
    "dim2d_step.cu",
    "dim2d_interior.cu",
    "dim2d_noalloc.cu",
    "dim2d_open.cu",
    "dim2d_nodebc.cu",
    "dim2d_strip.cu", "dim2d_batch.cu", "dim2d_server.cu",
    "dim2d_masked.cu", "dim2d_persist.cu",
]
HEADERS = ["dim2d_physics.cuh", "dim2d_kernels.cuh", "dim2d_internal.h", "dim2d_open.cuh",
           "dim2d_nodebc.cuh"]

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I", os.path.join(ROOT, "include"),
]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "dim2d.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    objs = []
    obj_dir = os.path.join(LIB_DIR, "_obj")
    os.makedirs(obj_dir, exist_ok=True)
    for s in SOURCES:
        o = os.path.join(obj_dir, s.replace(".cu", ".o"))
        cmd = [NVCC, "-c", os.path.join(CSRC, s), "-o", o] + FLAGS + list(extra)
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        objs.append(o)
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-shared", "-o", tmp] + objs + ["-gencode", "arch=compute_100a,code=sm_100a",
                                                 "-lcudart"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else ())
    print(LIB)

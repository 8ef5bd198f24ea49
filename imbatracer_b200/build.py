"""Builds libimbart.so in-tree for sm_100a with nvcc.

The shared library is the product: the C ABI declared in include/imbart.h. It is built
in place (imbatracer_b200/_lib/libimbart.so) so that it ships with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIBNAME = "libimbart.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Wno-deprecated-gpu-targets", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-Xptxas", "-O3"]

SOURCES_CU = ["trace.cu", "trace_w4.cu", "trace_flat.cu", "hashgrid.cu", "wavefront.cu", "server.cu", "vcm.cu", "gpu_build.cu"]
SOURCES_CPP = ["builder.cpp", "convert.cpp", "error.cpp", "camera.cpp", "accel_file.cpp"]
# Shading and sample generation mirror the reference's separately rounded single-precision
# arithmetic: no fused multiply-add in device code, no contraction in the host camera set-up.
# (The traversal kernels spell out their rounding with intrinsics and keep FMA elsewhere.)
EXTRA_FLAGS = {"wavefront.cu": ["-fmad=false"], "server.cu": ["-fmad=false"], "vcm.cu": ["-fmad=false"],
               "camera.cpp": ["-Xcompiler", "-ffp-contract=off"]}


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def lib_path() -> str:
    return os.path.join(LIBDIR, LIBNAME)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)


def build(verbose: bool = False, ptxas_verbose: bool = False) -> str:
    """Compiles every source into one shared library and returns its path."""
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    objs, cmds = [], []
    inc = ["-I", CSRC, "-I", os.path.join(HERE, "..", "include")]
    for src in SOURCES_CU:
        obj = os.path.join(objdir, src + ".o")
        extra = (["-Xptxas", "-v"] if ptxas_verbose else []) + EXTRA_FLAGS.get(src, [])
        cmds.append([nvcc(), *ARCH, *NVCC_FLAGS, *extra, *inc, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    for src in SOURCES_CPP:
        obj = os.path.join(objdir, src + ".o")
        cmds.append([nvcc(), *NVCC_FLAGS, *EXTRA_FLAGS.get(src, []), *inc, "-x", "c++", "-c", os.path.join(CSRC, src),
                     "-o", obj])
        objs.append(obj)
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        list(ex.map(lambda c: _run(c, verbose), cmds))
    out = lib_path()
    tmp = out + ".tmp"
    _run([nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs, "-lpthread"], verbose)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_verbose="--ptxas" in sys.argv))

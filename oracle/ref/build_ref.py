"""Recipe: compiles the reference's own C++ in place from /root/reference/src into
oracle/_ref/libref.so, against the shims in oracle/ref/shim (TBB subset, AnyDSL buffer
API, libpng declarations, fixed-seed random_device) and the drop-in traversal headers in
include/. Nothing is copied from the reference tree; its build system is not used.
TEST INFRASTRUCTURE ONLY (the product never loads libref.so).
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
ROOT = os.path.dirname(ORACLE)
REF = os.environ.get("IMBART_REFERENCE", "/root/reference")
OUT = os.path.join(ORACLE, "_ref")

REF_SOURCES = [
    "src/imbatracer/core/mesh.cpp",
    "src/imbatracer/core/cpu_adapter.cpp",
    "src/imbatracer/core/gpu_adapter.cpp",
    "src/imbatracer/render/scene.cpp",
    "src/imbatracer/loaders/load_bvh.cpp",
    "src/imbatracer/render/integrators/integrator.cpp",
    "src/imbatracer/render/integrators/pt.cpp",
    "src/imbatracer/render/integrators/vcm.cpp",
    "src/imbatracer/render/integrators/light_vertices.cpp",
    "src/imbatracer/frontend/build_scene.cpp",
    "src/imbatracer/loaders/load_obj.cpp",
    "src/imbatracer/loaders/load_tga.cpp",
    "src/imbatracer/loaders/load_hdr.cpp",
]
OWN_SOURCES = [os.path.join(HERE, "ref_harness.cpp"), os.path.join(HERE, "ref_vcm.cpp"),
               os.path.join(HERE, "ref_scene_io.cpp"), os.path.join(HERE, "ref_pt_rr.cpp")]
ORACLE_C = [os.path.join(ORACLE, "traversal.c")]

FLAGS = ["-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-w"]


def present() -> bool:
    return os.path.isdir(os.path.join(REF, "src", "imbatracer"))


def build(verbose: bool = False) -> str:
    if not present():
        raise SystemExit(f"reference tree not found at {REF}")
    os.makedirs(OUT, exist_ok=True)
    # Where the sources were found, for the CPU tests that read the reference's scene files
    # (oracle.refwrap.reference_root); they copy them elsewhere before loading them.
    with open(os.path.join(OUT, "reference_root.txt"), "w") as f:
        f.write(REF)
    objdir = os.path.join(OUT, "obj")
    os.makedirs(objdir, exist_ok=True)
    inc = ["-I", os.path.join(HERE, "shim"), "-I", os.path.join(REF, "src"), "-I", os.path.join(ROOT, "include"),
           "-include", os.path.join(HERE, "shim", "ref_prelude.h")]
    objs = compile_all(objdir, inc, [], verbose)
    lib = os.path.join(OUT, "libref.so")
    subprocess.run(["g++", "-shared", "-fopenmp", "-Wl,-Bsymbolic", "-o", lib, *objs, "-lm"], check=True)
    build_gpu_grid(verbose)
    build_imbart_linked(verbose)
    return lib


def compile_all(objdir, inc, defines, verbose):
    """The reference sources, the harness and the oracle's traversal into objdir (in parallel)."""
    cmds, objs = [], []
    for src in [os.path.join(REF, s) for s in REF_SOURCES] + OWN_SOURCES:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmds.append(["g++", "-std=c++14", *FLAGS, *defines, *inc, "-c", src, "-o", obj])
        objs.append(obj)
    for src in ORACLE_C:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmds.append(["gcc", "-std=c11", *FLAGS, "-c", src, "-o", obj])
        objs.append(obj)

    def run(cmd):
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        list(ex.map(run, cmds))
    return objs


def build_imbart_linked(verbose: bool = False) -> str | None:
    """The same harness with the reference's traversal entry points taken from libimbart (the
    drop-in boundary) instead of the oracle, and its AnyDSL Platform::Cuda arrays in GPU memory
    (shim_cuda ahead of shim): oracle/_ref/libref_imbart.so. Skipped when libimbart is not
    built yet."""
    imbart_lib = os.path.join(ROOT, "imbatracer_b200", "_lib")
    if not os.path.exists(os.path.join(imbart_lib, "libimbart.so")):
        return None
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    objdir = os.path.join(OUT, "obj_imbart")
    os.makedirs(objdir, exist_ok=True)
    inc = ["-I", os.path.join(HERE, "shim_cuda"), "-I", os.path.join(HERE, "shim"), "-I", os.path.join(REF, "src"),
           "-I", os.path.join(ROOT, "include"), "-include", os.path.join(HERE, "shim", "ref_prelude.h")]
    objs = compile_all(objdir, inc, ["-DIMBART_REF_TRAVERSAL_FROM_IMBART"], verbose)
    lib = os.path.join(OUT, "libref_imbart.so")
    subprocess.run(["g++", "-shared", "-fopenmp", "-Wl,-Bsymbolic", "-o", lib, *objs, "-L", imbart_lib, "-limbart",
                    "-Wl,-rpath,$ORIGIN/../../imbatracer_b200/_lib", "-L", os.path.join(cuda, "lib64"), "-lcudart",
                    "-Wl,-rpath," + os.path.join(cuda, "lib64"), "-lm"], check=True)
    return lib


def build_gpu_grid(verbose: bool = False) -> str | None:
    """The reference's LightVertices against libimbart's GPU photon grid: compiled with
    include/shadow ahead of the reference's src/ (its rangesearch.h replaced by the adapter)
    and linked to the in-tree libimbart; skipped when libimbart is not built yet."""
    imbart_lib = os.path.join(ROOT, "imbatracer_b200", "_lib")
    if not os.path.exists(os.path.join(imbart_lib, "libimbart.so")):
        return None
    inc = ["-I", os.path.join(ROOT, "include", "shadow"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(HERE, "shim"), "-I", os.path.join(REF, "src"),
           "-include", os.path.join(HERE, "shim", "ref_prelude.h")]
    out = os.path.join(OUT, "libref_gpu_grid.so")
    cmd = ["g++", "-std=c++14", *FLAGS, *inc, "-shared", "-o", out, os.path.join(HERE, "ref_gpu_grid.cpp"),
           "-L", imbart_lib, "-limbart", "-Wl,-rpath,$ORIGIN/../../imbatracer_b200/_lib"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    if "--if-present" in sys.argv and not present():
        print(f"reference tree not found at {REF}: oracle/_ref not built")
    else:
        print(build(verbose="-v" in sys.argv))

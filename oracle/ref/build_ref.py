"""Recipe: compiles the reference's own C++ in place from /root/reference/src into
oracle/_ref/libref.so, against the shims in oracle/ref/shim (TBB subset, AnyDSL buffer
API, libpng declarations, fixed-seed random_device) and the drop-in traversal headers in
include/. Nothing is copied from the reference tree; its build system is not used.
TEST INFRASTRUCTURE ONLY (the product never loads libref.so).
"""
import os
import subprocess
import sys

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
    objs = []
    for src in [os.path.join(REF, s) for s in REF_SOURCES] + OWN_SOURCES:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = ["g++", "-std=c++14", *FLAGS, *inc, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    for src in ORACLE_C:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        subprocess.run(["gcc", "-std=c11", *FLAGS, "-c", src, "-o", obj], check=True)
        objs.append(obj)
    lib = os.path.join(OUT, "libref.so")
    subprocess.run(["g++", "-shared", "-fopenmp", "-Wl,-Bsymbolic", "-o", lib, *objs, "-lm"], check=True)
    return lib


if __name__ == "__main__":
    if "--if-present" in sys.argv and not present():
        print(f"reference tree not found at {REF}: oracle/_ref not built")
    else:
        print(build(verbose="-v" in sys.argv))

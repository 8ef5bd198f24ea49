"""imbatracer_b200 — the wavefront hot path of imbatracer on NVIDIA B200 (sm_100a).

The product is libimbart.so (C ABI in include/imbart.h); this package holds its CUDA/C++
sources (csrc/), the in-tree build, ctypes bindings and the host-side mirror of the
reference's scene, ray-queue and integrator interfaces.
"""
__version__ = "0.1.0"

"""Build the CUDA library in-tree: relight_b200/librelight_b200.so (sm_100a).

    python -m relight_b200.build

--fmad=false: the bake kernels round every float expression as the
reference's C++ does (no contraction); the hot traversal code writes its
fused multiply-adds out with __fmaf_rn, which this flag does not affect.
The CUDA runtime is linked statically so the library does not depend on the
runtime version another library in the process (e.g. torch) brought along.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "librelight_b200.so")

SOURCES = ["rl_capi.cu", "rl_lbvh.cu", "rl_denoise.cu", "rl_knn.cu", "rl_bvh.cpp", os.path.join("host", "relight_api.cpp"),
           os.path.join("host", "obj_loader.cpp")]
HEADERS = ["rl_device.cuh", "rl_bvh.h", "rl_lbvh.h", "rl_photon_records.h", os.path.join("..", "..", "include", "relight_b200.h"),
           os.path.join("..", "..", "include", "relight", "Relight.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "--fmad=false", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-Xcompiler", "-ffp-contract=off",
    "-shared", "-cudart", "static",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", OUT + ".tmp"] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


def build_cpp_example(out_dir: str, name: str = "bake_room") -> str:
    """Compile tests/cpp/<name>.cpp, a Relight C++ program, against the C++
    API (include/relight/Relight.h) and this library."""
    src = os.path.join(ROOT, "tests", "cpp", name + ".cpp")
    exe = os.path.join(out_dir, name)
    cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-pthread", "-I", os.path.join(ROOT, "include"), src,
           "-L", HERE, "-lrelight_b200", "-Wl,-rpath," + HERE, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("C++ example failed to build:\n" + r.stdout + r.stderr)
    return exe


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

"""Build libtenes_gpu.so in-tree with nvcc for sm_100a.

    python -m tenes_b200.build          # incremental
    python -m tenes_b200.build --force  # rebuild everything

The library links cuSOLVER (dense projector SVD, simple-update QR) from the
CUDA toolkit and records its directory as the run path.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtenes_gpu.so")
SOURCES = ["kernels.cu", "cholqr.cu", "skinny.cu", "su_fused.cu", "adjoint.cu", "engine.cu", "api.cu",
           "noalloc.cu", "main_entry.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def cuda_home() -> str:
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and os.path.exists(os.path.join(c, "bin", "nvcc")):
            return c
    nvcc = shutil.which("nvcc")
    if nvcc:
        return os.path.dirname(os.path.dirname(os.path.realpath(nvcc)))
    raise RuntimeError("nvcc not found")


def python_defines():
    """Where tenes_gpu_main finds the Python runtime and the packages of the
    front end (numpy, scipy) when the calling process has no interpreter:
    this interpreter's shared libpython and site-packages."""
    import sysconfig
    lib = os.path.join(sysconfig.get_config_var("LIBDIR") or "", sysconfig.get_config_var("INSTSONAME") or "")
    if not os.path.exists(lib):
        lib = "libpython3.so"
    site = sysconfig.get_paths()["purelib"]
    return [f'-DTG_PY_LIB="{lib}"', f'-DTG_PY_SITE="{site}"']


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    cuda = cuda_home()
    nvcc = os.path.join(cuda, "bin", "nvcc")
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "tenes_gpu.h"))
    objs = []
    common = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
              "-I", CSRC, "--expt-relaxed-constexpr"] + ARCH
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if force or _newer(o, [s, __file__] + headers):
            cmd = [nvcc, "-c", s, "-o", o] + common + (python_defines() if src.endswith(".cpp") else [])
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    libdir = os.path.join(cuda, "lib64")
    if force or _newer(LIB, objs):
        cmd = [nvcc, "-shared", "-o", LIB] + objs + ARCH + [
            "-L", libdir, "-lcusolver", "-lcublas", "-ldl", "-Xlinker", "-rpath=" + libdir]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    sys.exit(0)

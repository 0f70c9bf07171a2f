"""In-tree build of libincrmt_gpu.so for sm_100a with nvcc.

Usage: python -m incrmt_b200.build   (or incrmt_b200.build.build(), and
build_host() for the C++ host programs in incrmt_b200/host)
The library lands next to this file so it travels with the repository
snapshot; nothing is installed into site-packages.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libincrmt_gpu.so")
SOURCES = ["capi.cu", "mg.cu", "sim.cu", "noalloc.cu", "unet.cu", "learned.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def _sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = _sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "incrmt.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compiles the CUDA sources into incrmt_b200/libincrmt_gpu.so if stale."""
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    cmd += _sources() + ["-o", LIB]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


def build_host(verbose=False):
    """Builds the C++ host programs (incrmt_b200/host: ftest_gpu) over the library."""
    build(verbose=verbose)
    out = None if verbose else subprocess.DEVNULL
    subprocess.run(["make", "-C", os.path.join(HERE, "host")], check=True, stdout=out)
    return os.path.join(HERE, "host", "ftest_gpu")


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    build_host(verbose=True)
    print(LIB)

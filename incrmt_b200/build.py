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
SOURCES = ["capi.cu", "mg.cu", "sim.cu", "noalloc.cu", "unet.cu", "learned.cu", "conv_tc.cu"]
# The CUDA runtime is linked as a shared library: in a process that also
# loads PyTorch, the library and torch then use one runtime (the soname
# libcudart.so.12 resolves to the copy already loaded), so neither's exit
# handlers tear down state the other still uses.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared", "-cudart", "shared",
]


def _sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = _sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps += [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include"))]
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compiles the CUDA sources into incrmt_b200/libincrmt_gpu.so if stale:
    each source to an object in incrmt_b200/_build (in parallel), then one
    link."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    nvcc = os.environ.get("NVCC", "nvcc")
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    flags = [f for f in NVCC_FLAGS if f != "-shared"]

    def compile_one(src):
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        cmd = [nvcc] + flags + inc + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        return obj, r

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, _sources()))
    for obj, r in results:
        if r.stdout or r.stderr:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise subprocess.CalledProcessError(r.returncode, "nvcc", r.stdout, r.stderr)
    cmd = [nvcc] + NVCC_FLAGS + [o for o, _ in results] + ["-o", LIB]
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

"""Build recipe for the fishfry_b200 native code (sm_100a only).

  python -m fishfry_b200.build          # lib/libfishfry.so and bin/fishfry

Everything is compiled in-tree with nvcc for `-gencode arch=compute_100a,code=sm_100a`;
no JIT cache and no other architecture.  Rebuilds only what is out of date.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "lib", "libfishfry.so")
BIN = os.path.join(HERE, "bin", "fishfry")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-pthread", "-I" + INCLUDE]

LIB_SOURCES = ["ff_solve.cu", "ff_bluestein.cu", "ff_field.cu", "ff_batch.cu", "ff_batch_f64.cu", "ff_batch_f32.cu",
               "ff_serve.cu", "ff_slab.cu"]
HEADERS = ["ff_fft.cuh", "ff_tiles.cuh", "ff_status.hpp", "ff_batch.hpp", "ff_batch_dev.cuh", "ff_bluestein.hpp",
           "ff_plan.hpp"]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _host_cxx():
    # the system g++ (the image also carries a wrapper that lacks some spec files)
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_lib(verbose=False, force=False):
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES]
    shared = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "fishfry.h"), os.path.abspath(__file__)]
    objdir = os.path.join(HERE, "lib", "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, os.path.basename(s) + ".o") for s in srcs]
    # a translation unit is rebuilt when it, a shared header or this recipe is newer than its object
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _stale(o, [s] + shared)]
    if not todo and not _stale(LIB, objs):
        return LIB
    # translation units compile in parallel (each is one nvcc process); each
    # object is written under a temporary name and renamed when complete
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        futs = [ex.submit(_run, [_nvcc()] + NVCC_FLAGS + ["-c", s, "-o", o + ".tmp"], verbose) for s, o in todo]
        for f in futs:
            f.result()
    for _, o in todo:
        os.replace(o + ".tmp", o)
    tmp = LIB + ".tmp"
    _run([_nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart", "-lpthread"], verbose)
    os.replace(tmp, LIB)
    return LIB


def build_bin(verbose=False, force=False):
    src = os.path.join(CSRC, "main.cpp")
    deps = [src, LIB, os.path.join(INCLUDE, "ParisPencil.hpp"), os.path.join(INCLUDE, "FishFry.hpp"),
            os.path.join(INCLUDE, "TimeStamp.hpp"), os.path.join(INCLUDE, "fishfry.h")]
    if not force and not _stale(BIN, deps):
        return BIN
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    cuda = os.path.dirname(os.path.dirname(_nvcc()))
    _run([_host_cxx(), "-O2", "-std=c++17", "-I" + INCLUDE, "-I" + os.path.join(cuda, "include"), src, "-o", BIN,
          "-L" + os.path.dirname(LIB), "-lfishfry", "-Wl,-rpath,$ORIGIN/../lib",
          "-L" + os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(cuda, "lib64")], verbose)
    return BIN


def build(verbose=False, force=False):
    build_lib(verbose, force)
    build_bin(verbose, force)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)

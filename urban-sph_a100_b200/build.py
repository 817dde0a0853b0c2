"""Builds lib/libsph_b200.so (every CUDA source of csrc/ for sm_100a) and
lib/sophia_b200, the native case runner (csrc/sophia_b200.cpp, host C++ over
the library's C ABI).

Usage: python build.py [-j N]    (also called by __graft_entry__.build)
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
OBJ_DIR = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(LIB_DIR, "libsph_b200.so")
DRIVER_SRC = os.path.join(CSRC, "sophia_b200.cpp")
DRIVER = os.path.join(LIB_DIR, "sophia_b200")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-ccbin", "/usr/bin/g++"]


def _compile(src, extra):
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "sph_isph.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj


def build(jobs=None, extra=()):
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    with cf.ThreadPoolExecutor(max_workers=jobs or len(srcs)) as ex:
        objs = list(ex.map(lambda s: _compile(s, list(extra)), srcs))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s" % r.stderr)
    build_driver()
    return LIB


def build_driver():
    """The native runner, linked to the library beside it (rpath $ORIGIN)."""
    deps = [DRIVER_SRC, LIB, os.path.join(ROOT, "include", "sph_isph.h")]
    if os.path.exists(DRIVER) and all(os.path.getmtime(DRIVER) >= os.path.getmtime(d) for d in deps):
        return DRIVER
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-I" + os.path.join(ROOT, "include"), DRIVER_SRC,
           "-L" + LIB_DIR, "-lsph_b200", "-Wl,-rpath,$ORIGIN", "-Wl,--allow-shlib-undefined", "-o", DRIVER]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("driver build failed:\n%s" % r.stderr)
    return DRIVER


if __name__ == "__main__":
    print(build())

"""Builds the reference's CUDA program for B200 (sm_100a), as a timed baseline.

The reference (hyen0929/Urban-SPH_A100) is one CUDA translation unit,
SOPHIA_gpu.cu, with no build system of its own.  This recipe copies its
sources into a temporary directory outside the repository, applies the patch
set below, compiles the copy with nvcc for sm_100a and keeps only the
executable, in baseline/_ref/ (git-ignored; it travels to the GPU box with
the repository).  The reference tree itself is never written.

Patch set (each anchor must match exactly, else the build stops):
  1. g_str / g_end get num_cells + 1 entries (allocation and both resets,
     ISPH_Calc.cuh:28,331-332,342-343).  KERNEL_reorder writes
     g_str[num_cells] / g_end[num_cells] for the dummy key num_cells
     (functions_NNPS.cuh:833-838), one entry past the shipped allocation,
     whenever a deck holds i_type 3 records.
  2. A wall-clock timer around the time loop of ISPH_Calc
     (ISPH_Calc.cuh:476-525): it starts after SOPHIA_WARMUP steps (default
     3; step 0 holds the NNPS and the VTK write) with a device synchronise
     and prints "SOPHIA_TIMED steps=<k> seconds=<s>" after the loop.
Everything else is as shipped: Real = float, the hard-wired Case-H
constants, one PPE sweep per step, cudaDeviceSynchronize after every launch.
The program reads ./input/solv.txt, ./input/data.txt and
./input/CaseH_n10.txt relative to its working directory and writes VTK into
./CaseH_n10_DDF(WL6,dt=2.5e-5,KGC,IBM_WM)/ (functions_OUTPUT.cuh:142-144).

    python baseline/build_ref_cuda.py [--ref DIR] [--double]

--double builds the FP64 variant (Variable_Type.cuh: typedef double Real).
"""
import argparse
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

# (the reference defines `count` as a macro, so no std::chrono here)
TIMER_DECL = """
#include <time.h>
static double sophia_wall_s() {
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
"""


def patch(src_dir):
    def edit(name, pairs):
        path = os.path.join(src_dir, name)
        with open(path) as f:
            s = f.read()
        for old, new, count in pairs:
            n = s.count(old)
            if n != count:
                raise RuntimeError(f"{name}: expected {count} match(es) of {old!r}, found {n}")
            s = s.replace(old, new)
        with open(path, "w") as f:
            f.write(s)

    edit("ISPH_Calc.cuh", [
        ("cudaMalloc((void**)&g_str,sizeof(int_t)*num_cells);",
         "cudaMalloc((void**)&g_str,sizeof(int_t)*(num_cells+1));", 1),
        ("cudaMalloc((void**)&g_end,sizeof(int_t)*num_cells);",
         "cudaMalloc((void**)&g_end,sizeof(int_t)*(num_cells+1));", 1),
        ("cudaMemset(g_str,cu_memset,sizeof(int_t)*num_cells);",
         "cudaMemset(g_str,cu_memset,sizeof(int_t)*(num_cells+1));", 2),
        ("cudaMemset(g_end,0,sizeof(int_t)*num_cells);",
         "cudaMemset(g_end,0,sizeof(int_t)*(num_cells+1));", 1),
        ("void*ISPH_Calc(void*arg){", TIMER_DECL + "void*ISPH_Calc(void*arg){", 1),
        ("\twhile(1){\n\n\t\tif(ngpu==1){",
         "\tint sophia_warm=getenv(\"SOPHIA_WARMUP\")?atoi(getenv(\"SOPHIA_WARMUP\")):3;\n"
         "\tint sophia_count0=count,sophia_c0=-1;\n\tdouble sophia_t0=0.0;\n"
         "\twhile(1){\n\t\tif(count-sophia_count0==sophia_warm){cudaDeviceSynchronize();"
         "sophia_t0=sophia_wall_s();sophia_c0=count;}\n\n\t\tif(ngpu==1){", 1),
        ("\t\tpthread_barrier_wait(&barrier);\n\t\tif(time>=time_end) break;\n\n\t}\n",
         "\t\tpthread_barrier_wait(&barrier);\n\t\tif(time>=time_end) break;\n\n\t}\n"
         "\tcudaDeviceSynchronize();\n"
         "\tif(sophia_c0>=0) printf(\"SOPHIA_TIMED steps=%d seconds=%.6f\\n\",count-sophia_c0,"
         "sophia_wall_s()-sophia_t0);\n\tfflush(stdout);\n", 1),
    ])


def build(ref_dir, double=False):
    if not os.path.isfile(os.path.join(ref_dir, "SOPHIA_gpu.cu")):
        raise FileNotFoundError(f"no SOPHIA_gpu.cu under {ref_dir}")
    os.makedirs(OUT_DIR, exist_ok=True)
    exe = os.path.join(OUT_DIR, "sophia_gpu_sm100a" + ("_fp64" if double else ""))
    tmp = tempfile.mkdtemp(prefix="sophia_ref_cuda.")
    try:
        for name in os.listdir(ref_dir):
            if name.endswith((".cu", ".cuh")):
                shutil.copy(os.path.join(ref_dir, name), tmp)
        for name in os.listdir(tmp):
            os.chmod(os.path.join(tmp, name), 0o644)
        patch(tmp)
        if double:
            path = os.path.join(tmp, "Variable_Type.cuh")
            with open(path) as f:
                s = f.read()
            if s.count("typedef float Real") != 1:
                raise RuntimeError("Variable_Type.cuh: no single 'typedef float Real'")
            with open(path, "w") as f:
                f.write(s.replace("typedef float Real", "typedef double Real"))
        cmd = [NVCC, "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "--expt-relaxed-constexpr",
               "-w", "SOPHIA_gpu.cu", "-lpthread", "-o", exe]
        r = subprocess.run(cmd, cwd=tmp, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stderr[-4000:])
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return exe


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--ref", default=os.environ.get("REF_DIR", "/root/reference"))
    ap.add_argument("--double", action="store_true")
    a = ap.parse_args()
    print(build(a.ref, a.double))
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Build recipe for libpfb200.so (sm_100a).  Run ``python -m pyfourier_b200._build``."""

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpfb200.so")
SOURCES = ["pfb_capi.cu", "pfb_plan.cu", "pfb_spread.cu", "pfb_interp.cu", "pfb_glue.cu", "pfb_noalloc.cu", "pfb_fast.cu",
           "pfb_fft.cu", "pfb_dcf.cu", "pfb_grog.cu", "pfb_psf.cu", "pfb_sort.cu", "pfb_pool.cu"]


def nvcc_path():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else shutil.which("nvcc")


def build(force=False, verbose=False, extra_flags=()):
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, "pfb_common.cuh"), os.path.join(ROOT, "include", "pfb200.h")]
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    nvcc = nvcc_path()
    if nvcc is None:
        raise RuntimeError("nvcc not found; set CUDA_HOME")
    cuda_home = os.path.dirname(os.path.dirname(nvcc))
    flags = ["-O3", "-std=c++17", "-lineinfo", "-gencode", "arch=compute_100a,code=sm_100a",
             "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"),
             *extra_flags]
    objdir = os.path.join(HERE, "_objs")
    os.makedirs(objdir, exist_ok=True)
    procs, objs = [], []
    for src in srcs:
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        cmd = [nvcc, *flags, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd)))
    failed = [src for src, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    link = [nvcc, "-shared", "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a",
            "-o", LIB + ".tmp", *objs, "-L", os.path.join(cuda_home, "lib64"), "-lcufft",
            "-Xlinker", "-rpath," + os.path.join(cuda_home, "lib64")]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra_flags=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])

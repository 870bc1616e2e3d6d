"""Build liblcmc.so (CUDA C++ for sm_100a) in-tree with nvcc.

``python -m parellel_mc_mpi_for_liquidcrystalsystems_b200.build`` or
``build_library()``.  Object files go to ``_build/`` beside this file, the
shared library to ``liblcmc.so`` in this package directory (both ignored by
git; the .so travels with the working tree).
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "liblcmc.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-I", os.path.join(REPO, "include"), "-Xptxas", "-warn-spills"]
# The FP64 kernel must not contract a*b+c into an FMA: it reproduces the CPU
# oracle bit for bit.
SOURCES = {
    "lcmc_sweep_exact.cu": ["-fmad=false"],
    "lcmc_sweep_fast.cu": [],
    "lcmc_rebin.cu": ["-fmad=false"],  # builds the trial moves (same arithmetic as the FP64 kernel)
    "lcmc_misc.cu": ["-fmad=false"],
    "lcmc_api.cu": ["-fmad=false"],
    "lcmc_pairtest.cu": [],
    "lcmc_pairtest64.cu": ["-fmad=false"],
    "lcmc_noalloc.cu": ["-fmad=false"],
    "lcmc_mlp.cu": [],
    "lcmc_da.cu": [],
    # FP32 pair terms contract freely; its FP64 distance and scaling use rounded
    # intrinsics (the FP64 kernel's arithmetic in any contraction setting)
    "lcmc_screen.cu": [],
    "lcmc_io.cu": [],
}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _needs(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(verbose=False, ptxas_info=False):
    os.makedirs(OUT, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(REPO, "include", "lcmc.h"))
    cc = nvcc()
    jobs = []
    objs = []
    for src, extra in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OUT, src.replace(".cu", ".o"))
        objs.append(o)
        if _needs(o, [s] + headers + [__file__]) or ptxas_info:
            cmd = [cc, *ARCH, *COMMON, *extra, "-c", s, "-o", o]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or ptxas_info or r.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError("nvcc failed: " + os.path.basename(cmd[-3]))
    if jobs or not os.path.exists(LIB):
        tmp = LIB + ".tmp"
        cmd = [cc, *ARCH, "-shared", "-o", tmp, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build_library(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))

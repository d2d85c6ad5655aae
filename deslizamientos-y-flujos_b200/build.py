"""Builds libgfsph.so (the CUDA C-ABI library) in this directory for sm_100a.

The kernels are compiled with --fmad=false: each FP32 multiply and add rounds
on its own, as in the reference's FP32 Fortran build, so the per-particle
arithmetic can be compared bit for bit with the CPU oracle.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libgfsph.so")
RUN_EXE = os.path.join(HERE, "gfsph_run")
BUILD_DIR = os.path.join(HERE, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC", "-Xptxas", "-v",
]


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, log):
    res = subprocess.run(cmd, capture_output=True, text=True)
    log.append(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError("build failed:\n" + log[-1])


def build(verbose=False, force=False):
    """Compiles csrc/ into libgfsph.so; returns the library path."""
    srcs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))]
    srcs += [os.path.join(HERE, "host", f) for f in sorted(os.listdir(os.path.join(HERE, "host")))]
    srcs += [os.path.join(HERE, "..", "include", "gfsph.h")]
    if not force and os.path.exists(OUT) and os.path.exists(RUN_EXE):
        newest = max(os.path.getmtime(s) for s in srcs)
        if os.path.getmtime(OUT) >= newest:
            return OUT
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    log = []
    api_o = os.path.join(BUILD_DIR, "gfsph_api.o")
    noalloc_o = os.path.join(BUILD_DIR, "gfsph_noalloc.o")
    cg_o = os.path.join(BUILD_DIR, "gfsph_cg.o")
    gfl_o = os.path.join(BUILD_DIR, "gfsph_gfl.o")
    dem_o = os.path.join(BUILD_DIR, "gfsph_dem.o")
    _run([nvcc, *NVCC_FLAGS, "-c", os.path.join(CSRC, "gfsph_api.cu"), "-o", api_o], log)
    _run([nvcc, *NVCC_FLAGS, "-c", os.path.join(CSRC, "gfsph_noalloc.cu"), "-o", noalloc_o], log)
    _run([nvcc, *NVCC_FLAGS, "-c", os.path.join(CSRC, "gfsph_cg.cu"), "-o", cg_o], log)
    _run([nvcc, *NVCC_FLAGS, "-c", os.path.join(CSRC, "gfsph_gfl.cu"), "-o", gfl_o], log)
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-c",
          os.path.join(CSRC, "gfsph_dem.cpp"), "-o", dem_o], log)
    tmp = OUT + ".tmp"
    _run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", api_o, noalloc_o, cg_o, gfl_o, dem_o,
          "-o", tmp, "-lcudart"], log)
    os.replace(tmp, OUT)
    # the C++ host driver (reads the reference's input files, drives the ABI)
    host = os.path.join(HERE, "host")
    run_tmp = RUN_EXE + ".tmp"
    _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", os.path.join(host, "gfsph_inputs.cpp"),
          os.path.join(host, "gfsph_run.cpp"), "-L" + HERE, "-lgfsph", "-Wl,-rpath,$ORIGIN", "-o", run_tmp], log)
    os.replace(run_tmp, RUN_EXE)
    with open(os.path.join(BUILD_DIR, "build.log"), "w") as f:
        f.write("\n".join(log))
    if verbose:
        print("\n".join(log))
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force=True)
    print(OUT)

"""Build libkfvm_b200.so in-tree: sm_100a CUDA kernels + host C++ (C ABI).

nvcc -gencode arch=compute_100a,code=sm_100a for the .cu files; g++ without FMA
contraction for the FP64 weight precompute (its LU must reproduce bit for bit);
LAPACK dgetrf/dgetrs from the OpenBLAS bundled with scipy.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libkfvm_b200.so")
RUN = os.path.join(HERE, "kfvm_run")
HOST_SOURCES = ["host/kfvm_host.cpp", "host/kfvm_run.cpp"]

CU_SOURCES = ["kernels.cu", "recon_tc.cu", "mlp.cu", "ic.cu", "errest.cu", "forcing.cu", "stats.cu", "exchange.cu",
              "capi.cu"]
CXX_SOURCES = ["stencil_weights.cpp", "plotfile.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _openblas():
    import scipy
    d = os.path.dirname(scipy.__file__) + ".libs"
    for f in sorted(os.listdir(d)):
        if f.startswith("libscipy_openblas") and f.endswith(".so"):
            return d, os.path.join(d, f)
    raise RuntimeError("scipy's bundled OpenBLAS not found")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False):
    """Compile every source of the library for sm_100a; returns the .so path."""
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "kfvm_b200.h"))
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", "-ccbin", "g++", "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            r = _run(cmd)
            if verbose or ptxas_info:
                sys.stdout.write(r.stdout + r.stderr)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-c", s, "-o", o])
    bdir, blas = _openblas()
    if _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", LIB, *objs, blas, "-ccbin", "g++",
              f"-Xlinker=-rpath,{bdir}", "-lcudart"])
    # C++ host driver (the counterpart of the reference's kfvm.ex)
    host = [os.path.join(HERE, f) for f in HOST_SOURCES]
    hdeps = host + [os.path.join(HERE, "host", "kfvm_host.hpp"), os.path.join(ROOT, "include", "kfvm_b200.h"), LIB]
    if _stale(RUN, hdeps):
        _run(["g++", "-O2", "-std=c++17", "-o", RUN, *host, f"-L{HERE}", "-lkfvm_b200",
              "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))

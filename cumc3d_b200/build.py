"""Build recipe of the CUDA engine (sm_100a) into an in-tree shared library.

    python -m cumc3d_b200.build

Three translation units:
  engine.cu     stage kernels, ghost fills, time loop, C-ABI   (--fmad=false)
  flux_fp64.cu  fused face-flux kernel, plain FP64 form          (--fmad=false)
  flux_fp32.cu  fused face-flux kernel, FP32 form                (FMA, fast div/sqrt)
--fmad=false keeps every FP64 expression in the reference's rounding order
(no contraction into fused multiply-adds), which is what makes the plain form
reproduce the Fortran semantics bit for bit.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libcumc3d_gpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr"]
UNITS = [
    ("engine.cu", ["--fmad=false"]),
    ("flux_fp64.cu", ["--fmad=false"]),
    ("flux_fp32.cu", ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]),
    ("batch_host.cu", ["--fmad=false"]),
    ("batch_fp64.cu", ["--fmad=false"]),
    ("batch_fp32.cu", ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]),
    ("noalloc.cu", ["--fmad=false"]),
    ("learned.cu", ["--fmad=false"]),
    ("poisson.cu", ["--fmad=false"]),
]


def _nvcc():
    for c in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if os.path.exists(c) or c == "nvcc":
            return c


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "cumc3d_gpu.h"))
    objs = []
    jobs = []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [_nvcc()] + ARCH + COMMON + flags + ["-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
        return r.stderr

    with ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        outs = list(ex.map(run, jobs))
    if verbose:
        for o in outs:
            sys.stderr.write(o)
    if force or jobs or not os.path.exists(LIB):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

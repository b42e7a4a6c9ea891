"""Build the B200 FFT libraries in-tree.

    python notorious-fft_b200/build.py            # both precisions
    python notorious-fft_b200/build.py --only d   # double only

Outputs (git-ignored, shipped with the tree):
    notorious-fft_b200/lib/libnotorious_fft.so    notorious_fft_real = double
    notorious-fft_b200/lib/libnotorious_fftf.so   notorious_fft_real = float

Every CUDA source is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with line info for ncu.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["nfft_kernels.cu", "nfft_plan.cu", "nfft_api.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
PRECISIONS = {
    "d": ("libnotorious_fft.so", ["-DNFFT_REAL=double"]),
    "f": ("libnotorious_fftf.so", ["-DNFFT_REAL=float", "-DNOTORIOUS_FFT_SINGLE"]),
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "notorious_fft.h"))
    return hs


def compile_one(src: str, prec: str, extra: list[str], verbose_ptxas: bool) -> str:
    obj = os.path.join(BUILD, f"{os.path.splitext(src)[0]}_{prec}.o")
    deps = [os.path.join(CSRC, src)] + _headers()
    if _newer(obj, deps) and not verbose_ptxas:
        return obj
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
           "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src} ({prec}):\n{r.stderr}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    return obj


def build(only: str | None = None, jobs: int = 6, verbose_ptxas: bool = False) -> list[str]:
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    precs = [only] if only else list(PRECISIONS)
    outs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = {}
        for p in precs:
            for s in SOURCES:
                futs[(p, s)] = ex.submit(compile_one, s, p, PRECISIONS[p][1], verbose_ptxas)
        objs = {k: f.result() for k, f in futs.items()}
    for p in precs:
        name = PRECISIONS[p][0]
        out = os.path.join(LIB, name)
        pobjs = [objs[(p, s)] for s in SOURCES]
        if not _newer(out, pobjs):
            cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-Xlinker", "-Bsymbolic", "-o", out, *pobjs,
                   "-lcudart_static", "-ldl", "-lrt", "-lpthread"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link failed for {name}:\n{r.stderr}")
        outs.append(out)
    return outs


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=sorted(PRECISIONS))
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v resource usage")
    ap.add_argument("-j", type=int, default=6)
    args = ap.parse_args()
    for o in build(args.only, args.j, args.ptxas):
        print(o)

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
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

QUEUE_BRANCHES = [f"nfft_queue_b{k}.cu" for k in range(5)]
SOURCES = ["nfft_kernels.cu", "nfft_plan.cu", "nfft_api.cu", "nfft_noalloc.cu", "nfft_tc.cu",
           "nfft_queue_build.cu", "nfft_queue_kernel.cu"] + QUEUE_BRANCHES + [f"nfft_lean_s{k}.cu" for k in range(8)]
# The persistent queue kernel and its branch functions are relocatable device
# code (linked by nvcc -dlink), so the branch units compile in parallel.  They
# read data that other CTAs wrote earlier in the same launch: global loads
# must be served by L2 (-dlcm=cg).  The branches get the kernel's register
# budget (256 threads, 2 CTAs per SM).
RDC_SOURCES = ["nfft_queue_kernel.cu"] + QUEUE_BRANCHES
_QUEUE_FLAGS = ["-rdc=true", "-Xptxas", "-dlcm=cg"]
SOURCE_FLAGS = {"nfft_queue_kernel.cu": _QUEUE_FLAGS}
SOURCE_FLAGS.update({b: _QUEUE_FLAGS + ["-maxrregcount=128"] for b in QUEUE_BRANCHES})
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
PRECISIONS = {
    "d": ("libnotorious_fft.so", ["-DNFFT_REAL=double"]),
    "f": ("libnotorious_fftf.so", ["-DNFFT_REAL=float", "-DNFFT_REAL_IS_FLOAT=1", "-DNOTORIOUS_FFT_SINGLE"]),
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _digest(deps: list[str], cmd: list[str]) -> str:
    h = hashlib.sha256(" ".join(cmd).encode())
    for d in sorted(deps):
        with open(d, "rb") as f:
            h.update(d.encode())
            h.update(f.read())
    return h.hexdigest()


def _fresh(target: str, deps: list[str], cmd: list[str]) -> bool:
    """True when target exists and was built from exactly these inputs."""
    stamp = target + ".stamp"
    if not (os.path.exists(target) and os.path.exists(stamp)):
        return False
    with open(stamp) as f:
        return f.read().strip() == _digest(deps, cmd)


def _stamp(target: str, deps: list[str], cmd: list[str]) -> None:
    with open(target + ".stamp", "w") as f:
        f.write(_digest(deps, cmd))


def _includes(path: str, seen: set) -> None:
    """Local headers included by `path`, transitively."""
    import re
    with open(path) as f:
        for name in re.findall(r'^\s*#\s*include\s+"([^"]+)"', f.read(), flags=re.M):
            for base in (os.path.dirname(path), CSRC, INCLUDE):
                cand = os.path.normpath(os.path.join(base, name))
                if os.path.exists(cand):
                    if cand not in seen:
                        seen.add(cand)
                        _includes(cand, seen)
                    break


def _headers(src: str) -> list[str]:
    seen: set = set()
    _includes(os.path.join(CSRC, src), seen)
    return sorted(seen)


def compile_one(src: str, prec: str, extra: list[str], verbose_ptxas: bool) -> str:
    obj = os.path.join(BUILD, f"{os.path.splitext(src)[0]}_{prec}.o")
    deps = [os.path.join(CSRC, src)] + _headers(src)
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
           "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    if _fresh(obj, deps, cmd) and not verbose_ptxas:
        return obj
    digest = _digest(deps, cmd)   # inputs as compiled (edits during the compile force a rebuild next time)
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src} ({prec}):\n{r.stderr}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    with open(obj + ".stamp", "w") as f:
        f.write(digest)
    return obj


def build(only: str | None = None, jobs: int = 8, verbose_ptxas: bool = False) -> list[str]:
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    precs = [only] if only else list(PRECISIONS)
    outs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = {}
        for p in precs:
            for s in SOURCES:
                futs[(p, s)] = ex.submit(compile_one, s, p, PRECISIONS[p][1] + SOURCE_FLAGS.get(s, []), verbose_ptxas)
        objs = {k: f.result() for k, f in futs.items()}
    for p in precs:
        name = PRECISIONS[p][0]
        out = os.path.join(LIB, name)
        # device link of the relocatable queue objects
        robjs = [objs[(p, s)] for s in RDC_SOURCES]
        dlink = os.path.join(BUILD, f"queue_dlink_{p}.o")
        dcmd = [nvcc(), *ARCH, "-dlink", "-Xcompiler", "-fPIC", "-o", dlink, *robjs]
        ddeps = robjs + [o + ".stamp" for o in robjs]
        if not _fresh(dlink, ddeps, dcmd):
            r = subprocess.run(dcmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"device link failed for {name}:\n{r.stderr}")
            _stamp(dlink, ddeps, dcmd)
        pobjs = [objs[(p, s)] for s in SOURCES] + [dlink]
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-Xlinker", "-Bsymbolic", "-Xlinker", "--no-undefined",
               "-o", out, *pobjs, "-lcudart_static", "-ldl", "-lrt", "-lpthread"]
        deps = pobjs + [o + ".stamp" for o in pobjs]
        if not _fresh(out, deps, cmd):
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link failed for {name}:\n{r.stderr}")
            _stamp(out, deps, cmd)
        outs.append(out)
    return outs


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=sorted(PRECISIONS))
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v resource usage")
    ap.add_argument("-j", type=int, default=8)
    args = ap.parse_args()
    for o in build(args.only, args.j, args.ptxas):
        print(o)

"""Benchmark of the B200 FFT engine (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2c|c1|ragged|split_tc|bluestein]

Workloads (synthetic, seeded; no dataset is involved):
  c2c  (default) batched complex DFT, FP64, N = 65536 x 4096 transforms per
       GPU; one step = notorious_fft_dft then notorious_fft_invdft over the
       batch.  The split-tensor-core FP32 form runs the same shape and is
       reported beside it.  4 GiB per array > L2, so no L2 flush is needed.
  c1   256 x N=4096 FP64 dft + invdft (32 MiB per array < L2: the L2 is
       flushed by a 256 MiB write between timed steps).
  ragged, split_tc, bluestein  profiling workloads (one ragged batch; the
       float library's split-TC or plain form on N = 65536 x 512; FP64
       Bluestein N = 1,000,003 x 4): time per call only.

Metric: HBM GB/s of algorithmic traffic (one read + one write of every
transform's input and output, 2 N sizeof(cmpl) bytes per transform) on the
device-resident batch, whole job (sum over GPUs).  `e2e` is the same metric
through the C ABI with pinned host buffers (host<->device copies inside the
timed region); `e2e_pageable` the same calls on pageable host buffers (the
library stages them through its own pinned buffers).  Multi-GPU runs shard the batch: every rank runs its own
4096 transforms (weak scaling), no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "notorious-fft_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "HBM GB/s, % roofline: FP64 drop-in vs batched split-TC form at stated error"

# DRAM bytes per transform (dram__bytes_read.sum + dram__bytes_write.sum over
# both pass kernels) from an ncu capture of 256 transforms of the same shape;
# scaled to the batch for roofline.traffic.
MEASURED_TRAFFIC_PER_TRANSFORM = {("c2c", 65536): 3.82e6}

WORKLOADS = {
    "c2c": dict(N=65536, batch=4096, l2="inputs 4 GiB per array > L2 (no flush)", flush=False),
    "c1": dict(N=4096, batch=256, l2="L2 flushed (256 MiB write) between steps", flush=True),
    # ragged batch in one persistent launch; `batch` = number of transforms
    "ragged": dict(N=0, batch=20000, l2="L2 flushed (256 MiB write) between steps", flush=True),
    # profiling workload: the FP64 Bluestein case of the transform mix (prime N)
    "bluestein": dict(N=1000003, batch=4, l2="arrays 64 MiB (no flush)", flush=False),
    # profiling workload: the float library's precision forms on N = 65536 x batch
    "split_tc": dict(N=65536, batch=512, l2="inputs 256 MiB per array > L2 (no flush)", flush=False),
}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "25",
                                       "-i", str(index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        # wait (at most ~2 s) for the first sample, so the sampler is running
        # when the timed region starts
        t0 = time.time()
        while self.p is not None and time.time() - t0 < 2.0:
            self.f.flush()
            if os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.strip().split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def cpu_run(kinds, dims, batch, threads, reps, lib="libref_d_avx2.so", prec="f64", listfile=None):
    """Run the reference's own CPU path (oracle/_ref, compiled from the
    reference sources) through oracle/_build/cpu_bench on the host cores.
    Returns the harness's JSON record (best-of-reps seconds and every rep's
    seconds), or None when the reference build is missing."""
    exe = os.path.join(ROOT, "oracle", "_build", "cpu_bench")
    so = os.path.join(ROOT, "oracle", "_ref", lib)
    if not (os.path.exists(exe) and os.path.exists(so)):
        return None
    if listfile is not None:
        cmd = [exe, so, prec, "ragged", listfile, "-", str(threads), str(reps)]
    else:
        cmd = [exe, so, prec, ",".join(kinds), "x".join(map(str, dims)), str(batch), str(threads), str(reps)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        return None
    return json.loads(r.stdout.strip().splitlines()[-1])


def cpu_entry(rec, nbytes, sample, lib, threads, extra=None):
    """A configuration's cpu_baseline object from a cpu_bench record."""
    if rec is None:
        return {"unavailable": "reference CPU build missing (oracle/_ref)"}
    e = {"ms": round(rec["seconds"] * 1e3, 3), "gb_s": round(nbytes / rec["seconds"] / 1e9, 2),
         "cores": threads, "cpu": cpu_model(), "kind": "reference", "build": lib, "sample": sample}
    if extra:
        e.update(extra)
    return e


def run_reference_arm(args, wl):
    """The reference's own CPU implementation of the workload, timed on the
    host cores: every step is the whole batch (dft then invdft of all its
    transforms), OpenMP over the batch with one aux per thread, the
    reference built -O3 -fopenmp -mavx2 -mfma from its sources.  The first W
    reps are warm-up; the K reps after them are the timed steps."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    threads = host_cores()
    N, B = wl["N"], wl["batch"]
    t0 = time.time()
    rec = cpu_run(["dft", "invdft"], [N], B, threads, args.warmup + args.steps)
    if rec is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build missing (oracle/_ref)"}))
        return
    steps = rec["rep_seconds"][args.warmup:]
    sec = sum(steps) / len(steps)
    bytes_per_step = 2 * B * 2 * N * 16
    gbs = bytes_per_step / sec / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(gbs, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (uniform[-1,1), splitmix64 seeded)",
        "config": {"workload": f"c2c fp64 N={N} x{B} dft+invdft per GPU", "N": N, "batch": B, "l2": wl["l2"],
                   "parallelism": f"batch-sharded x{world}"},
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "cpu": cpu_model(),
                         "kind": "reference",
                         "sample": f"the whole batch every step ({B} x dft then {B} x invdft in place, N={N}), "
                                   f"OpenMP over the batch with one aux per thread, "
                                   f"reference built -O3 -fopenmp -mavx2 -mfma"},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_seconds": [round(t, 4) for t in steps],
        "wall_s": round(time.time() - t0, 2),
    }
    print(json.dumps(line))


def bench_float_forms(args, wl, x64, stream, ms_fp64, rank, world, dist):
    """Plain FP32 and split-tensor-core FP32 forms on the FP64 run's shape:
    GB/s (8-byte complex), transforms/s relative to the FP64 drop-in, and the
    worst per-transform relative L2 error against the FP64 results of the same
    inputs (a sample of the batch)."""
    import torch

    from notorious_fft import FORM_SPLIT_TC, load

    Lf = load(single=True)
    Lf.set_stream(stream.cuda_stream)
    Ld = load(single=False)
    N, B = wl["N"], wl["batch"]
    xf = x64.to(torch.complex64)
    yf = torch.empty_like(xf)
    zf = torch.empty_like(xf)
    out = {}
    # FP64 reference results for a sample of the same (rounded) inputs
    ns = min(B, 16)
    xs = xf[:ns].to(torch.complex128)
    ys = torch.empty_like(xs)
    with Ld.mkaux("dft", [N]) as a64:
        a64.batched("dft", xs, ys, ns, N, N)
    torch.cuda.synchronize()
    for name, form in (("fp32_plain", 0), ("split_tc", FORM_SPLIT_TC)):
        aux = Lf.mkaux("dft", [N])
        aux.set_form(form)

        def step():
            aux.batched("dft", xf, yf, B, N, N)
            aux.batched("invdft", yf, zf, B, N, N)

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        if dist:
            tt = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
        aux.batched("dft", xf[:ns], yf[:ns], ns, N, N)
        torch.cuda.synchronize()
        d = (yf[:ns].to(torch.complex128) - ys)
        errs = torch.linalg.vector_norm(d, dim=1) / torch.linalg.vector_norm(ys, dim=1)
        aux.free()
        gbs = 2 * B * 2 * N * 8 * world / (ms * 1e-3) / 1e9
        out[name] = {"value": round(gbs, 1), "unit": "GB/s", "ms_per_step": round(ms, 4),
                     "transforms_per_s": round(2 * B * world / (ms * 1e-3), 1),
                     "speedup_vs_fp64_transforms": round(ms_fp64 / ms, 3),
                     "max_rel_l2_vs_fp64": float(errs.max().item()), "error_sample_transforms": ns,
                     "dtype": "f32 storage" + (", radix-16 as fp16 hi+lo tensor-core products" if form else "")}
    return out


def _uneven_config(count, seed, nmax=1 << 18):
    """Kinds and lengths of the ragged-batch configuration: N log-uniform on
    [16, nmax], 80% powers of two, the rest split between primes and composite
    lengths; 50% c2c / 30% realdft / 20% DCT-2 (seeded)."""
    import numpy as np

    def is_prime(n):
        if n < 2:
            return False
        i = 2
        while i * i <= n:
            if n % i == 0:
                return False
            i += 1
        return True

    rng = np.random.default_rng(seed)
    kinds, Ns = [], []
    lo, hi = math.log2(16), math.log2(nmax)
    for _ in range(count):
        u = rng.random()
        kind = "dft" if u < 0.5 else ("realdft" if u < 0.8 else "dct2")
        e = rng.uniform(lo, hi)
        v = rng.random()
        if v < 0.8:
            n = 1 << int(round(e))
        else:
            n = max(17, int(round(2 ** e)))
            if v < 0.9:
                while not is_prime(n):
                    n += 1
            else:
                if n & (n - 1) == 0:
                    n += 1
                while is_prime(n) or n & (n - 1) == 0:
                    n += 1
        kinds.append(kind)
        Ns.append(n)
    return kinds, Ns


def bench_configs(args, stream):
    """The other configurations of the reference's benchmark set on this GPU:
    time per call (CUDA events, warm, median; L2 flushed before every timed
    call), algorithmic GB/s (one read of the input and one write of the output
    per transform) and the largest relative L2 error of a sample against an
    independent FP64 FFT (torch / scipy)."""
    import numpy as np
    import scipy.fft as sf
    import torch

    from notorious_fft import FORM_SPLIT_TC, load

    Ld, Lf = load(single=False), load(single=True)
    Ld.set_stream(stream.cuda_stream)
    Lf.set_stream(stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    steps = max(3, min(args.steps, 7))
    g = torch.Generator(device="cuda")
    g.manual_seed(20261203)

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = []
        for _ in range(steps):
            flush.fill_(1)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms)

    def uni(*shape, dt=torch.float64):
        return torch.rand(*shape, generator=g, device="cuda", dtype=dt) * 2 - 1

    def cuni(*shape, dt=torch.complex128):
        r = torch.float64 if dt == torch.complex128 else torch.float32
        return torch.complex(uni(*shape, dt=r), uni(*shape, dt=r))

    def rel(a, b):
        a, b = np.asarray(a, dtype=np.complex128), np.asarray(b, dtype=np.complex128)
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    out = {}
    T = host_cores()
    cpu_on = not args.no_cpu

    def cpu(kinds, dims, batch, nbytes, sample, threads=None, lib="libref_d_avx2.so", prec="f64", reps=3, **kw):
        """The reference's CPU path on the same configuration (same run, host cores)."""
        if not cpu_on:
            return None
        th = T if threads is None else threads
        rec = cpu_run(kinds, dims, batch, th, reps, lib=lib, prec=prec, **kw)
        return cpu_entry(rec, nbytes, sample, lib, th)

    def entry(name, ms, nbytes, err, **kw):
        e = {"ms": round(ms, 4), "gb_s": round(nbytes / (ms * 1e-3) / 1e9, 1), "max_rel_l2": err}
        e.update(kw)
        out[name] = e

    # C1: 256 x 4096 FP64 dft + invdft (fits L2: flushed before every call)
    x = cuni(256, 4096)
    y, z = torch.empty_like(x), torch.empty_like(x)
    with Ld.mkaux("dft", [4096]) as a:
        ms = timed(lambda: (a.batched("dft", x, y, 256, 4096, 4096), a.batched("invdft", y, z, 256, 4096, 4096)))
        torch.cuda.synchronize()
        err = rel(y[:4].cpu(), torch.fft.fft(x[:4], dim=1).cpu())
    entry("c1_dft_invdft_4096x256_f64", ms, 2 * 256 * 4096 * 32, err,
          cpu_baseline=cpu(["dft", "invdft"], [4096], 256, 2 * 256 * 4096 * 32,
                           "256 x dft then invdft in place, OpenMP over the batch, one aux per thread"))
    del x, y, z

    # C2: realdft 2^20 x 16
    n = 1 << 20
    x = uni(16, n)
    zc = torch.empty(16, n // 2 + 1, dtype=torch.complex128, device="cuda")
    with Ld.mkaux("realdft", [n]) as a:
        ms = timed(lambda: a.batched("realdft", x, zc, 16, n, n // 2 + 1))
        torch.cuda.synchronize()
        err = rel(zc[:2].cpu(), torch.fft.rfft(x[:2], dim=1).cpu())
    entry("c2_realdft_1048576x16_f64", ms, 16 * (n * 8 + (n // 2 + 1) * 16), err,
          cpu_baseline=cpu(["realdft"], [n], 16, 16 * (n * 8 + (n // 2 + 1) * 16),
                           "16 transforms, OpenMP over the batch, one aux per thread"))
    del x, zc
    # C2: DCT-2 / DST-2 / DCT-4, 8192 x 512
    n, b = 8192, 512
    x = uni(b, n)
    y = torch.empty_like(x)
    for kind, fam, ref in (("dct2", "t2t3", lambda v: sf.dct(v, 2)), ("dst2", "t2t3", lambda v: sf.dst(v, 2)),
                           ("dct4", "t4", lambda v: sf.dct(v, 4))):
        with Ld.mkaux(fam, [n]) as a:
            ms = timed(lambda: a.batched(kind, x, y, b, n, n))
            torch.cuda.synchronize()
            xs, ys = x[:2].cpu().numpy(), y[:2].cpu().numpy()
            err = max(rel(ys[i], ref(xs[i])) for i in range(2))
        entry(f"c2_{kind}_8192x512_f64", ms, b * n * 16, err,
              cpu_baseline=cpu([kind], [n], b, b * n * 16, "512 transforms, OpenMP over the batch, one aux per thread"))
    del x, y
    # C2: 2-D 2048^2 and 3-D 256^3 complex
    for dims in ((2048, 2048), (256, 256, 256)):
        x = cuni(*dims)
        y = torch.empty_like(x)
        with Ld.mkaux("dft", list(dims)) as a:
            ms = timed(lambda: a("dft", x, y))
            torch.cuda.synchronize()
            err = rel(y.cpu(), torch.fft.fftn(x).cpu())
        entry("c2_dft_" + "x".join(map(str, dims)) + "_f64", ms, x.numel() * 32, err,
              cpu_baseline=cpu(["dft"], list(dims), 1, x.numel() * 32,
                               "one N-D call, as the reference runs it (no parallelism in its N-D path)",
                               threads=1, reps=2))
        del x, y
    # C2: Bluestein, N = 1,000,003 x 4
    n = 1000003
    x = cuni(4, n)
    y = torch.empty_like(x)
    with Ld.mkaux("dft", [n]) as a:
        ms = timed(lambda: a.batched("dft", x, y, 4, n, n))
        torch.cuda.synchronize()
        err = rel(y[:1].cpu(), torch.fft.fft(x[:1], dim=1).cpu())
    entry("c2_bluestein_dft_1000003x4_f64", ms, 4 * n * 32, err,
          cpu_baseline=cpu(["dft"], [n], 4, 4 * n * 32,
                           "4 transforms, OpenMP over the batch; scalar double build, the only reference build "
                           "whose Bluestein output is correct", lib="libref_d_scalar.so", reps=2))
    del x, y

    # the batched c2c range of the FP64 roofline target: N = 2^12 .. 2^20, both
    # precisions, 1 GiB per array, dft and invdft alternating
    for L, tag, es in ((Ld, "f64", 16), (Lf, "f32", 8)):
        for logn in range(12, 21):
            n = 1 << logn
            b = (1 << 30) // (n * es)
            x = cuni(b, n, dt=torch.complex128 if es == 16 else torch.complex64)
            y = torch.empty_like(x)
            with L.mkaux("dft", [n]) as a:
                ms = timed(lambda: a.batched("dft", x, y, b, n, n))
                torch.cuda.synchronize()
                err = rel(y[:1].cpu(), torch.fft.fft(x[:1].to(torch.complex128), dim=1).cpu())
            entry(f"sweep_c2c_{tag}_n{n}", ms, b * n * 2 * es, err, batch=b)
            del x, y

    # C3: split tensor-core FP32 form, N = 2^16, 10% of the transforms x 1e4
    n, b = 1 << 16, 1024
    x = cuni(b, n, dt=torch.complex64)
    sel = torch.randperm(b, generator=torch.Generator().manual_seed(3))[: b // 10].cuda()
    x[sel] *= 1e4
    y = torch.empty_like(x)
    x64 = x[:64].to(torch.complex128)
    ref = torch.fft.fft(x64, dim=1)
    c3_cpu = cpu(["dft"], [n], b, b * n * 16,
                 f"{b} transforms, OpenMP over the batch; NOTORIOUS_FFT_SINGLE scalar build", lib="libref_s_scalar.so",
                 prec="f32", reps=2)
    for name, form in (("fp32_plain", 0), ("split_tc", FORM_SPLIT_TC)):
        with Lf.mkaux("dft", [n]) as a:
            a.set_form(form)
            ms = timed(lambda: a.batched("dft", x, y, b, n, n))
            torch.cuda.synchronize()
            d = (y[:64].to(torch.complex128) - ref)
            errs = torch.linalg.vector_norm(d, dim=1) / torch.linalg.vector_norm(ref, dim=1)
        entry(f"c3_{name}_65536x{b}_scaled10pct", ms, b * n * 16, float(errs.max().item()),
              transforms_per_s=round(b / (ms * 1e-3), 1), scaled_in_sample=int((sel < 64).sum().item()),
              cpu_baseline=c3_cpu)
    del x, y, x64, ref

    # C4: ragged batch of 20,000 transforms, one persistent launch (CUDA graph)
    kinds, Ns = _uneven_config(20000, seed=2026)
    listfile = tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False)
    listfile.write("".join(f"{k} {nn}\n" for k, nn in zip(kinds, Ns)))
    listfile.close()
    for L, tag, rs in ((Ld, "f64", 8), (Lf, "f32", 4)):
        t0 = time.perf_counter()
        bt = L.mkbatch(kinds, Ns)
        build_s = time.perf_counter() - t0
        dt = torch.float64 if rs == 8 else torch.float32
        xi = uni(bt.in_size, dt=dt)
        yo = torch.empty(bt.out_size, dtype=dt, device="cuda")
        ms = timed(lambda: bt.execute(xi, yo))
        assert bt.status() == 0
        nbytes = 0
        for k, nn in zip(kinds, Ns):
            ci = 2 * nn if k == "dft" else nn
            co = 2 * nn if k == "dft" else (2 * (nn // 2 + 1) if k == "realdft" else nn)
            nbytes += (ci + co) * rs
        # error sample: the first c2c transform of the packed layout
        i0 = kinds.index("dft")
        off = 0
        for k, nn in zip(kinds[:i0], Ns[:i0]):
            off += 2 * nn if k == "dft" else nn
            off += off & 1
        ooff = 0
        for k, nn in zip(kinds[:i0], Ns[:i0]):
            ooff += 2 * nn if k == "dft" else (2 * (nn // 2 + 1) if k == "realdft" else nn)
            ooff += ooff & 1
        n0 = Ns[i0]
        xin = xi[off: off + 2 * n0].double().view(n0, 2)
        got = yo[ooff: ooff + 2 * n0].double().view(n0, 2)
        refc = torch.fft.fft(torch.complex(xin[:, 0], xin[:, 1]))
        err = rel(torch.complex(got[:, 0], got[:, 1]).cpu(), refc.cpu())
        info = bt.info()
        bt.free()
        c4_cpu = None
        if cpu_on:
            lib = "libref_d_scalar.so" if rs == 8 else "libref_s_scalar.so"
            rec = cpu_run(None, None, None, T, 2, lib=lib, prec=tag, listfile=listfile.name)
            c4_cpu = cpu_entry(rec, rec["gbs"] * rec["seconds"] * 1e9 if rec else 0,
                               "the same 20,000 (kind, N) list: one aux per distinct (kind, N), OpenMP over the "
                               "groups, plan building excluded (seconds_with_plans includes it); the transforms "
                               "the reference has no plan for (realdft / DCT-2 of lengths that are not powers "
                               "of two) are not run and not counted", lib, T,
                               extra=None if rec is None else {
                                   "transforms_per_s": round(rec["transforms_per_s"], 1), "executed": rec["executed"],
                                   "skipped_no_plan": rec["skipped_no_plan"],
                                   "seconds_with_plans": round(rec["seconds_with_plans"], 3)})
        entry(f"c4_ragged_20000_{tag}", ms, nbytes, err, transforms_per_s=round(20000 / (ms * 1e-3), 1),
              build_s=round(build_s, 2), items=info["items"], tiles=info["tiles"], ctas=info["ctas"],
              launches_per_call=1, graph=True, cpu_baseline=c4_cpu)
        del xi, yo

    # C5: one forward + backward step of L = sum w |rfft2(x)|^2 + sum v DCT2(rowmean(x)), x 64 x 512 x 512 FP32
    B5, N1, N2 = 64, 512, 512
    x = torch.randn(B5, N1, N2, generator=g, device="cuda", dtype=torch.float32)
    w = torch.rand(B5, N1, N2 // 2 + 1, generator=g, device="cuda", dtype=torch.float32) + 0.5
    v = torch.rand(B5, N1, generator=g, device="cuda", dtype=torch.float32) + 0.5
    rf, dc = Lf.mkaux("realdft", [N1, N2]), Lf.mkaux("t2t3", [N1])
    zz = torch.empty(B5, N1, N2 // 2 + 1, dtype=torch.complex64, device="cuda")
    gz = torch.empty_like(zz)
    gx = torch.empty_like(x)
    dd, gm = torch.empty(B5, N1, device="cuda"), torch.empty(B5, N1, device="cuda")
    w2 = 2 * w   # the constant weights of dL/dz = 2 w z

    def step5():
        rf.batched("realdft", x, zz, B5, N1 * N2, N1 * (N2 // 2 + 1))
        m = x.mean(dim=2)
        dc.batched("dct2", m, dd, B5, N1, N1)
        # one sweep for the cotangent, one for the loss: sum w |z|^2 = Re <z, 2 w z> / 2
        torch.mul(zz, w2, out=gz)
        loss = 0.5 * torch.vdot(zz.reshape(-1), gz.reshape(-1)).real + (v * dd).sum()
        rf.vjp_batched("realdft", gz, gx, B5, N1 * (N2 // 2 + 1), N1 * N2)
        dc.vjp_batched("dct2", v, gm, B5, N1, N1)
        gx.add_(gm.unsqueeze(2), alpha=1.0 / N2)
        return loss

    ms = timed(step5)
    rf.free()
    dc.free()
    entry("c5_loss_forward_backward_64x512x512_f32", ms, 2 * (x.numel() * 4 + zz.numel() * 8), None,
          note="realdft 2-D + DCT-2 forward, their adjoint kernels backward, torch elementwise glue",
          cpu_baseline={"unavailable": "the reference's multi-dimensional realdft crashes (its N-D real path "
                                       "dereferences a null scratch pointer; src/07_legacy.h:1492-1524) and it has "
                                       "no adjoints"})
    os.unlink(listfile.name)
    return out


def run_ragged(args, wl):
    """Profiling workload: one ragged batch (FP64) of `batch` transforms of the
    uneven configuration, executed through the persistent queue."""
    import torch

    from notorious_fft import load

    L = load(single=False)
    stream = torch.cuda.current_stream()
    L.set_stream(stream.cuda_stream)
    kinds, Ns = _uneven_config(wl["batch"], seed=2026)
    b = L.mkbatch(kinds, Ns)
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    x = torch.rand(b.in_size, generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    y = torch.empty(b.out_size, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        b.execute(x, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for _ in range(args.steps):
        flush.fill_(1)
        e0.record(stream)
        b.execute(x, y)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    assert b.status() == 0
    nbytes = 0
    for k, n in zip(kinds, Ns):
        ci = 2 * n if k == "dft" else n
        co = 2 * n if k == "dft" else (2 * (n // 2 + 1) if k == "realdft" else n)
        nbytes += (ci + co) * 8
    m = statistics.median(ms)
    print(json.dumps({"workload": f"ragged fp64 x{wl['batch']}", "ms": round(m, 4),
                      "gb_s": round(nbytes / (m * 1e-3) / 1e9, 1),
                      "transforms_per_s": round(wl["batch"] / (m * 1e-3), 1), "info": b.info()}))
    b.free()


def run_split_tc(args, wl):
    """Profiling workload: the float library's split tensor-core form (or, with
    --form plain, the plain FP32 form) on a batch of N = 65536 complex
    transforms, dft only; prints the time per call."""
    import torch

    from notorious_fft import FORM_SPLIT_TC, load

    L = load(single=True)
    stream = torch.cuda.current_stream()
    L.set_stream(stream.cuda_stream)
    N, B = wl["N"], wl["batch"]
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    x = torch.randn(B, N, generator=g, device="cuda", dtype=torch.complex64)
    y = torch.empty_like(x)
    with L.mkaux("dft", [N]) as a:
        a.set_form(0 if args.form == "plain" else FORM_SPLIT_TC)
        for _ in range(args.warmup):
            a.batched("dft", x, y, B, N, N)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            a.batched("dft", x, y, B, N, N)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({"workload": f"{args.form} fp32 N={N} x{B} dft", "ms": round(ms, 4),
                      "gb_s": round(B * N * 16 / (ms * 1e-3) / 1e9, 1)}))


def run_bluestein(args, wl):
    """Profiling workload: FP64 Bluestein dft of the prime N = 1,000,003 on a
    batch of 4 (six specialized passes over M = 2^21: chirp premultiply, two
    plain, filter product, plain, window + chirp); prints the time per call."""
    import torch

    from notorious_fft import load

    L = load(single=False)
    stream = torch.cuda.current_stream()
    L.set_stream(stream.cuda_stream)
    N, B = wl["N"], wl["batch"]
    g = torch.Generator(device="cuda")
    g.manual_seed(12)
    x = torch.randn(B, N, generator=g, device="cuda", dtype=torch.complex128)
    y = torch.empty_like(x)
    with L.mkaux("dft", [N]) as a:
        for _ in range(args.warmup):
            a.batched("dft", x, y, B, N, N)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            a.batched("dft", x, y, B, N, N)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({"workload": f"bluestein fp64 N={N} x{B} dft", "ms": round(ms, 4),
                      "gb_s": round(B * N * 32 / (ms * 1e-3) / 1e9, 1)}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c2c")
    ap.add_argument("--batch", type=int, default=0, help="override the workload's batch (profiling runs)")
    ap.add_argument("--form", choices=["split_tc", "plain"], default="split_tc",
                    help="precision form of the split_tc profiling workload")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the float-library forms")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configurations (C1-C5)")
    args = ap.parse_args()
    wl = dict(WORKLOADS[args.workload])
    if args.batch:
        wl["batch"] = args.batch
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args, wl)
    if args.workload == "ragged":
        return run_ragged(args, wl)
    if args.workload == "split_tc":
        return run_split_tc(args, wl)
    if args.workload == "bluestein":
        return run_bluestein(args, wl)

    import numpy as np
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from notorious_fft import load

    L = load(single=False)
    N, B = wl["N"], wl["batch"]
    stream = torch.cuda.current_stream()
    L.set_stream(stream.cuda_stream)
    g = torch.Generator(device="cuda")
    g.manual_seed(1 + rank)
    x = torch.complex(torch.rand(B, N, generator=g, device="cuda", dtype=torch.float64) * 2 - 1,
                      torch.rand(B, N, generator=g, device="cuda", dtype=torch.float64) * 2 - 1)
    y = torch.empty_like(x)
    z = torch.empty_like(x)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda") if wl["flush"] else None
    aux = L.mkaux("dft", [N])

    def step():
        aux.batched("dft", x, y, B, N, N)
        aux.batched("invdft", y, z, B, N, N)

    # clock samples: the sampler runs from before the warm-up steps (all under
    # load) until the end of the timed region
    clocks = Clocks(local)
    for _ in range(args.warmup):
        step()
        if flush is not None:
            flush.fill_(1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    times = []
    launches0 = L.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    total_ms = 0.0
    for _ in range(args.steps):
        if flush is not None:
            flush.fill_(1)
        ev0.record(stream)
        step()
        ev1.record(stream)
        ev1.synchronize()
        t = ev0.elapsed_time(ev1)
        times.append(t)
        total_ms += t
    torch.cuda.synchronize()
    launches = L.launch_count() - launches0
    ck = clocks.stop()
    if dist:
        dist.barrier()
    ms_step = total_ms / args.steps
    if dist:
        tt = torch.tensor([ms_step], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_step = float(tt.item())
    bytes_per_step = 2 * B * 2 * N * 16            # dft + invdft, each reads and writes the batch
    value = bytes_per_step * world / (ms_step * 1e-3) / 1e9
    # correctness spot check of this run (round trip)
    err = float(torch.linalg.vector_norm(z[:4] / N - x[:4]) / torch.linalg.vector_norm(x[:4]))

    peak, peak_kind = peaks()
    # dominant kernel: the batched FFT itself (all passes of one transform over
    # the batch), timed with CUDA events on the launching stream
    per_transform_ms = ms_step / 2
    achieved = (B * 2 * N * 16) / (per_transform_ms * 1e-3) / 1e9
    tpt = MEASURED_TRAFFIC_PER_TRANSFORM.get((args.workload, N))
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": (round(tpt * B) if tpt else None),
            "traffic_unit": "bytes per batched transform (ncu, scaled from 256 transforms)",
            "algorithmic_bytes": B * 2 * N * 16, "peak_kind": peak_kind,
            "kernel": "lean_pass_kernel<double> pass 1 + pass 2 (one batched c2c transform of N=65536)"}

    # ---- the float library on the same shape: plain FP32 and split tensor-core form ----
    forms = {}
    if not args.no_forms:
        forms = bench_float_forms(args, wl, x, stream, ms_step, rank, world, dist)

    configs = None
    if not args.no_configs and rank == 0 and world == 1:
        configs = bench_configs(args, stream)

    e2e = None
    e2e_pageable = None
    if not args.no_e2e and rank == 0 and world == 1:
        xh = x.cpu().pin_memory()
        yh = torch.empty_like(xh).pin_memory()
        zh = torch.empty_like(xh).pin_memory()
        aux.batched("dft", xh, yh, B, N, N)
        torch.cuda.synchronize()
        ks = min(3, args.steps)
        t0 = time.perf_counter()
        for _ in range(ks):
            aux.batched("dft", xh, yh, B, N, N)
            aux.batched("invdft", yh, zh, B, N, N)
        dt = (time.perf_counter() - t0) / ks
        e2e = {"value": round(bytes_per_step / dt / 1e9, 3), "unit": "GB/s", "h2d_bytes_per_step": 2 * B * N * 16,
               "d2h_bytes_per_step": 2 * B * N * 16, "steps": ks, "timing": "host wall clock around synchronous C-ABI calls",
               "host_memory": "pinned (page-locked)"}
        del xh, yh, zh
        # the same calls on pageable host buffers (what a reference caller's
        # malloc gives): staged through the library's pinned buffers
        xp = x.cpu()
        yp = torch.empty_like(xp)
        zp = torch.empty_like(xp)
        aux.batched("dft", xp, yp, B, N, N)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ks):
            aux.batched("dft", xp, yp, B, N, N)
            aux.batched("invdft", yp, zp, B, N, N)
        dt = (time.perf_counter() - t0) / ks
        e2e_pageable = {"value": round(bytes_per_step / dt / 1e9, 3), "unit": "GB/s",
                        "h2d_bytes_per_step": 2 * B * N * 16, "d2h_bytes_per_step": 2 * B * N * 16, "steps": ks,
                        "timing": "host wall clock around synchronous C-ABI calls", "host_memory": "pageable"}
        del xp, yp, zp

    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        # the reference's CPU path on the same workload: the whole batch,
        # dft then invdft, best of 2 (about 1.5 s of 16-core work)
        threads = host_cores()
        rec = cpu_run(["dft", "invdft"], [N], B, threads, 2)
        if rec is not None:
            cpu = {"value": round(bytes_per_step / rec["seconds"] / 1e9, 3), "unit": "GB/s", "cores": threads,
                   "cpu": cpu_model(), "kind": "reference", "ms_per_step": round(rec["seconds"] * 1e3, 2),
                   "sample": f"the whole batch ({B} x dft then {B} x invdft in place, N={N}), best of 2, "
                             f"OpenMP over the batch with one aux per thread, -O3 -fopenmp -mavx2 -mfma"}
    aux.free()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (uniform[-1,1), torch seeded generator)",
            "config": {"workload": f"c2c fp64 N={N} x{B} dft+invdft per GPU", "N": N, "batch": B, "l2": wl["l2"],
                       "parallelism": f"batch-sharded x{world}"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "e2e_pageable": e2e_pageable, "gpu_launches": launches,
            "clocks": ck, "round_trip_rel_err": err,
        }
        line.update(forms)
        if configs is not None:
            line["configs"] = configs
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

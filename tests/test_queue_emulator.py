"""Ragged batches through the persistent queue, on the CPU emulator.

The emulator runs the queue's items in claim order with the kernels' own tile
functions (every global / shared access bounds-checked, fresh device memory
NaN-filled).  These tests check the queue builder -- buckets, offset tables,
dependency groups, item order, the size-1 branch, Bluestein with real-input
operators -- against the oracle, plus the error paths and the bounded-wait
status.  The GPU tests (test_gpu_queue.py) run the same batches on the device.
"""
import os

import numpy as np
import pytest
import scipy.fft as sf

from oracle import rel_l2

CPLX_IN = {"dft", "invdft", "invrealdft"}


def _pow2(n):
    return n > 0 and (n & (n - 1)) == 0


def in_reals(kind, n):
    if kind == "invrealdft":
        return 2 * (n // 2 + 1)
    return 2 * n if kind in CPLX_IN else n


def out_reals(kind, n):
    if kind == "realdft":
        return 2 * (n // 2 + 1)
    return 2 * n if kind in ("dft", "invdft") else n


def packed_offsets(kinds, Ns, size_fn):
    off, pos = [], 0
    for k, n in zip(kinds, Ns):
        off.append(pos)
        pos += size_fn(k, n)
        pos += pos & 1
    return off


def expected(oracle, kind, x, n):
    """Oracle output of one transform (x: reals as laid out in the buffer)."""
    if kind in ("dft", "invdft"):
        xc = x[0::2] + 1j * x[1::2]
        return oracle.transform(kind, xc)
    if kind == "realdft":
        if _pow2(n):
            return oracle.transform("realdft", x)
        return oracle.transform("dft", x.astype(np.complex128))[: n // 2 + 1]
    if kind == "invrealdft":
        return oracle.invrealdft(x[0::2] + 1j * x[1::2], n)
    if n == 1:
        return np.array([{"dct2": 2.0, "dst2": 2.0, "dct4": 2 ** 0.5, "dst4": 2 ** 0.5}.get(kind, 1.0) * x[0]])
    if not _pow2(n):
        assert kind == "dct2"
        return sf.dct(x.astype(np.longdouble).astype(np.float64), type=2)
    return oracle.transform(kind, x)


def got_of(kind, y):
    return y[0::2] + 1j * y[1::2] if kind in ("dft", "invdft", "realdft") else y


def run_and_check(lib, oracle, kinds, Ns, in_off=None, out_off=None, seed=0, tol=None, inplace=False):
    b = lib.mkbatch(kinds, Ns, in_off, out_off)
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, b.in_size).astype(lib.rdt)
    y = x if inplace else np.full(b.out_size, np.nan, lib.rdt)
    x0 = x.copy()
    b.execute(x, y)
    assert b.status() == 0
    io = in_off if in_off is not None else packed_offsets(kinds, Ns, in_reals)
    oo = out_off if out_off is not None else packed_offsets(kinds, Ns, out_reals)
    worst = 0.0
    for i, (k, n) in enumerate(zip(kinds, Ns)):
        xi = x0[io[i]: io[i] + in_reals(k, n)].astype(np.float64)
        ref = expected(oracle, k, xi, n)
        got = got_of(k, y[oo[i]: oo[i] + out_reals(k, n)].astype(np.float64))
        e = rel_l2(got, ref)
        worst = max(worst, e)
        lim = tol if tol is not None else (3e-15 if lib.single is False else 3e-6) * max(1, np.log2(max(n, 2)))
        assert e <= lim, (i, k, n, e)
    b.free()
    return worst


def test_mixed_small(emu_d, oracle_d):
    kinds = ["dft", "realdft", "dct2", "dft", "invdft", "dft", "realdft", "dct2", "dft", "dst2", "dct3", "dst4",
             "invrealdft", "dct4", "dst3"]
    Ns = [64, 128, 256, 16, 64, 7, 6, 9, 1, 32, 64, 128, 64, 16, 256]
    run_and_check(emu_d, oracle_d, kinds, Ns)


def test_multi_pass_and_bluestein(emu_d, oracle_d):
    # 2^13 c2c and 2^14 realdft / DCT-2 need two 4096-point passes (+ the unpack
    # epilogue for the real ones); 5000 / 3001 go through multi-pass Bluestein
    kinds = ["dft", "dft", "realdft", "dct2", "dft", "invdft", "realdft", "dct2", "dft"]
    Ns = [8192, 8192, 16384, 16384, 5000, 3001, 2500, 2049, 4096]
    run_and_check(emu_d, oracle_d, kinds, Ns, seed=1)


def test_offsets_tables_and_groups(emu_d, oracle_d):
    # many transforms per bucket (offset tables), scattered offsets with gaps,
    # and small dependency groups (one transform per group)
    os.environ["NOTORIOUS_FFT_QUEUE_GROUP_KB"] = "1"
    try:
        rng = np.random.default_rng(5)
        kinds = ["dft"] * 5 + ["realdft"] * 4 + ["dct2"] * 3 + ["dft"] * 3
        Ns = [8192] * 5 + [128] * 4 + [512] * 3 + [30] * 3
        order = rng.permutation(len(kinds))
        kinds = [kinds[i] for i in order]
        Ns = [Ns[i] for i in order]
        io, oo, pi, po = [], [], 6, 10
        for k, n in zip(kinds, Ns):
            io.append(pi)
            oo.append(po)
            pi += in_reals(k, n) + 2 * int(rng.integers(0, 5))
            po += out_reals(k, n) + 2 * int(rng.integers(0, 5))
        run_and_check(emu_d, oracle_d, kinds, Ns, io, oo, seed=2)
    finally:
        del os.environ["NOTORIOUS_FFT_QUEUE_GROUP_KB"]


def test_in_place(emu_d, oracle_d):
    kinds = ["dft", "dct2", "dft", "dst4"]
    Ns = [8192, 64, 100, 32]
    run_and_check(emu_d, oracle_d, kinds, Ns, inplace=True)


def test_float_build(emu_f, oracle_d):
    kinds = ["dft", "realdft", "dct2", "dft", "realdft", "dct2"]
    Ns = [16384, 2048, 1024, 1000, 999, 77]
    run_and_check(emu_f, oracle_d, kinds, Ns, seed=3)


def test_errors(emu_d):
    from notorious_fft import NotoriousFFTError
    with pytest.raises(NotoriousFFTError):
        emu_d.mkbatch(["dct3"], [100])          # r2r other than DCT-2 needs a power of two
    with pytest.raises(NotoriousFFTError):
        emu_d.mkbatch(["dft"], [64], [1], [0])  # complex data at an odd offset
    with pytest.raises(NotoriousFFTError):
        emu_d.mkbatch(["dft"], [0])
    # device buffers: in place needs every transform to map onto itself
    import ctypes
    b = emu_d.mkbatch(["realdft"], [64])
    emu_d.lib.nfft_emu_malloc.restype = ctypes.c_void_p
    emu_d.lib.nfft_emu_malloc.argtypes = [ctypes.c_size_t]
    emu_d.lib.nfft_emu_free.argtypes = [ctypes.c_void_p]
    d = emu_d.lib.nfft_emu_malloc(8 * max(b.in_size, b.out_size))
    try:
        with pytest.raises(NotoriousFFTError):
            b.execute(d, d)
        with pytest.raises(NotoriousFFTError):
            b.execute(d, d + 8)                  # overlapping, not identical
    finally:
        emu_d.lib.nfft_emu_free(d)


def test_empty_batch(emu_d):
    b = emu_d.mkbatch([], [])
    assert b.in_size == 0 and b.out_size == 0
    b.execute(np.zeros(1), np.zeros(1))
    assert b.status() == 0


def test_withheld_dependency_times_out(emu_d, oracle_d):
    """A dependency that is never published ends the launch with TIMEOUT and
    the next execution of the same batch is correct."""
    kinds, Ns = ["dft", "dft"], [8192, 64]
    b = emu_d.mkbatch(kinds, Ns)
    x = np.random.default_rng(0).uniform(-1, 1, b.in_size)
    y = np.zeros(b.out_size)
    from notorious_fft import NotoriousFFTError
    b.withhold(1000)
    with pytest.raises(NotoriousFFTError, match="error 5"):
        b.execute(x, y)
    b.execute(x, y)
    assert b.status() == 0
    xc = x[0::2] + 1j * x[1::2]
    assert rel_l2(y[: 2 * 8192][0::2] + 1j * y[: 2 * 8192][1::2], oracle_d.transform("dft", xc[:8192])) < 1e-14


def test_queue_structure(emu_d):
    """Items of a multi-pass bucket: one group per transform at a 1 KB group
    target, two dependent stages each; every item runs in the emulated launch."""
    os.environ["NOTORIOUS_FFT_QUEUE_GROUP_KB"] = "1"
    os.environ["NOTORIOUS_FFT_QUEUE_TILES_MULTI"] = "1"
    try:
        b = emu_d.mkbatch(["dft"] * 3, [8192] * 3)
    finally:
        del os.environ["NOTORIOUS_FFT_QUEUE_GROUP_KB"]
        del os.environ["NOTORIOUS_FFT_QUEUE_TILES_MULTI"]
    info = b.info()
    # 8192 points = 2 tiles of 4096 per pass, two passes, one tile per item
    assert info["tiles"] == 3 * 2 * 2 and info["items"] == 12
    assert info["scratch_bytes"] >= 3 * 8192 * 16


def test_unusable_cached_split_falls_back(tmp_path):
    """A tune-cache entry for this device whose split the planner rejects is
    ignored: the batch is planned with the default schedule."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cache = tmp_path / "tune.json"
    cache.write_text('{"format": "notorious_fft tune cache 1", "entries": [\n'
                     '{"device": "emulated sm_100 sm_100 driver 0", "key": "f64:dft:8192", "split": [1, 12], "us": 1.0}'
                     '\n]}\n')
    child = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from notorious_fft import Library
L = Library(sys.argv[2])
print(L.tune_lookup("dft", 8192))
b = L.mkbatch(["dft"], [8192])
x = np.random.default_rng(0).uniform(-1, 1, b.in_size); y = np.zeros(b.out_size)
b.execute(x, y)
xc = x[0::2] + 1j * x[1::2]
print(float(np.abs((y[0::2] + 1j * y[1::2]) - np.fft.fft(xc)).max() / np.abs(np.fft.fft(xc)).max()))
"""
    env = dict(os.environ, NOTORIOUS_FFT_TUNE_CACHE=str(cache))
    r = subprocess.run([sys.executable, "-c", child, os.path.join(root, "notorious-fft_b200"),
                        os.path.join(root, "tests", "emu", "_build", "libnfft_emu_d.so")],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    assert json.loads(lines[0]) == [1, 12]          # the entry was read
    assert float(lines[1]) < 1e-14                   # and the batch ran on the default schedule

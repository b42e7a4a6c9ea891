"""Host logic on the CPU: the library's planner and C ABI compiled against an
emulated CUDA runtime (tests/emu), running the kernels' own per-thread phase
functions with every global and shared-memory access bounds-checked.

Checks every transform family at single-pass, multi-pass and Bluestein
sizes, N-D shapes (including the reference's length-1-axis rules), batched
calls with padded distances, in-place calls, the error conventions of the C
API, and the adjoints against the transposed transforms and finite
differences.  Tolerances are the north-star ones (1e-13 log2 N for double,
1e-6 log2 N for float).
"""
import ctypes
import json
import math
import os
import subprocess
import sys

import numpy as np
import pytest
import scipy.fft as sf

from oracle import rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
R2R = ["dct2", "dst2", "dct3", "dst3", "dct4", "dst4"]


def tol(n, single=False):
    return (1e-6 if single else 1e-13) * max(1.0, math.log2(max(n, 2)))


def cx(rng, *shape):
    return rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)


@pytest.mark.parametrize("n", [1, 2, 4, 8, 16, 32, 64, 128, 512, 2048, 4096, 8192, 16384, 1 << 16])
def test_emu_complex_pow2(emu_d, oracle_d, n):
    x = cx(np.random.default_rng(n), n)
    with emu_d.mkaux("dft", [n]) as a:
        for k in ("dft", "invdft"):
            assert rel_l2(a(k, x), oracle_d.transform(k, x)) <= tol(n), k


@pytest.mark.parametrize("n", [3, 5, 6, 7, 10, 12, 15, 20, 100, 1000, 4097])
def test_emu_bluestein(emu_d, oracle_d, n):
    x = cx(np.random.default_rng(n), n)
    with emu_d.mkaux("dft", [n]) as a:
        for k in ("dft", "invdft"):
            assert rel_l2(a(k, x), oracle_d.transform(k, x)) <= tol(n), k


@pytest.mark.parametrize("n", [1, 2, 4, 8, 16, 64, 1024, 8192, 16384, 1 << 15, 1 << 16])
def test_emu_real_families(emu_d, oracle_d, n):
    rng = np.random.default_rng(n + 1)
    x = rng.uniform(-1, 1, n)
    with emu_d.mkaux("realdft", [n]) as a:
        z = oracle_d.transform("realdft", x)
        assert rel_l2(a("realdft", x), z) <= tol(n)
        z2 = z + 0.25j * rng.uniform(-1, 1, z.shape)     # invrealdft ignores Im z_0, Im z_{N/2}
        assert rel_l2(a("invrealdft", z2), oracle_d.invrealdft(z2, n)) <= tol(n)
    with emu_d.mkaux("t2t3", [n]) as a:
        for k in R2R[:4]:
            assert rel_l2(a(k, x), oracle_d.transform(k, x)) <= tol(n), k
    with emu_d.mkaux("t4", [n]) as a:
        for k in R2R[4:]:
            assert rel_l2(a(k, x), oracle_d.transform(k, x)) <= tol(n), k


ND_SHAPES = [(4, 4), (8, 16), (32, 32), (4, 4, 4), (4, 8, 8), (1, 8), (8, 1), (1, 1), (2, 1, 4), (16, 1, 1),
             (64, 128), (2048, 4), (2, 4096)]


@pytest.mark.parametrize("dims", ND_SHAPES + [(3, 5), (6, 10, 12), (4, 3000)])
def test_emu_nd_complex(emu_d, oracle_d, dims):
    x = cx(np.random.default_rng(len(dims)), *dims)
    with emu_d.mkaux("dft", dims) as a:
        for k in ("dft", "invdft"):
            assert rel_l2(a(k, x), oracle_d.nd(k, x)) <= tol(int(np.prod(dims))), k


@pytest.mark.parametrize("dims", ND_SHAPES)
def test_emu_nd_real(emu_d, oracle_d, dims):
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, dims)
    n = int(np.prod(dims))
    with emu_d.mkaux("t2t3", dims) as a:
        for k in R2R[:4]:
            assert rel_l2(a(k, x), oracle_d.nd(k, x)) <= tol(n), k
    with emu_d.mkaux("t4", dims) as a:
        for k in R2R[4:]:
            assert rel_l2(a(k, x), oracle_d.nd(k, x)) <= tol(n), k
    with emu_d.mkaux("realdft", dims) as a:
        z = oracle_d.nd("realdft", x)
        assert rel_l2(a("realdft", x), z) <= tol(n)
        assert rel_l2(a("invrealdft", z), oracle_d.nd("invrealdft", z, dims)) <= tol(n)


@pytest.mark.parametrize("n,B", [(64, 5), (4096, 3), (1 << 15, 2), (100, 4), (16384, 3)])
def test_emu_batched_padded(emu_d, oracle_d, n, B):
    rng = np.random.default_rng(n)
    xb = cx(rng, B, n + 7)
    yb = np.zeros((B, n + 3), complex)
    with emu_d.mkaux("dft", [n]) as a:
        a.batched("dft", xb, yb, B, n + 7, n + 3)
    assert rel_l2(yb[:, :n], oracle_d.transform("dft", xb[:, :n])) <= tol(n)
    if n & (n - 1) == 0:
        xr = rng.uniform(-1, 1, (B, n + 5))
        yr = np.zeros((B, n + 2))
        with emu_d.mkaux("t2t3", [n]) as a:
            a.batched("dct3", xr, yr, B, n + 5, n + 2)
        assert rel_l2(yr[:, :n], oracle_d.transform("dct3", xr[:, :n])) <= tol(n)
        zr = np.zeros((B, n // 2 + 3), complex)
        with emu_d.mkaux("realdft", [n]) as a:
            a.batched("realdft", xr, zr, B, n + 5, n // 2 + 3)
        assert rel_l2(zr[:, :n // 2 + 1], oracle_d.transform("realdft", xr[:, :n])) <= tol(n)


def test_emu_inplace(emu_d, oracle_d):
    rng = np.random.default_rng(3)
    for n in (1024, 1 << 15, 1000):
        x = cx(rng, n)
        y = x.copy()
        with emu_d.mkaux("dft", [n]) as a:
            emu_d._call(emu_d.lib.notorious_fft_dft, y, y, a)
        assert rel_l2(y, oracle_d.transform("dft", x)) <= tol(n)


def test_emu_float(emu_f, oracle_d):
    rng = np.random.default_rng(11)
    for n in (16, 4096, 1 << 15, 1000):
        x = cx(rng, n).astype(np.complex64)
        with emu_f.mkaux("dft", [n]) as a:
            assert rel_l2(a("dft", x), oracle_d.transform("dft", x.astype(np.complex128))) <= tol(n, True)
        if n & (n - 1) == 0:
            xr = rng.uniform(-1, 1, n).astype(np.float32)
            with emu_f.mkaux("t2t3", [n]) as a:
                assert rel_l2(a("dct2", xr), oracle_d.transform("dct2", xr.astype(np.float64))) <= tol(n, True)


# ---------------------------------------------------------------------------
# C API conventions
# ---------------------------------------------------------------------------
def test_emu_null_conventions(emu_d):
    for fam in ("realdft", "t2t3", "t4"):
        assert not emu_d.mkaux_1d_raw(fam, 12)
        assert not emu_d.mkaux_1d_raw(fam, 0)
        assert emu_d.last_error()[0] == 1
    assert not emu_d.mkaux_1d_raw("dft", 0)
    assert not emu_d.mkaux_1d_raw("dft", -3)
    p = emu_d.mkaux_1d_raw("dft", 12)
    assert p
    emu_d.free_raw(p)
    emu_d.free_raw(None)
    assert not emu_d.mkaux_raw("t2t3", [4, 6])      # any non-power-of-two dimension


def test_emu_wrong_family_and_null_aux(emu_d):
    x = np.zeros(16)
    y = np.zeros(16)
    with emu_d.mkaux("dft", [16]) as a:
        with pytest.raises(Exception):
            emu_d._call(emu_d.lib.notorious_fft_dct2, x, y, a)
    emu_d.lib.notorious_fft_dct2(x.ctypes.data, y.ctypes.data, None)   # NULL aux: silent no-op + error code
    assert emu_d.last_error()[0] == 1


# ---------------------------------------------------------------------------
# adjoints
# ---------------------------------------------------------------------------
def _real_view(a):
    return np.concatenate([a.real.ravel(), a.imag.ravel()]) if np.iscomplexobj(a) else a.ravel()


@pytest.mark.parametrize("kind", ["dft", "invdft", "realdft", "invrealdft"] + R2R)
@pytest.mark.parametrize("dims", [(16,), (1000,), (8, 4), (1 << 15,)])
def test_emu_vjp_inner_product(emu_d, kind, dims):
    """<g, A x> == <A^T g, x> for random x, g (real inner product on pairs)."""
    fam = {"dft": "dft", "invdft": "dft", "realdft": "realdft", "invrealdft": "realdft"}.get(kind, "t4" if kind in ("dct4", "dst4") else "t2t3")
    if fam != "dft" and any(d & (d - 1) for d in dims):
        pytest.skip("power-of-two only")
    rng = np.random.default_rng(1)
    with emu_d.mkaux(fam, dims) as a:
        ins, outs = a.in_shape(kind), a.out_shape(kind)
        cin = kind in ("dft", "invdft", "invrealdft")
        cout = kind in ("dft", "invdft", "realdft")
        x = cx(rng, *ins) if cin else rng.uniform(-1, 1, ins)
        if kind == "invrealdft":
            x = np.fft.rfftn(rng.uniform(-1, 1, dims))     # Hermitian-consistent input (edge bins real)
        g = cx(rng, *outs) if cout else rng.uniform(-1, 1, outs)
        y = a(kind, x)
        gx = a.vjp(kind, g)
    lhs = np.dot(_real_view(g), _real_view(y))
    rhs = np.dot(_real_view(gx), _real_view(x))
    assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs)) * math.log2(max(np.prod(dims), 2))


@pytest.mark.parametrize("kind", ["dct2", "dst3", "realdft", "dft"])
def test_emu_vjp_finite_differences(emu_d, kind):
    fam = {"dft": "dft", "realdft": "realdft"}.get(kind, "t2t3")
    n = 64
    rng = np.random.default_rng(5)
    with emu_d.mkaux(fam, [n]) as a:
        x = cx(rng, n) if kind == "dft" else rng.uniform(-1, 1, n)
        outs = a.out_shape(kind)
        g = cx(rng, *outs) if kind in ("dft", "realdft") else rng.uniform(-1, 1, outs)
        gx = a.vjp(kind, g)

        def L(v):
            return np.dot(_real_view(g), _real_view(a(kind, v)))

        h = 1e-6
        for idx in rng.choice(n, 8, replace=False):
            e = np.zeros(n)
            e[idx] = 1
            if kind == "dft":
                for part, unit in ((np.real, 1.0), (np.imag, 1j)):
                    fd = (L(x + h * unit * e) - L(x - h * unit * e)) / (2 * h)
                    assert abs(fd - part(gx[idx])) < 1e-6 * max(1, abs(fd))
            else:
                fd = (L(x + h * e) - L(x - h * e)) / (2 * h)
                assert abs(fd - gx[idx]) < 1e-6 * max(1, abs(fd))


def test_emu_vjp_matches_reference_transform_on_cotangent(emu_d, oracle_d):
    """The adjoint of DCT-2 is DCT-3 of the cotangent with entry 0 doubled
    (and the others as defined), evaluated by the oracle's transforms."""
    n = 256
    g = np.random.default_rng(9).uniform(-1, 1, n)
    with emu_d.mkaux("t2t3", [n]) as a:
        gx = a.vjp("dct2", g)
    gg = g.copy()
    gg[0] *= 2
    assert rel_l2(gx, oracle_d.transform("dct3", gg)) <= tol(n)
    with emu_d.mkaux("realdft", [n]) as a:
        gz = np.random.default_rng(10).uniform(-1, 1, n // 2 + 1) + 0j
        gx = a.vjp("realdft", gz)
    w = gz.copy()
    w[1:-1] *= 0.5
    assert rel_l2(gx, oracle_d.invrealdft(w, n)) <= tol(n)


def test_emu_pipelined_host_batches(emu_d, oracle_d):
    """Batched calls with both buffers in (emulated) pinned host memory go
    through the chunked copy-in / transform / copy-out pipeline."""
    rng = np.random.default_rng(21)
    n, B = 1 << 15, 9                      # > one 64 MiB chunk is not needed: the loop runs per chunk
    x = cx(rng, B, n)
    y = np.zeros_like(x)
    with emu_d.mkaux("dft", [n]) as a:
        a.batched("dft", x, y, B, n, n)
    assert rel_l2(y, oracle_d.transform("dft", x)) <= tol(n)
    xr = rng.uniform(-1, 1, (6, 4096))
    zr = np.zeros((6, 2049), complex)
    with emu_d.mkaux("realdft", [4096]) as a:
        a.batched("realdft", xr, zr, 6, 4096, 2049)
    assert rel_l2(zr, oracle_d.transform("realdft", xr)) <= tol(4096)


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("n", [64, 1024, 8192])
def test_emu_real_rows_odd_batch_stride(emu_d, emu_f, oracle_d, n, single):
    """Batched single-pass real transforms whose input stride is odd: every other
    transform starts off the vector boundary (the packed realdft row loads fall
    back to scalar loads there); realdft, DCT-2 / DST-2, DCT-4 / DST-4."""
    lib = emu_f if single else emu_d
    B, idist = 3, n + 1
    rng = np.random.default_rng(n + 7)
    x = rng.uniform(-1, 1, B * idist).astype(lib.rdt)
    with lib.mkaux("realdft", [n]) as a:
        z = np.zeros(B * (n // 2 + 1), lib.cdt)
        a.batched("realdft", x, z, B, idist, n // 2 + 1)
        for b in range(B):
            ref = oracle_d.transform("realdft", x[b * idist: b * idist + n].astype(np.float64))
            assert rel_l2(z[b * (n // 2 + 1):(b + 1) * (n // 2 + 1)], ref) <= tol(n, single), b
    for fam, kinds in (("t2t3", ("dct2", "dst2")), ("t4", ("dct4", "dst4"))):
        with lib.mkaux(fam, [n]) as a:
            for k in kinds:
                y = np.zeros(B * n, lib.rdt)
                a.batched(k, x, y, B, idist, n)
                for b in range(B):
                    ref = oracle_d.transform(k, x[b * idist: b * idist + n].astype(np.float64))
                    assert rel_l2(y[b * n:(b + 1) * n], ref) <= tol(n, single), (k, b)


def test_emu_pass_cap_override_keeps_four_passes(tmp_path):
    """NOTORIOUS_FFT_MAX_PASS_LOG=4 on a 2^17 axis would ask for five passes;
    the schedule holds four, so the cap is raised to ceil(17 / 4) and the
    transform stays exact (child process: the switch is read once)."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    child = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from notorious_fft import Library
L = Library(sys.argv[2])
n = 1 << 17
rng = np.random.default_rng(3)
x = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
with L.mkaux("dft", [n]) as a:
    y = a("dft", x)
ref = np.fft.fft(x)
print(float(np.linalg.norm(y - ref) / np.linalg.norm(ref)))
"""
    env = dict(os.environ, NOTORIOUS_FFT_MAX_PASS_LOG="4")
    r = subprocess.run([sys.executable, "-c", child, os.path.join(root, "notorious-fft_b200"),
                        os.path.join(root, "tests", "emu", "_build", "libnfft_emu_d.so")],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert float(r.stdout.strip().splitlines()[-1]) < 1e-13 * 17


@pytest.mark.parametrize("n,batch,pad,kinds", [(1 << 16, 3, 0, [1, 0, 1]), (1 << 16, 2, 2, [1, 0, 1]),
                                               (1 << 16, 1, 0, [1, 0, 1]), (1 << 17, 2, 0, [0, 0, 1])])
def test_emu_split_tc_tcgen05_model(emu_f, oracle_d, n, batch, pad, kinds, monkeypatch):
    """The tcgen05 radix-256 pass through its CPU model (tensor copy with the
    64-byte swizzle, operands read through the descriptor strides: stage 1
    K-major, stage 2 M-major; tensor stores): the row-out first pass and the
    column-out last pass of 2^16 (batches of 3, 2 with a batch stride of
    n + 2 points, and 1), the column-out radix-256 pass of 2^17 (512 x 256);
    one transform scaled by 1e4 and one by 1e-4 (per-line power-of-two
    scaling), forward and inverse, every transform within the split form's
    bar of the FP64 oracle and the model launched for the expected output
    kinds (row, column split at Ns, column)."""
    from notorious_fft import FORM_SPLIT_TC
    monkeypatch.setenv("NOTORIOUS_FFT_TC_UMMA", "1")
    count = emu_f.lib.nfft_emu_umma_kind_launches
    count.restype = ctypes.c_longlong
    count.argtypes = [ctypes.c_int]
    rng = np.random.default_rng(n + batch + pad)
    x = rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))
    x[0] *= 1e4
    x[-1] *= 1e-4
    x = x.astype(np.complex64)
    dist = n + pad
    xb = np.zeros(batch * dist, np.complex64)
    for b in range(batch):
        xb[b * dist:b * dist + n] = x[b]
    bar = max(2e-6, 1e-6 * ((n.bit_length() - 1 + 7) // 8))
    with emu_f.mkaux("dft", [n]) as a:
        a.set_form(FORM_SPLIT_TC)
        for kind in ("dft", "invdft"):
            before = [count(k) for k in range(3)]
            yb = np.zeros(batch * dist, np.complex64)
            a.batched(kind, xb, yb, batch, dist, dist)
            assert [count(k) - before[k] for k in range(3)] == kinds
            ref = oracle_d.transform(kind, x.astype(np.complex128))
            errs = [rel_l2(yb[b * dist:b * dist + n], ref[b]) for b in range(batch)]
            assert max(errs) <= bar, (kind, errs)


UMMA_SPLIT_CHILD = r"""
import ctypes, json, sys, numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[2])
from notorious_fft import Library, FORM_SPLIT_TC
from oracle import Oracle, rel_l2
L = Library(sys.argv[3])
kinds = L.lib.nfft_emu_umma_kind_launches
kinds.restype = ctypes.c_longlong
kinds.argtypes = [ctypes.c_int]
n, B = 1 << 15, 2
rng = np.random.default_rng(15)
x = (rng.standard_normal((B, n)) + 1j * rng.standard_normal((B, n))).astype(np.complex64)
x[1] *= 300.0
out = {}
with L.mkaux("dft", [n]) as a:
    a.set_form(FORM_SPLIT_TC)
    out["split"] = a.schedule()[0]
    for kind in ("dft", "invdft"):
        k0 = [kinds(k) for k in range(3)]
        y = np.zeros_like(x)
        a.batched(kind, x, y, B, n, n)
        ref = Oracle().transform(kind, x.astype(np.complex128))
        out[kind] = {"kinds": [kinds(k) - k0[k] for k in range(3)],
                     "err": max(rel_l2(y[b], ref[b]) for b in range(B))}
print(json.dumps(out))
"""


def test_emu_split_tc_tcgen05_model_column_split(tmp_path):
    """The column-out pass with the line index split at Ns (a radix-256 pass
    in the middle of a transform: 2^15 as 8 x 256 x 16 through a tune-cache
    split; Ns = 8 < 128 lines) through the tcgen05 model, forward and inverse,
    one transform scaled by 300 (lines above the unscaled range)."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "emu")], check=True)
    cache = tmp_path / "tune.json"
    entry = {"device": "emulated sm_100 sm_100 driver 0", "key": "f32:plan:dft:32768", "split": [3, 8, 4],
             "logt": 0, "us": 1.0}
    cache.write_text('{"format": "notorious_fft tune cache 1", "entries": [\n' + json.dumps(entry) + "\n]}\n")
    env = dict(os.environ, NOTORIOUS_FFT_TUNE_CACHE=str(cache), NOTORIOUS_FFT_TC_UMMA="1")
    r = subprocess.run([sys.executable, "-c", UMMA_SPLIT_CHILD, os.path.join(ROOT, "notorious-fft_b200"),
                        os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "emu", "_build", "libnfft_emu_f.so")],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["split"] == [3, 8, 4]
    for kind in ("dft", "invdft"):
        assert res[kind]["kinds"] == [0, 1, 0], res
        assert res[kind]["err"] <= 3e-6, res


@pytest.mark.parametrize("n,batch", [(256, 5), (1 << 16, 3), (4096, 3)])
@pytest.mark.parametrize("tc_lean", ["1", "0"])
def test_emu_split_tc_form(emu_f, oracle_d, n, batch, tc_lean, monkeypatch):
    """The split tensor-core form on the emulator (host model of the FP16
    mma.sync fragments): radix-256 passes in the specialized kernel
    (NOTORIOUS_FFT_TC_LEAN=1, 256 and 2^16) or all passes in the generic
    tensor-core pass (=0; 4096 always), forward and inverse, one transform
    scaled by 1e4 and one by 1e-4 -- every transform within 2e-6 of the
    FP64 oracle."""
    from notorious_fft import FORM_SPLIT_TC
    monkeypatch.setenv("NOTORIOUS_FFT_TC_LEAN", tc_lean)
    monkeypatch.setenv("NOTORIOUS_FFT_TC_UMMA", "0")
    rng = np.random.default_rng(n + batch)
    x = rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))
    x[0] *= 1e4
    x[-1] *= 1e-4
    x = x.astype(np.complex64)
    with emu_f.mkaux("dft", [n]) as a:
        a.set_form(FORM_SPLIT_TC)
        for kind in ("dft", "invdft"):
            y = np.zeros_like(x)
            a.batched(kind, x, y, batch, n, n)
            ref = oracle_d.transform(kind, x.astype(np.complex128))
            errs = [rel_l2(y[b], ref[b]) for b in range(batch)]
            assert max(errs) <= 2e-6, (kind, errs)

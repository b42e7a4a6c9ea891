"""GPU parity of the CUDA library against the oracle (long-double CPU
restatement, pinned to the reference's own outputs in tests/test_oracle_pin.py).

Every call goes through the C ABI of notorious-fft_b200/lib/libnotorious_fft*.so.
Bar: relative L2 error <= 1e-13 * log2(N) for the double library (the
reference double build's north-star tolerance) and <= 1e-6 * log2(N) for the
float library (its NOTORIOUS_FFT_SINGLE build), with log2(N) floored at 1.
"""
import math

import numpy as np
import pytest

from oracle import ref_fill, rel_l2

pytestmark = pytest.mark.gpu

TOL_D = 1e-13
TOL_F = 1e-6
REF_SIZES = [1, 2, 4, 8, 16, 32, 64, 128, 256, 1024]        # tests/test_notoriousfft.c:673
BLUESTEIN_SIZES = [3, 5, 6, 7, 10, 12, 15, 20, 100]         # tests/test_notoriousfft.c:770
R2R = ["dct2", "dst2", "dct3", "dst3", "dct4", "dst4"]


def tol(n, single=False):
    return (TOL_F if single else TOL_D) * max(1.0, math.log2(max(n, 2)))


def cx(rng, *shape):
    return rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)


# ---------------------------------------------------------------------------
# the reference test suite's cases, with its sin fixture
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n", REF_SIZES)
def test_reference_suite_1d(lib_d, oracle_d, n):
    f = ref_fill(2 * n)
    x = f[0::2] + 1j * f[1::2]
    xr = ref_fill(n)
    with lib_d.mkaux("dft", [n]) as a:
        for k in ("dft", "invdft"):
            assert rel_l2(a(k, x), oracle_d.transform(k, x)) <= tol(n), k
    with lib_d.mkaux("realdft", [n]) as a:
        z = a("realdft", xr)
        assert rel_l2(z, oracle_d.transform("realdft", xr)) <= tol(n)
        if n > 1:  # the reference suite skips invrealdft N=1
            zz = oracle_d.transform("realdft", xr)
            assert rel_l2(a("invrealdft", zz), oracle_d.invrealdft(zz, n)) <= tol(n)
    with lib_d.mkaux("t2t3", [n]) as a:
        for k in R2R[:4]:
            assert rel_l2(a(k, xr), oracle_d.transform(k, xr)) <= tol(n), k
    with lib_d.mkaux("t4", [n]) as a:
        for k in R2R[4:]:
            assert rel_l2(a(k, xr), oracle_d.transform(k, xr)) <= tol(n), k


@pytest.mark.parametrize("n", BLUESTEIN_SIZES)
def test_reference_bluestein_kat(lib_d, n):
    """Known-answer test of the reference suite: O(N^2) DFT, 1e-9 max-abs
    (tests/test_notoriousfft.c:609-670)."""
    i = np.arange(n)
    xr = np.sin(i * 1.23456789 + 0.1 * i * i)
    xi = np.sin(i * 2.71828 + 0.5)
    x = xr + 1j * xi
    ang = -2.0 * np.pi * np.outer(i, i) / n
    ref = (np.cos(ang) + 1j * np.sin(ang)) @ x
    with lib_d.mkaux("dft", [n]) as a:
        y = a("dft", x)
    assert np.max(np.abs(np.concatenate([(y - ref).real, (y - ref).imag]))) < 1e-9
    assert rel_l2(y, ref) <= tol(n)


@pytest.mark.parametrize("dims", [(4, 4), (8, 16), (32, 32), (4, 4, 4), (4, 8, 8)])
def test_reference_suite_nd(lib_d, oracle_d, dims):
    total = int(np.prod(dims))
    f = ref_fill(2 * total)
    x = (f[0::2] + 1j * f[1::2]).reshape(dims)
    xr = ref_fill(total).reshape(dims)
    with lib_d.mkaux("dft", dims) as a:
        for k in ("dft", "invdft"):
            assert rel_l2(a(k, x), oracle_d.nd(k, x)) <= tol(total), k
    with lib_d.mkaux("t2t3", dims) as a:
        for k in R2R[:4]:
            assert rel_l2(a(k, xr), oracle_d.nd(k, xr)) <= tol(total), k
    with lib_d.mkaux("t4", dims) as a:
        for k in R2R[4:]:
            assert rel_l2(a(k, xr), oracle_d.nd(k, xr)) <= tol(total), k


# ---------------------------------------------------------------------------
# sizes: single-pass, multi-pass, Bluestein
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n", [2048, 4096, 8192, 16384, 65536, 1 << 17, 1 << 20])
def test_dft_pow2_sizes(lib_d, oracle_d, n):
    rng = np.random.default_rng(n)
    x = cx(rng, n)
    with lib_d.mkaux("dft", [n]) as a:
        for k in ("dft", "invdft"):
            assert rel_l2(a(k, x), oracle_d.transform(k, x)) <= tol(n), k


@pytest.mark.parametrize("n", [17, 255, 1000, 4097, 65537, 1000003])
def test_dft_bluestein_sizes(lib_d, oracle_d, n):
    rng = np.random.default_rng(n)
    x = cx(rng, n)
    with lib_d.mkaux("dft", [n]) as a:
        for k in ("dft", "invdft"):
            assert rel_l2(a(k, x), oracle_d.transform(k, x)) <= tol(n), k


@pytest.mark.parametrize("n", [4096, 8192, 16384, 32768, 1 << 20])
def test_real_families_sizes(lib_d, oracle_d, n):
    rng = np.random.default_rng(n + 1)
    x = rng.uniform(-1, 1, n)
    with lib_d.mkaux("realdft", [n]) as a:
        z = oracle_d.transform("realdft", x)
        assert rel_l2(a("realdft", x), z) <= tol(n)
        assert rel_l2(a("invrealdft", z), oracle_d.invrealdft(z, n)) <= tol(n)
    if n <= 32768:
        with lib_d.mkaux("t2t3", [n]) as a:
            for k in R2R[:4]:
                assert rel_l2(a(k, x), oracle_d.transform(k, x)) <= tol(n), k
        with lib_d.mkaux("t4", [n]) as a:
            for k in R2R[4:]:
                assert rel_l2(a(k, x), oracle_d.transform(k, x)) <= tol(n), k


# ---------------------------------------------------------------------------
# the C1 configuration: 256 x N=4096 forward + inverse, device memory
# ---------------------------------------------------------------------------
def test_config1_batched_device(lib_d, oracle_d):
    import torch
    rng = np.random.default_rng(1)
    x = (rng.uniform(-1, 1, (256, 4096)) + 1j * rng.uniform(-1, 1, (256, 4096))).astype(np.complex128)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    zd = torch.empty_like(xd)
    with lib_d.mkaux("dft", [4096]) as a:
        a.batched("dft", xd, yd, 256, 4096, 4096)
        a.batched("invdft", yd, zd, 256, 4096, 4096)
        lib_d.synchronize()
    y = yd.cpu().numpy()
    ref = oracle_d.transform("dft", x)
    for b in range(256):
        assert rel_l2(y[b], ref[b]) <= tol(4096)
    assert rel_l2(zd.cpu().numpy(), x * 4096) <= 2 * tol(4096)


# ---------------------------------------------------------------------------
# the C2 mix (sizes of the configuration; batch trimmed where the oracle is slow)
# ---------------------------------------------------------------------------
def test_config2_realdft_2p20(lib_d, oracle_d):
    import torch
    n, B = 1 << 20, 16
    rng = np.random.default_rng(20)
    x = rng.standard_normal((B, n))
    xd = torch.from_numpy(x).cuda()
    zd = torch.empty((B, n // 2 + 1), dtype=torch.complex128, device="cuda")
    with lib_d.mkaux("realdft", [n]) as a:
        a.batched("realdft", xd, zd, B, n, n // 2 + 1)
        lib_d.synchronize()
    z = zd.cpu().numpy()
    for b in (0, B - 1):
        assert rel_l2(z[b], oracle_d.transform("realdft", x[b])) <= tol(n)
    # the rest against numpy (double FFT, accurate to ~1e-16 log2 N)
    assert rel_l2(z, np.fft.rfft(x, axis=1)) <= tol(n)


@pytest.mark.parametrize("kind", ["dct2", "dst2", "dct4"])
def test_config2_r2r_8192x512(lib_d, oracle_d, kind):
    import torch
    n, B = 8192, 512
    rng = np.random.default_rng(8192)
    x = rng.uniform(-1, 1, (B, n))
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    fam = "t4" if kind == "dct4" else "t2t3"
    with lib_d.mkaux(fam, [n]) as a:
        a.batched(kind, xd, yd, B, n, n)
        lib_d.synchronize()
    y = yd.cpu().numpy()
    ref = oracle_d.transform(kind, x[:16])
    assert rel_l2(y[:16], ref) <= tol(n)
    import scipy.fft as sf
    t = {"dct2": (sf.dct, 2), "dst2": (sf.dst, 2), "dct4": (sf.dct, 4)}[kind]
    assert rel_l2(y, t[0](x, type=t[1], axis=1)) <= tol(n)


@pytest.mark.parametrize("dims", [(2048, 2048), (256, 256, 256)])
def test_config2_nd(lib_d, oracle_d, dims):
    import torch
    rng = np.random.default_rng(len(dims))
    x = cx(rng, *dims)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    with lib_d.mkaux("dft", dims) as a:
        a.batched("dft", xd, yd, 1, 0, 0)
        lib_d.synchronize()
    assert rel_l2(yd.cpu().numpy(), oracle_d.nd("dft", x)) <= tol(int(np.prod(dims)))


def test_config2_bluestein_1000003x4(lib_d, oracle_d):
    import torch
    n, B = 1000003, 4
    rng = np.random.default_rng(1000003)
    x = cx(rng, B, n)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    with lib_d.mkaux("dft", [n]) as a:
        a.batched("dft", xd, yd, B, n, n)
        lib_d.synchronize()
    y = yd.cpu().numpy()
    assert rel_l2(y[0], oracle_d.transform("dft", x[0])) <= tol(n)
    assert rel_l2(y, np.fft.fft(x, axis=1)) <= tol(n)


# ---------------------------------------------------------------------------
# API behaviour
# ---------------------------------------------------------------------------
def test_invalid_sizes_return_null(lib_d):
    for fam in ("realdft", "t2t3", "t4"):
        assert not lib_d.mkaux_1d_raw(fam, 12)      # non-power-of-two: NULL (src/07_legacy.h:1442,1579)
        assert not lib_d.mkaux_1d_raw(fam, 0)
    assert not lib_d.mkaux_1d_raw("dft", 0)
    assert not lib_d.mkaux_1d_raw("dft", -5)
    p = lib_d.mkaux_1d_raw("dft", 12)                 # non-power-of-two dft is valid (Bluestein)
    assert p
    lib_d.free_raw(p)
    lib_d.free_raw(None)                              # free_aux(NULL) is a no-op


def test_inplace_and_strided(lib_d, oracle_d):
    rng = np.random.default_rng(7)
    for n in (1024, 1 << 16, 1000):
        x = cx(rng, n)
        y = x.copy()
        with lib_d.mkaux("dft", [n]) as a:
            lib_d._call(lib_d.lib.notorious_fft_dft, y, y, a)
        assert rel_l2(y, oracle_d.transform("dft", x)) <= tol(n)
    n, B = 4096, 5
    xb = cx(rng, B, n + 9)
    yb = np.zeros((B, n + 3), complex)
    with lib_d.mkaux("dft", [n]) as a:
        a.batched("dft", xb, yb, B, n + 9, n + 3)
    assert rel_l2(yb[:, :n], oracle_d.transform("dft", xb[:, :n])) <= tol(n)


# ---------------------------------------------------------------------------
# float library (NOTORIOUS_FFT_SINGLE)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n", [1, 2, 16, 1024, 8192, 65536, 1000])
def test_float_library(lib_f, oracle_d, n):
    rng = np.random.default_rng(n)
    x = cx(rng, n).astype(np.complex64)
    xr = rng.uniform(-1, 1, n).astype(np.float32)
    with lib_f.mkaux("dft", [n]) as a:
        for k in ("dft", "invdft"):
            assert rel_l2(a(k, x), oracle_d.transform(k, x.astype(np.complex128))) <= tol(n, True), k
    if n & (n - 1) == 0:
        with lib_f.mkaux("t2t3", [n]) as a:
            for k in R2R[:4]:
                assert rel_l2(a(k, xr), oracle_d.transform(k, xr.astype(np.float64))) <= tol(n, True), k
        with lib_f.mkaux("realdft", [n]) as a:
            assert rel_l2(a("realdft", xr), oracle_d.transform("realdft", xr.astype(np.float64))) <= tol(n, True)


# ---------------------------------------------------------------------------
# split tensor-core precision form (float library): configuration C3 shape
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n", [1 << 16, 4096, 1 << 14])
def test_split_tc_form_error_per_transform(lib_f, oracle_d, n):
    """FP32 storage, radix-16 DFTs as FP16 hi+lo tensor-core products: every
    transform within 2e-6 relative L2 of the FP64 oracle, including a 10%
    subset scaled by 1e4 (per-butterfly power-of-two scaling)."""
    import torch
    from notorious_fft import FORM_SPLIT_TC
    B = 20
    rng = np.random.default_rng(n)
    x = (rng.standard_normal((B, n)) + 1j * rng.standard_normal((B, n)))
    big = rng.choice(B, 2, replace=False)
    x[big] *= 1e4
    x = x.astype(np.complex64)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    with lib_f.mkaux("dft", [n]) as a:
        a.set_form(FORM_SPLIT_TC)
        assert a.form == FORM_SPLIT_TC
        for kind in ("dft", "invdft"):
            a.batched(kind, xd, yd, B, n, n)
            lib_f.synchronize()
            y = yd.cpu().numpy()
            ref = oracle_d.transform(kind, x.astype(np.complex128))
            errs = [rel_l2(y[b], ref[b]) for b in range(B)]
            assert max(errs) <= 2e-6, (kind, max(errs))


def test_split_tc_form_rejected_by_double_library(lib_d):
    from notorious_fft import FORM_SPLIT_TC, NotoriousFFTError
    with lib_d.mkaux("dft", [4096]) as a:
        with pytest.raises(NotoriousFFTError):
            a.set_form(FORM_SPLIT_TC)


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("n", [64, 4096, 16384])
def test_real_rows_odd_batch_stride(lib_d, lib_f, oracle_d, single, n):
    """Batched single-pass real transforms with an odd input stride (every other
    transform off the 16-byte boundary): realdft, DCT-2 / DST-2, DCT-4 / DST-4."""
    lib = lib_f if single else lib_d
    lim = (1e-6 if single else 1e-13) * max(1.0, math.log2(n))
    B, idist = 5, n + 1
    rng = np.random.default_rng(n + 9)
    x = rng.uniform(-1, 1, B * idist).astype(lib.rdt)
    with lib.mkaux("realdft", [n]) as a:
        z = np.zeros(B * (n // 2 + 1), lib.cdt)
        a.batched("realdft", x, z, B, idist, n // 2 + 1)
        for b in range(B):
            ref = oracle_d.transform("realdft", x[b * idist: b * idist + n].astype(np.float64))
            assert rel_l2(z[b * (n // 2 + 1):(b + 1) * (n // 2 + 1)], ref) <= lim, b
    for fam, kinds in (("t2t3", ("dct2", "dst2")), ("t4", ("dct4", "dst4"))):
        with lib.mkaux(fam, [n]) as a:
            for k in kinds:
                y = np.zeros(B * n, lib.rdt)
                a.batched(k, x, y, B, idist, n)
                for b in range(B):
                    ref = oracle_d.transform(k, x[b * idist: b * idist + n].astype(np.float64))
                    assert rel_l2(y[b * n:(b + 1) * n], ref) <= lim, (k, b)

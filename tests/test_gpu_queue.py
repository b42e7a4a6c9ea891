"""Ragged batches on the GPU: one persistent launch per batch.

Parity of the queue against the oracle (the same cases as the emulator tests,
plus a batch shaped like the uneven-batch configuration: N log-uniform on
[16, 2^18], 20% lengths that are not powers of two -- half of them prime --,
50% c2c / 30% realdft / 20% DCT-2), graph and direct launches, device
tensors, and the bounded dependency wait (a withheld counter ends the launch
with NOTORIOUS_FFT_ERR_TIMEOUT; the context stays usable).
"""
import numpy as np
import pytest
import scipy.fft as sf

from oracle import rel_l2
from test_queue_emulator import expected, got_of, in_reals, out_reals, packed_offsets, run_and_check

pytestmark = pytest.mark.gpu


def _is_prime(n):
    if n < 2:
        return False
    i = 2
    while i * i <= n:
        if n % i == 0:
            return False
        i += 1
    return True


def uneven_config(count, seed, nmax=1 << 18):
    """Kinds and lengths of the uneven-batch configuration (seeded)."""
    rng = np.random.default_rng(seed)
    kinds, Ns = [], []
    lo, hi = np.log2(16), np.log2(nmax)
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
                while not _is_prime(n):
                    n += 1
            else:
                if n & (n - 1) == 0:
                    n += 1
                while _is_prime(n) or n & (n - 1) == 0:
                    n += 1
        kinds.append(kind)
        Ns.append(min(n, nmax) if n & (n - 1) == 0 else n)
    return kinds, Ns


@pytest.mark.parametrize("single", [False, True])
def test_mixed(lib_d, lib_f, oracle_d, single):
    lib = lib_f if single else lib_d
    kinds = ["dft", "realdft", "dct2", "dft", "invdft", "dft", "realdft", "dct2", "dft", "dst2", "dct3", "dst4",
             "invrealdft", "dct4", "dst3", "dft", "realdft", "dct2", "dft"]
    Ns = [64, 128, 256, 16, 64, 7, 6, 9, 1, 32, 64, 128, 64, 16, 256, 65536, 1 << 18, 1 << 15, 100003]
    run_and_check(lib, oracle_d, kinds, Ns, seed=4)


def test_multi_pass_and_bluestein(lib_d, oracle_d):
    kinds = ["dft", "dft", "realdft", "dct2", "dft", "invdft", "realdft", "dct2", "dft", "dft"]
    Ns = [8192, 8192, 16384, 16384, 5000, 3001, 2500, 2049, 4096, 1 << 18]
    run_and_check(lib_d, oracle_d, kinds, Ns, seed=1)


@pytest.mark.parametrize("single", [False, True])
def test_uneven_config_subset(lib_d, lib_f, oracle_d, single):
    """1,000 transforms of the uneven configuration; every output against
    scipy in FP64, 150 random transforms against the oracle."""
    lib = lib_f if single else lib_d
    kinds, Ns = uneven_config(1000, seed=11)
    b = lib.mkbatch(kinds, Ns)
    rng = np.random.default_rng(12)
    x = rng.uniform(-1, 1, b.in_size).astype(lib.rdt)
    y = np.full(b.out_size, np.nan, lib.rdt)
    b.execute(x, y)
    assert b.status() == 0
    io = packed_offsets(kinds, Ns, in_reals)
    oo = packed_offsets(kinds, Ns, out_reals)
    tol = 3e-6 if single else 3e-15
    check = set(rng.choice(len(kinds), 150, replace=False).tolist())
    for i, (k, n) in enumerate(zip(kinds, Ns)):
        xi = x[io[i]: io[i] + in_reals(k, n)].astype(np.float64)
        got = got_of(k, y[oo[i]: oo[i] + out_reals(k, n)].astype(np.float64))
        if k == "dft":
            ref = np.fft.fft(xi[0::2] + 1j * xi[1::2])
        elif k == "realdft":
            ref = np.fft.rfft(xi)
        else:
            ref = sf.dct(xi, type=2)
        lim = tol * max(1, np.log2(n))
        assert rel_l2(got, ref) <= 4 * lim, (i, k, n)
        if i in check:
            assert rel_l2(got, expected(oracle_d, k, xi, n)) <= lim, (i, k, n)


def test_graph_and_direct_agree(lib_d):
    kinds, Ns = uneven_config(300, seed=3, nmax=1 << 16)
    b = lib_d.mkbatch(kinds, Ns)
    x = np.random.default_rng(0).uniform(-1, 1, b.in_size)
    y1 = np.zeros(b.out_size)
    y2 = np.zeros(b.out_size)
    b.set_graph(True)
    b.execute(x, y1)
    b.execute(x, y1)
    b.set_graph(False)
    b.execute(x, y2)
    assert np.array_equal(y1, y2)


def test_device_tensors_one_launch(lib_d, oracle_d):
    import torch
    kinds = ["dft", "realdft", "dct2", "dft"] * 8
    Ns = [4096, 1 << 15, 8192, 1 << 17] * 8
    b = lib_d.mkbatch(kinds, Ns)
    x = torch.rand(b.in_size, dtype=torch.float64, device="cuda") * 2 - 1
    y = torch.zeros(b.out_size, dtype=torch.float64, device="cuda")
    n0 = lib_d.launch_count()
    b.execute(x, y)
    assert lib_d.launch_count() - n0 == 1
    assert b.status() == 0
    xh, yh = x.cpu().numpy(), y.cpu().numpy()
    io, oo = packed_offsets(kinds, Ns, in_reals), packed_offsets(kinds, Ns, out_reals)
    for i in (0, 1, 2, 3):
        k, n = kinds[i], Ns[i]
        ref = expected(oracle_d, k, xh[io[i]: io[i] + in_reals(k, n)], n)
        assert rel_l2(got_of(k, yh[oo[i]: oo[i] + out_reals(k, n)]), ref) <= 3e-15 * np.log2(n)


def test_withheld_dependency_times_out(lib_d, oracle_d):
    """A counter that nothing publishes: the waiting CTA gives up after the
    spin limit, raises the abort flag, and the launch ends with TIMEOUT; the
    next launch of the same batch is correct."""
    from notorious_fft import NotoriousFFTError
    kinds, Ns = ["dft"] * 4, [1 << 16] * 4
    b = lib_d.mkbatch(kinds, Ns)
    x = np.random.default_rng(0).uniform(-1, 1, b.in_size)
    y = np.zeros(b.out_size)
    b.withhold(20000)
    with pytest.raises(NotoriousFFTError, match="error 5"):
        b.execute(x, y)
    b.execute(x, y)
    assert b.status() == 0
    n = 1 << 16
    xc = x[: 2 * n][0::2] + 1j * x[: 2 * n][1::2]
    assert rel_l2(y[: 2 * n][0::2] + 1j * y[: 2 * n][1::2], oracle_d.transform("dft", xc)) <= 3e-15 * 16

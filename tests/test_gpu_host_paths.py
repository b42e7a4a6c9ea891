"""Host-memory and multi-stream calls through the C ABI, against the oracle.

* Pinned host buffers on a batch of >= 4 transforms take the pipelined path
  (csrc/nfft_api.cu run_pipelined: chunks of ~64 MiB, copy-in of chunk k+1
  and copy-out of chunk k-1 overlapping the transform of chunk k on two copy
  streams).  The batches here span at least three chunks, in both
  libraries, out of place, in place (x == y) and with odd distances.  The
  reference's own callers pass host pointers (benchmarks/bench.c:35-55).
* Pageable host buffers on a batch of >= 4 transforms take the same chunked
  pipeline with pinned bounce buffers filled and drained by host threads
  (csrc/nfft_api.cu run_pageable_pipelined); smaller batches the staged path
  (one copy in, one copy out).
* Two device-pointer calls on one aux from two streams: the plan's scratch is
  shared, so the second call waits for the first (csrc/nfft_api.cu
  order_after_previous_call); both results must match the oracle.
"""
import math

import numpy as np
import pytest

from oracle import rel_l2

pytestmark = pytest.mark.gpu


def _tol(n, single):
    return (1e-6 if single else 1e-13) * max(1.0, math.log2(n))


def _pinned(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t, t.numpy()


def _sample(batch):
    """Transforms checked against the oracle: both ends and every chunk boundary region."""
    return sorted({0, 1, batch // 3, batch // 2, 2 * batch // 3, batch - 2, batch - 1})


@pytest.mark.parametrize("single", [False, True], ids=["double", "float"])
@pytest.mark.parametrize("in_place", [False, True], ids=["out-of-place", "in-place"])
def test_pipelined_c2c(lib_d, lib_f, oracle_d, single, in_place):
    lib = lib_f if single else lib_d
    es = 8 if single else 16
    n = 4096
    idist = n + 3                                  # odd distance
    batch = 3 * (64 << 20) // (idist * es) + 7     # a little over three 64 MiB chunks
    rng = np.random.default_rng(batch)
    x = (rng.uniform(-1, 1, batch * idist) + 1j * rng.uniform(-1, 1, batch * idist)).astype(lib.cdt)
    xt, xh = _pinned(x)
    if in_place:
        yt, yh = xt, xh
        odist = idist
    else:
        odist = n + 1
        yt, yh = _pinned(np.full(batch * odist, np.nan, lib.cdt))
    with lib.mkaux("dft", [n]) as a:
        a.batched("dft", xh, yh, batch, idist, odist)
    got = yh.reshape(-1)
    tol = _tol(n, single)
    for b in _sample(batch):
        ref = oracle_d.transform("dft", x[b * idist: b * idist + n].astype(np.complex128))
        assert rel_l2(got[b * odist: b * odist + n], ref) <= tol, b
    # every transform of the batch against numpy's double FFT
    xb = np.lib.stride_tricks.as_strided(x, (batch, n), (idist * x.itemsize, x.itemsize))
    yb = np.lib.stride_tricks.as_strided(got, (batch, n), (odist * got.itemsize, got.itemsize))
    assert rel_l2(yb, np.fft.fft(xb.astype(np.complex128), axis=1)) <= tol


@pytest.mark.parametrize("single", [False, True], ids=["double", "float"])
def test_pipelined_realdft_odd_distance(lib_d, lib_f, oracle_d, single):
    lib = lib_f if single else lib_d
    rs = 4 if single else 8
    n = 8192
    idist = n + 1                                  # odd distance of the real input
    odist = n // 2 + 1
    batch = 3 * (64 << 20) // (idist * rs) + 5
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, batch * idist).astype(lib.rdt)
    _, xh = _pinned(x)
    _, zh = _pinned(np.full(batch * odist, np.nan, lib.cdt))
    with lib.mkaux("realdft", [n]) as a:
        a.batched("realdft", xh, zh, batch, idist, odist)
        tol = _tol(n, single)
        for b in _sample(batch):
            ref = oracle_d.transform("realdft", x[b * idist: b * idist + n].astype(np.float64))
            assert rel_l2(zh[b * odist:(b + 1) * odist], ref) <= tol, b
        # and back: the adjoint through the pipelined path (cotangent -> N reals)
        g = (rng.uniform(-1, 1, batch * odist) + 1j * rng.uniform(-1, 1, batch * odist)).astype(lib.cdt)
        _, gh = _pinned(g)
        _, gxh = _pinned(np.full(batch * n, np.nan, lib.rdt))
        a.vjp_batched("realdft", gh, gxh, batch, odist, n)
    for b in _sample(batch):
        w = g[b * odist:(b + 1) * odist].astype(np.complex128)
        w[1:-1] *= 0.5
        assert rel_l2(gxh[b * n:(b + 1) * n], oracle_d.invrealdft(w, n)) <= tol, b


@pytest.mark.parametrize("single", [False, True], ids=["double", "float"])
@pytest.mark.parametrize("in_place", [False, True], ids=["out-of-place", "in-place"])
def test_pageable_pipelined_c2c(lib_d, lib_f, oracle_d, single, in_place):
    """Pageable numpy buffers over more than three 64 MiB chunks, odd distances."""
    lib = lib_f if single else lib_d
    es = 8 if single else 16
    n = 4096
    idist = n + 3
    batch = 3 * (64 << 20) // (idist * es) + 7
    rng = np.random.default_rng(batch + 1)
    x = (rng.uniform(-1, 1, batch * idist) + 1j * rng.uniform(-1, 1, batch * idist)).astype(lib.cdt)
    x0 = x.copy()
    if in_place:
        y, odist = x, idist
    else:
        odist = n + 1
        y = np.full(batch * odist, np.nan, lib.cdt)
    with lib.mkaux("dft", [n]) as a:
        a.batched("dft", x, y, batch, idist, odist)
    tol = _tol(n, single)
    for b in _sample(batch):
        ref = oracle_d.transform("dft", x0[b * idist: b * idist + n].astype(np.complex128))
        assert rel_l2(y[b * odist: b * odist + n], ref) <= tol, b
    xb = np.lib.stride_tricks.as_strided(x0, (batch, n), (idist * x0.itemsize, x0.itemsize))
    yb = np.lib.stride_tricks.as_strided(y, (batch, n), (odist * y.itemsize, y.itemsize))
    assert rel_l2(yb, np.fft.fft(xb.astype(np.complex128), axis=1)) <= tol


def test_pageable_host_batched_dct2(lib_d, oracle_d):
    n, batch = 2048, 9
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, (batch, n + 5))
    y = np.zeros((batch, n + 2))
    with lib_d.mkaux("t2t3", [n]) as a:
        a.batched("dct2", x, y, batch, n + 5, n + 2)
    assert rel_l2(y[:, :n], oracle_d.transform("dct2", x[:, :n])) <= _tol(n, False)


@pytest.mark.parametrize("single", [False, True], ids=["double", "float"])
def test_two_streams_share_one_aux(lib_d, lib_f, oracle_d, single):
    """A long batched call on stream A, then a call on stream B with the same
    aux issued without any host wait: B must wait for A (shared scratch)."""
    import torch
    lib = lib_f if single else lib_d
    cdt = torch.complex64 if single else torch.complex128
    n = 1 << 16
    ba, bb = 512, 64
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    xa = torch.randn(ba, n, generator=g, device="cuda", dtype=cdt)
    xb = torch.randn(bb, n, generator=g, device="cuda", dtype=cdt)
    ya, yb = torch.empty_like(xa), torch.empty_like(xb)
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    sa.wait_stream(torch.cuda.current_stream())
    sb.wait_stream(torch.cuda.current_stream())
    try:
        with lib.mkaux("dft", [n]) as a:
            for _ in range(2):
                lib.set_stream(sa)
                a.batched("dft", xa, ya, ba, n, n)
                lib.set_stream(sb)
                a.batched("invdft", xb, yb, bb, n, n)
            torch.cuda.synchronize()
    finally:
        lib.set_stream(None)
    tol = _tol(n, single)
    xa64, xb64 = xa.cpu().numpy().astype(np.complex128), xb.cpu().numpy().astype(np.complex128)
    ya_, yb_ = ya.cpu().numpy(), yb.cpu().numpy()
    for b in (0, ba // 2, ba - 1):
        assert rel_l2(ya_[b], oracle_d.transform("dft", xa64[b])) <= tol, ("A", b)
    for b in (0, bb - 1):
        assert rel_l2(yb_[b], oracle_d.transform("invdft", xb64[b])) <= tol, ("B", b)
    assert rel_l2(ya_, np.fft.fft(xa64, axis=1)) <= tol
    assert rel_l2(yb_, np.fft.ifft(xb64, axis=1) * n) <= tol

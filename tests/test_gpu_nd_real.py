"""Multi-dimensional realdft / invrealdft on the GPU against the oracle.

The reference declares mkaux_realdft_{2d,3d,(d)} (src/07_legacy.h:1492-1524
of Notorious-FFT) with the FFTW layout its README documents (the last axis
becomes Ns[d-1]/2+1 bins, then complex DFTs along the other axes), but its
execution path crashes there, so the oracle's restatement of that layout
(oracle/nfft_oracle.c realdft_nd / invrealdft_nd) is the pin.  Both
libraries, through the C ABI, on the differentiation configuration's
512 x 512 plane, a 3-D shape, the reference suite's 2-D shapes, and a batch
of 512 x 512 planes with device pointers.  Bars: relative L2 <= 1e-13 log2 N
(double), <= 1e-6 log2 N (float), N the total size.
"""
import math

import numpy as np
import pytest

from oracle import rel_l2

pytestmark = pytest.mark.gpu

SHAPES = [(512, 512), (16, 32, 64), (4, 4), (8, 16), (32, 32), (64, 2048), (2, 8, 4, 16)]


def _tol(dims, single):
    return (1e-6 if single else 1e-13) * max(1.0, math.log2(int(np.prod(dims))))


@pytest.mark.parametrize("single", [False, True], ids=["double", "float"])
@pytest.mark.parametrize("dims", SHAPES, ids=lambda d: "x".join(map(str, d)))
def test_nd_realdft_and_inverse(lib_d, lib_f, oracle_d, single, dims):
    lib = lib_f if single else lib_d
    rng = np.random.default_rng(int(np.prod(dims)) + len(dims))
    x = rng.standard_normal(dims).astype(lib.rdt)
    x64 = x.astype(np.float64)
    tol = _tol(dims, single)
    with lib.mkaux("realdft", dims) as a:
        z = a("realdft", x)
        zref = oracle_d.nd("realdft", x64)
        assert z.shape == zref.shape
        assert rel_l2(z, zref) <= tol
        # the inverse of a Hermitian spectrum (a round trip) ...
        y = a("invrealdft", zref.astype(lib.cdt))
        assert rel_l2(y, oracle_d.nd("invrealdft", zref, dims)) <= tol
        assert rel_l2(y, x64 * np.prod(dims)) <= 2 * tol
        # ... and of an arbitrary one: complex inverse DFTs along the leading
        # axes, then the inverse real DFT of each last-axis line, which reads
        # only the real parts of bins 0 and Ns[d-1]/2
        w = (rng.uniform(-1, 1, zref.shape) + 1j * rng.uniform(-1, 1, zref.shape)).astype(lib.cdt)
        assert rel_l2(a("invrealdft", w), oracle_d.nd("invrealdft", w.astype(np.complex128), dims)) <= tol


@pytest.mark.parametrize("single", [False, True], ids=["double", "float"])
def test_nd_realdft_batched_device(lib_d, lib_f, oracle_d, single):
    import torch
    lib = lib_f if single else lib_d
    B, N1, N2 = 4, 512, 512
    rng = np.random.default_rng(512)
    x = rng.standard_normal((B, N1, N2)).astype(lib.rdt)
    xd = torch.from_numpy(x).cuda()
    zd = torch.empty((B, N1, N2 // 2 + 1), dtype=torch.complex64 if single else torch.complex128, device="cuda")
    yd = torch.empty_like(xd)
    tol = _tol((N1, N2), single)
    with lib.mkaux("realdft", [N1, N2]) as a:
        a.batched("realdft", xd, zd, B, N1 * N2, N1 * (N2 // 2 + 1))
        a.batched("invrealdft", zd, yd, B, N1 * (N2 // 2 + 1), N1 * N2)
        lib.synchronize()
    z, y = zd.cpu().numpy(), yd.cpu().numpy()
    for b in range(B):
        zref = oracle_d.nd("realdft", x[b].astype(np.float64))
        assert rel_l2(z[b], zref) <= tol, b
        assert rel_l2(y[b], oracle_d.nd("invrealdft", z[b].astype(np.complex128), (N1, N2))) <= tol, b

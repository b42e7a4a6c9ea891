"""GPU test of the allocation-free entry point notorious_fft_dft_noalloc.

Some callers of this library cannot call cudaMalloc (code inside another
framework's memory manager, latency-critical code that cannot take its
implicit synchronization).  For them the library exports one more C entry
point whose scratch is a fixed __device__ array instead of allocated memory.
This file checks, through the C ABI, that it returns what the regular
batched entry point returns and what the oracle returns (same tolerance as
the parity tests), on two calls in a row (the second call reuses the shared
scratch array left by the first), for lengths that need the scratch (two
passes in the whole array, three passes alternating between its halves) and
for one that does not, in both libraries and in place.  The file name sorts
last so that a run stopping at the first failure has already run every other
test.
"""
import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_fn(lib):
    fn = lib.lib.notorious_fft_dft_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _rel(a, b):
    import torch
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def _check(lib, n, batch, inverse, in_place=False):
    import torch

    from oracle import Oracle
    fn = _noalloc_fn(lib)
    rdt = torch.float32 if lib.single else torch.float64
    g = torch.Generator(device="cuda")
    g.manual_seed(n + inverse)
    x = torch.complex(torch.rand(batch, n, generator=g, device="cuda", dtype=rdt) * 2 - 1,
                      torch.rand(batch, n, generator=g, device="cuda", dtype=rdt) * 2 - 1)
    ref = torch.empty_like(x)
    kind = "invdft" if inverse else "dft"
    with lib.mkaux("dft", [n]) as a:
        a.batched(kind, x, ref, batch, n, n)
    torch.cuda.synchronize()
    tol = (1e-6 if lib.single else 1e-13) * max(1.0, math.log2(n))
    # the oracle (long double) on the first and last transform of the batch
    oracle = Oracle(single=False)
    xs = x[[0, batch - 1]].cpu().numpy().astype(np.complex128)
    oref = oracle.transform(kind, xs)
    for _ in range(2):
        y = x.clone() if in_place else torch.full_like(x, float("nan"))
        src = y if in_place else x
        rc = fn(src.data_ptr(), y.data_ptr(), n, batch, inverse, torch.cuda.current_stream().cuda_stream)
        assert rc == 0, lib.last_error()
        torch.cuda.synchronize()
        assert _rel(y, ref) <= tol
        ys = y[[0, batch - 1]].cpu().numpy()
        for i in range(2):
            assert np.linalg.norm(ys[i] - oref[i]) <= tol * np.linalg.norm(oref[i])


# 2^19 / 2^20 run three passes by default (FP64 2^20 fills the whole scratch
# and takes the two-pass schedule); 4096 is a single pass
@pytest.mark.parametrize("n,batch", [(1 << 16, 8), (1 << 20, 3), (1 << 19, 5), (1 << 14, 5), (4096, 7)])
@pytest.mark.parametrize("inverse", [0, 1])
def test_noalloc_matches_batched_entry(lib_d, n, batch, inverse):
    _check(lib_d, n, batch, inverse)


@pytest.mark.parametrize("n,batch", [(1 << 20, 3), (1 << 17, 9), (4096, 7)])
@pytest.mark.parametrize("inverse", [0, 1])
def test_noalloc_float_library(lib_f, n, batch, inverse):
    _check(lib_f, n, batch, inverse)


# 4096 is one pass straight from x to y (no scratch), the in-place case of
# the single-pass branch
@pytest.mark.parametrize("single,n", [(False, 1 << 19), (False, 1 << 20), (False, 1 << 16), (True, 1 << 20),
                                      (False, 4096), (True, 4096)])
def test_noalloc_in_place(lib_d, lib_f, single, n):
    _check(lib_f if single else lib_d, n, 3, 0, in_place=True)


def test_noalloc_rejects_oversize_and_non_power_of_two(lib_d):
    import torch
    fn = _noalloc_fn(lib_d)
    x = torch.zeros(16, dtype=torch.complex128, device="cuda")
    assert fn(x.data_ptr(), x.data_ptr(), (1 << 20) * 2, 1, 0, None) == 1
    assert "2^20" in lib_d.last_error()[1] or "1048576" in lib_d.last_error()[1]
    assert fn(x.data_ptr(), x.data_ptr(), 12, 1, 0, None) == 1

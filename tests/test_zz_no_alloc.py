"""GPU test of the allocation-free entry point notorious_fft_dft_noalloc.

Some callers of this library cannot call cudaMalloc (code inside another
framework's memory manager, latency-critical code that cannot take its
implicit synchronization).  For them the library exports one more C entry
point whose scratch is a fixed __device__ array instead of allocated memory.
This file checks, through the C ABI, that it returns what the regular
batched entry point returns (same tolerance as the parity tests), on two
calls in a row (the second call reuses the shared scratch array left by the
first), for lengths that need the scratch and for one that does not.  The
file name sorts last so that a run stopping at the first failure has already
run every other test.
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


@pytest.mark.parametrize("n,batch", [(1 << 16, 8), (1 << 20, 3), (1 << 14, 5), (4096, 7)])
@pytest.mark.parametrize("inverse", [0, 1])
def test_noalloc_matches_batched_entry(lib_d, n, batch, inverse):
    import torch
    fn = _noalloc_fn(lib_d)
    g = torch.Generator(device="cuda")
    g.manual_seed(n + inverse)
    x = torch.complex(torch.rand(batch, n, generator=g, device="cuda", dtype=torch.float64) * 2 - 1,
                      torch.rand(batch, n, generator=g, device="cuda", dtype=torch.float64) * 2 - 1)
    ref = torch.empty_like(x)
    kind = "invdft" if inverse else "dft"
    with lib_d.mkaux("dft", [n]) as a:
        a.batched(kind, x, ref, batch, n, n)
    torch.cuda.synchronize()
    tol = 1e-13 * max(1.0, math.log2(n))
    for _ in range(2):
        y = torch.full_like(x, float("nan"))
        rc = fn(x.data_ptr(), y.data_ptr(), n, batch, inverse, torch.cuda.current_stream().cuda_stream)
        assert rc == 0, lib_d.last_error()
        torch.cuda.synchronize()
        assert _rel(y, ref) <= tol


def test_noalloc_rejects_oversize_and_non_power_of_two(lib_d):
    import torch
    fn = _noalloc_fn(lib_d)
    x = torch.zeros(16, dtype=torch.complex128, device="cuda")
    assert fn(x.data_ptr(), x.data_ptr(), (1 << 20) * 2, 1, 0, None) == 1
    assert "2^20" in lib_d.last_error()[1] or "1048576" in lib_d.last_error()[1]
    assert fn(x.data_ptr(), x.data_ptr(), 12, 1, 0, None) == 1

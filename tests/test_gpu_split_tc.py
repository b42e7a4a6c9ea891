"""GPU parity of the split tensor-core form (float library) on every pass
layout its radix-256 kernels take.

The form's radix-256 passes run on tcgen05 when their lines are unit-stride
and the buffers and batch strides are 16-byte aligned: the row-out first pass
(2^16, 2^24), the column-out middle pass with the line index split at Ns
(2^24) and the column-out last pass with Ns >= lines (2^16, 2^24, and the
second pass of 2^17 = 512 x 256).  2^20 runs passes of 2^7, 2^7, 2^6 (the
generic tensor-core pass).  Odd batch strides take the warp-level kernel.
Every transform is compared with the FP64 oracle (bar: 2e-6 relative L2 up to
2^16, 1e-6 per radix-256 pass beyond), the inverse included, and
notorious_fft_synchronize must report no wait that gave up.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bar(n):
    passes = max(1, (n.bit_length() - 1 + 7) // 8)
    return max(2e-6, 1e-6 * passes)


def run_split(lib_f, x, kind, n, B, idist=None, odist=None):
    import torch
    from notorious_fft import FORM_SPLIT_TC
    idist = idist or n
    odist = odist or n
    xd = torch.zeros(B * idist, dtype=torch.complex64, device="cuda")
    for b in range(B):
        xd[b * idist:b * idist + n] = torch.from_numpy(x[b])
    yd = torch.zeros(B * odist, dtype=torch.complex64, device="cuda")
    with lib_f.mkaux("dft", [n]) as a:
        a.set_form(FORM_SPLIT_TC)
        a.batched(kind, xd, yd, B, idist, odist)
        lib_f.synchronize()
    y = yd.cpu().numpy()
    return np.stack([y[b * odist:b * odist + n] for b in range(B)])


@pytest.mark.parametrize("n,B", [(1 << 20, 2), (1 << 24, 1), (1 << 17, 3)])
def test_split_tc_multipass(lib_f, oracle_d, n, B):
    """Three-pass (2^20: 128 x 128 x 64; 2^24: 256^3, one transform) and
    two-pass (2^17: 512 x 256) transforms: the middle pass of 2^24 writes
    columns split at Ns, its last pass and the radix-256 pass of 2^17 write
    columns with Ns >= lines."""
    rng = np.random.default_rng(n + B)
    x = (rng.standard_normal((B, n)) + 1j * rng.standard_normal((B, n))).astype(np.complex64)
    for kind in ("dft", "invdft"):
        y = run_split(lib_f, x, kind, n, B)
        ref = oracle_d.transform(kind, x.astype(np.complex128))
        errs = [rel_l2(y[b], ref[b]) for b in range(B)]
        assert max(errs) <= bar(n), (kind, errs)


@pytest.mark.parametrize("n", [1 << 16, 1 << 14])
def test_split_tc_odd_batch_stride(lib_f, oracle_d, n):
    """Batch strides of n + 1 complex points (every other transform off the
    16-byte boundary): the radix-256 passes take the warp-level kernel."""
    B = 3
    rng = np.random.default_rng(7 + n)
    x = (rng.standard_normal((B, n)) + 1j * rng.standard_normal((B, n))).astype(np.complex64)
    y = run_split(lib_f, x, "dft", n, B, idist=n + 1, odist=n + 3)
    ref = oracle_d.transform("dft", x.astype(np.complex128))
    assert max(rel_l2(y[b], ref[b]) for b in range(B)) <= bar(n)


CHILD = r"""
import json, sys, numpy as np, torch
sys.path.insert(0, "notorious-fft_b200")
from notorious_fft import load, FORM_SPLIT_TC
lib = load(single=True)
n, B = int(sys.argv[2]), int(sys.argv[3])
rng = np.random.default_rng(3)
x = (rng.standard_normal((B, n)) + 1j * rng.standard_normal((B, n))).astype(np.complex64)
xd = torch.from_numpy(x).cuda().reshape(-1)
yd = torch.empty_like(xd)
with lib.mkaux("dft", [n]) as a:
    a.set_form(FORM_SPLIT_TC)
    a.batched("dft", xd, yd, B, n, n)
    lib.synchronize()
np.save(sys.argv[1], yd.cpu().numpy().reshape(B, n))
"""


@pytest.mark.parametrize("n,B", [(1 << 16, 4), (1 << 16, 1), (1 << 24, 1)])
def test_split_tc_tcgen05_and_warp_kernels_agree(tmp_path, oracle_d, n, B):
    """The same batch through the tcgen05 pass (default) and the warp-level
    pass (NOTORIOUS_FFT_TC_UMMA=0, a child process each): both within the bar
    of the FP64 oracle and within the bar of each other.  2^16 covers the
    row-out and column-out passes (a batch, and one transform); 2^24 adds the
    column-out pass with the line index split at Ns."""
    outs = {}
    for mode in ("1", "0"):
        f = tmp_path / f"y{mode}.npy"
        env = dict(os.environ, NOTORIOUS_FFT_TC_UMMA=mode)
        r = subprocess.run([sys.executable, "-c", CHILD, str(f), str(n), str(B)], cwd=ROOT, env=env,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs[mode] = np.load(f)
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((B, n)) + 1j * rng.standard_normal((B, n))).astype(np.complex64)
    ref = oracle_d.transform("dft", x.astype(np.complex128))
    for mode, y in outs.items():
        assert max(rel_l2(y[b], ref[b]) for b in range(B)) <= bar(n), mode
    assert max(rel_l2(outs["1"][b], outs["0"][b]) for b in range(B)) <= bar(n)


WITHHOLD_CHILD = r"""
import sys, numpy as np, torch
sys.path.insert(0, "notorious-fft_b200")
sys.path.insert(0, "oracle")
from notorious_fft import load, FORM_SPLIT_TC, NotoriousFFTError
from oracle import Oracle, rel_l2
F = load(single=True)
n, B = 65536, 2
x = torch.ones(B * n, dtype=torch.complex64, device="cuda")
y = torch.empty_like(x)
raised = False
with F.mkaux("dft", [n]) as a:
    a.set_form(FORM_SPLIT_TC)
    a.batched("dft", x, y, B, n, n)
    try:
        F.synchronize()
    except NotoriousFFTError as e:
        raised = "gave up" in str(e)
print("raised", raised)
# the context stays usable: a double-library transform against the oracle
D = load(single=False)
rng = np.random.default_rng(1)
xd = rng.uniform(-1, 1, (4, 4096)) + 1j * rng.uniform(-1, 1, (4, 4096))
with D.mkaux("dft", [4096]) as a:
    yd = a("dft", xd[0])
print("after", rel_l2(yd, Oracle().transform("dft", xd[0])))
"""


def test_split_tc_wait_gives_up_and_reports():
    """Failure detection of the tcgen05 pass without a GPU fault: with the first
    input copy withheld (NOTORIOUS_FFT_TC_UMMA_WITHHOLD=1) every CTA's first
    wait runs out after a short poll limit, the kernel frees its tensor memory
    and returns, notorious_fft_synchronize reports the wait, and the context
    still runs transforms correctly."""
    env = dict(os.environ, NOTORIOUS_FFT_TC_UMMA_WITHHOLD="1", NOTORIOUS_FFT_TC_UMMA_SPIN="2000")
    r = subprocess.run([sys.executable, "-c", WITHHOLD_CHILD], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = dict(l.split(" ", 1) for l in r.stdout.strip().splitlines() if " " in l)
    assert lines.get("raised") == "True", r.stdout
    assert float(lines["after"]) <= 1e-13 * 12, r.stdout

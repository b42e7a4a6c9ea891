"""Adjoint (vjp) kernels on the GPU: the differentiation configuration.

Loss  L = sum_k w_k |rfft2(x)_k|^2 + sum_j v_j DCT2(rowmean(x))_j  for x float32
of shape 64 x 512 x 512 ~ N(0, 1), w (64 x 512 x 257) and v (64 x 512) uniform
[0.5, 1.5).  rowmean averages the last axis (64 x 512), DCT-2 runs along its
length-512 rows.  The forward transforms and their adjoints are this library's
kernels (notorious_fft_realdft / dct2 and notorious_fft_vjp_batched), wrapped in
torch.autograd.Function here, in the test harness only.  The gradient is checked
against FP64 central finite differences on 1,000 random coordinates and the
adjoints against the oracle's transforms applied to the cotangents.
"""
import math
import zlib

import numpy as np
import pytest
import scipy.fft as sf

from oracle import rel_l2

pytestmark = pytest.mark.gpu

B, N1, N2 = 64, 512, 512


def _autograd_fns(lib):
    import torch

    rf = lib.mkaux("realdft", [N1, N2])
    dc = lib.mkaux("t2t3", [N1])

    class RFFT2(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x):
            z = torch.empty((x.shape[0], N1, N2 // 2 + 1), dtype=torch.complex64, device=x.device)
            rf.batched("realdft", x, z, x.shape[0], N1 * N2, N1 * (N2 // 2 + 1))
            return z

        @staticmethod
        def backward(ctx, gz):
            # torch's complex gradient convention is dL/dRe + i dL/dIm: the same pairs of reals
            gz = gz.contiguous()
            gx = torch.empty((gz.shape[0], N1, N2), dtype=torch.float32, device=gz.device)
            rf.vjp_batched("realdft", gz, gx, gz.shape[0], N1 * (N2 // 2 + 1), N1 * N2)
            return gx

    class DCT2(torch.autograd.Function):
        @staticmethod
        def forward(ctx, m):
            m = m.contiguous()
            y = torch.empty_like(m)
            dc.batched("dct2", m, y, m.shape[0], N1, N1)
            return y

        @staticmethod
        def backward(ctx, g):
            g = g.contiguous()
            gm = torch.empty_like(g)
            dc.vjp_batched("dct2", g, gm, g.shape[0], N1, N1)
            return gm

    return RFFT2, DCT2, (rf, dc)


def _loss64(x, w, v):
    """FP64 loss of one batch element (numpy / scipy)."""
    z = np.fft.rfft2(x)
    d = sf.dct(x.mean(axis=1), type=2)
    return float(np.sum(w * (z.real ** 2 + z.imag ** 2)) + np.sum(v * d))


def test_differentiation_config(lib_f):
    import torch
    rng = np.random.default_rng(55)
    x = rng.standard_normal((B, N1, N2)).astype(np.float32)
    w = rng.uniform(0.5, 1.5, (B, N1, N2 // 2 + 1)).astype(np.float32)
    v = rng.uniform(0.5, 1.5, (B, N1)).astype(np.float32)
    RFFT2, DCT2, keep = _autograd_fns(lib_f)
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    wt, vt = torch.from_numpy(w).cuda(), torch.from_numpy(v).cuda()
    z = RFFT2.apply(xt)
    loss = (wt * (z.real ** 2 + z.imag ** 2)).sum() + (vt * DCT2.apply(xt.mean(dim=2))).sum()
    loss.backward()
    lib_f.synchronize()
    g = xt.grad.detach().cpu().numpy().astype(np.float64)

    # the loss itself against FP64
    x64 = x.astype(np.float64)
    ref_loss = sum(_loss64(x64[b], w[b], v[b]) for b in range(B))
    assert abs(float(loss.item()) - ref_loss) <= 1e-5 * abs(ref_loss)

    # FP64 central differences on 1,000 random coordinates (the loss is a sum
    # over batch elements, so only the touched element is re-evaluated)
    coords = rng.integers(0, [B, N1, N2], size=(1000, 3))
    h = 1e-3
    scale = np.sqrt(np.mean(g ** 2))
    worst = 0.0
    for b, i, j in coords:
        xp = x64[b].copy()
        xp[i, j] += h
        lp = _loss64(xp, w[b], v[b])
        xp[i, j] -= 2 * h
        lm = _loss64(xp, w[b], v[b])
        fd = (lp - lm) / (2 * h)
        worst = max(worst, abs(g[b, i, j] - fd) / (abs(fd) + scale))
    assert worst <= 1e-4, worst


def test_adjoints_equal_reference_transforms_on_cotangent(lib_f, oracle_d):
    """realdft adjoint = invrealdft of the cotangent with the last axis's
    interior bins halved; DCT-2 adjoint = DCT-3 of the cotangent with entry 0
    doubled (oracle transforms, FP64)."""
    import torch
    rng = np.random.default_rng(8)
    gz = (rng.uniform(-1, 1, (N1, N2 // 2 + 1)) + 1j * rng.uniform(-1, 1, (N1, N2 // 2 + 1))).astype(np.complex64)
    gv = rng.uniform(-1, 1, N2).astype(np.float32)
    with lib_f.mkaux("realdft", [N1, N2]) as a:
        gx = a.vjp("realdft", gz)
    ww = gz.astype(np.complex128)
    ww[:, 1:-1] *= 0.5
    assert rel_l2(gx, oracle_d.nd("invrealdft", ww, (N1, N2))) <= 1e-6 * 18
    with lib_f.mkaux("t2t3", [N2]) as a:
        gm = a.vjp("dct2", gv)
    vv = gv.astype(np.float64)
    vv[0] *= 2
    assert rel_l2(gm, oracle_d.transform("dct3", vv)) <= 1e-6 * 9


@pytest.mark.parametrize("kind", ["dft", "invdft", "realdft", "invrealdft", "dct2", "dst2", "dct3", "dst3", "dct4", "dst4"])
@pytest.mark.parametrize("n", [1024, 1000, 1 << 16])
def test_vjp_inner_product_double(lib_d, kind, n):
    """<g, A x> = <A^T g, x> on the GPU for every transform (double library)."""
    fam = {"dft": "dft", "invdft": "dft", "realdft": "realdft", "invrealdft": "realdft", "dct4": "t4",
           "dst4": "t4"}.get(kind, "t2t3")
    if fam != "dft" and n & (n - 1):
        pytest.skip("power-of-two only")
    rng = np.random.default_rng(n)

    def cx(*s):
        return rng.uniform(-1, 1, s) + 1j * rng.uniform(-1, 1, s)

    def rv(a):
        return np.concatenate([a.real.ravel(), a.imag.ravel()]) if np.iscomplexobj(a) else a.ravel()

    with lib_d.mkaux(fam, [n]) as a:
        ins, outs = a.in_shape(kind), a.out_shape(kind)
        x = cx(*ins) if kind in ("dft", "invdft") else rng.uniform(-1, 1, ins)
        if kind == "invrealdft":
            x = np.fft.rfft(rng.uniform(-1, 1, n))
        g = cx(*outs) if kind in ("dft", "invdft", "realdft") else rng.uniform(-1, 1, outs)
        lhs = np.dot(rv(g), rv(a(kind, x)))
        rhs = np.dot(rv(a.vjp(kind, g)), rv(x))
    assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs)) * math.log2(n)


# ---------------------------------------------------------------------------
# every adjoint against the oracle's transforms of the cotangent
# ---------------------------------------------------------------------------
ALL_KINDS = ["dft", "invdft", "realdft", "invrealdft", "dct2", "dst2", "dct3", "dst3", "dct4", "dst4"]
FAMILY = {"dft": "dft", "invdft": "dft", "realdft": "realdft", "invrealdft": "realdft", "dct4": "t4", "dst4": "t4",
          "dct2": "t2t3", "dst2": "t2t3", "dct3": "t2t3", "dst3": "t2t3"}


def _scale_edges(w, index, factor):
    """Multiply every entry whose index along any axis equals `index` by `factor` (once per such axis)."""
    w = w.copy()
    for ax in range(w.ndim):
        sl = [slice(None)] * w.ndim
        sl[ax] = index
        w[tuple(sl)] *= factor
    return w


def adjoint_reference(oracle, kind, g, dims):
    """A^T g from the oracle's forward transforms (FP64), with the weights of
    the adjoint relations:
      dft -> invdft (unnormalized; N x the reference's 1/N inverse off powers of two)
      invdft -> dft (1/N off powers of two)
      realdft -> invrealdft with the last axis's interior bins halved
      invrealdft -> realdft with the last axis's interior bins doubled
      dct2 -> dct3 with entry 0 doubled; dst2 -> dst3 with entry N-1 doubled
      dct3 -> dct2 with entry 0 halved;  dst3 -> dst2 with entry N-1 halved
      dct4, dst4 -> themselves                         (per axis for N-D)."""
    dims = tuple(dims)
    n = int(np.prod(dims))
    nd = len(dims) > 1
    pow2 = all(d & (d - 1) == 0 for d in dims)

    def T(k, v, shape=None):
        if nd:
            return oracle.nd(k, v, shape or dims)
        if k == "invrealdft":
            return oracle.invrealdft(v, dims[-1])
        return oracle.transform(k, v)

    g = np.asarray(g, dtype=np.complex128 if np.iscomplexobj(g) else np.float64)
    if kind == "dft":
        return T("invdft", g) * (1.0 if pow2 else n)
    if kind == "invdft":
        return T("dft", g) / (1.0 if pow2 else n)
    if kind == "realdft":
        w = g.copy()
        w[..., 1:-1] *= 0.5
        return T("invrealdft", w)
    if kind == "invrealdft":
        w = T("realdft", g)
        w[..., 1:-1] *= 2.0
        return w
    if kind == "dct2":
        return T("dct3", _scale_edges(g, 0, 2.0))
    if kind == "dst2":
        return T("dst3", _scale_edges(g, -1, 2.0))
    if kind == "dct3":
        return _scale_edges(T("dct2", g), 0, 0.5)
    if kind == "dst3":
        return _scale_edges(T("dst2", g), -1, 0.5)
    return T(kind, g)


def _forward_reference(oracle, kind, x, dims):
    if len(dims) > 1:
        return oracle.nd(kind, x, dims)
    if kind == "invrealdft":
        return oracle.invrealdft(x, dims[-1])
    return oracle.transform(kind, x)


def _shapes(kind, dims):
    ins = dims[:-1] + (dims[-1] // 2 + 1,) if kind == "invrealdft" else dims
    outs = dims[:-1] + (dims[-1] // 2 + 1,) if kind == "realdft" else dims
    return ins, outs


def _cplx_in(kind):
    return kind in ("dft", "invdft", "invrealdft")


def _cplx_out(kind):
    return kind in ("dft", "invdft", "realdft")


CASES = [(k, (1024,)) for k in ALL_KINDS] + [(k, (1 << 16,)) for k in ALL_KINDS] + \
        [("dft", (1000,)), ("invdft", (1000,)), ("dft", (4097,)), ("invdft", (4097,))] + \
        [(k, (16, 32)) for k in ALL_KINDS] + [(k, (8, 4, 16)) for k in ("dft", "realdft", "invrealdft", "dct2",
                                                                         "dst3", "dct4")]


@pytest.mark.parametrize("single", [False, True], ids=["double", "float"])
@pytest.mark.parametrize("kind,dims", CASES, ids=[f"{k}-{'x'.join(map(str, d))}" for k, d in CASES])
def test_adjoint_equals_oracle_on_cotangent(lib_d, lib_f, oracle_d, single, kind, dims):
    lib = lib_f if single else lib_d
    rng = np.random.default_rng(zlib.crc32(f"{kind}{dims}".encode()))
    _, outs = _shapes(kind, dims)
    if _cplx_out(kind):
        g = rng.uniform(-1, 1, outs) + 1j * rng.uniform(-1, 1, outs)
    else:
        g = rng.uniform(-1, 1, outs)
    g = g.astype(lib.cdt if _cplx_out(kind) else lib.rdt)
    with lib.mkaux(FAMILY[kind], list(dims)) as a:
        gx = a.vjp(kind, g)
    ref = adjoint_reference(oracle_d, kind, g, dims)
    lim = (1e-6 if single else 1e-13) * max(1.0, math.log2(int(np.prod(dims))))
    assert rel_l2(gx, ref) <= lim


@pytest.mark.parametrize("kind,dims", [(k, (256,)) for k in ALL_KINDS] + [("dft", (100,)), ("realdft", (8, 32)),
                                                                        ("dct3", (8, 16))])
def test_adjoint_fp64_central_differences(lib_d, oracle_d, kind, dims):
    """dL/dx for L(x) = <g, A x> by FP64 central differences (A evaluated by
    the oracle, h = 1e-3) on 24 random coordinates -- real and imaginary parts
    of complex inputs -- against the adjoint kernel's A^T g."""
    rng = np.random.default_rng(len(kind) * 1000 + int(np.prod(dims)))
    ins, outs = _shapes(kind, dims)
    x = rng.uniform(-1, 1, ins) + (1j * rng.uniform(-1, 1, ins) if _cplx_in(kind) else 0)
    g = rng.uniform(-1, 1, outs) + (1j * rng.uniform(-1, 1, outs) if _cplx_out(kind) else 0)

    def L(v):
        y = _forward_reference(oracle_d, kind, v, dims)
        return float(np.sum(np.real(g) * np.real(y)) + np.sum(np.imag(g) * np.imag(y)))

    with lib_d.mkaux(FAMILY[kind], list(dims)) as a:
        gx = a.vjp(kind, g)
    scale = np.sqrt(np.mean(np.abs(gx) ** 2))
    h = 1e-3
    flat = x.reshape(-1)
    for _ in range(24):
        i = int(rng.integers(flat.size))
        part = 1j if (_cplx_in(kind) and rng.random() < 0.5) else 1.0
        xp = flat.copy()
        xp[i] += h * part
        xm = flat.copy()
        xm[i] -= h * part
        fd = (L(xp.reshape(ins)) - L(xm.reshape(ins))) / (2 * h)
        got = gx.reshape(-1)[i]
        got = got.imag if part == 1j else got.real
        assert abs(got - fd) <= 1e-9 * scale, (i, part, got, fd)

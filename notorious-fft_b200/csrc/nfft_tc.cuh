// nfft_tc.cuh -- radix-16 sub-stages on the tensor cores (float library,
// NOTORIOUS_FFT_FORM_SPLIT_TC).
//
// A warp computes 8 radix-16 butterflies at a time as one matrix product
//   Y (16 x 8, complex) = F16 (16 x 16, complex) X (16 x 8, complex),
// F16[m][k] = e^{-2 pi i m k / 16}, with mma.sync.m16n8k16 (FP16 operands,
// FP32 accumulation).  Both operands are split into FP16 hi + lo parts and
// the product is accumulated from the three leading terms
//   Fhi Xhi + Fhi Xlo + Flo Xhi      (~22 significant bits),
// separately for Yr = Fr Xr - Fi Xi and Yi = Fi Xr + Fr Xi: 12 MMAs per 8
// butterflies.  Every butterfly (a column of X) is scaled by a power of two so
// that its largest component is just below 2^14 before the split, which keeps
// FP16 in range for any input magnitude; the scale is removed exactly from the
// FP32 outputs.  Twiddles and sums stay in FP32.
//
// Fragment layouts (PTX ISA, mma.m16n8k16 with .f16 A/B and .f32 C/D; lane =
// 4 g + t4):  A reg r holds rows g + 8 (r & 1), columns 2 t4 + 8 (r >> 1) + {0,1};
// B reg r holds rows (k) 2 t4 + 8 r + {0,1} of column g;  D holds rows
// g + 8 (r >> 1), columns 2 t4 + (r & 1).
#pragma once

#include <cuda_fp16.h>

#include "nfft_pass.cuh"

namespace nfft {

// Per-lane A fragments of F16: real / imaginary parts, hi / lo, and -Fi.
struct __align__(16) TcA {
    uint32_t rh[4], rl[4], ih[4], il[4], nih[4], nil[4];
};

NFFT_HD uint32_t tc_pack(__half lo16, __half hi16) {
    return (uint32_t)__half_as_ushort(lo16) | ((uint32_t)__half_as_ushort(hi16) << 16);
}

NFFT_HD void tc_split(float x, __half& hi, __half& lo) {
    hi = __float2half_rn(x);
    lo = __float2half_rn(x - __half2float(hi));
}

NFFT_HD void tc_make_A(int lane, TcA& A) {
    // cos / sin(2 pi j / 16), j = 0..15
    const float c16[16] = {1.0f, 0.92387953251128675613f, 0.70710678118654752440f, 0.38268343236508977173f,
                           0.0f, -0.38268343236508977173f, -0.70710678118654752440f, -0.92387953251128675613f,
                           -1.0f, -0.92387953251128675613f, -0.70710678118654752440f, -0.38268343236508977173f,
                           0.0f, 0.38268343236508977173f, 0.70710678118654752440f, 0.92387953251128675613f};
    const int g = lane >> 2, t4 = lane & 3;
    for (int r = 0; r < 4; ++r) {
        const int row = g + 8 * (r & 1);
        __half rh[2], rl[2], ih[2], il[2], nih[2], nil[2];
        for (int h = 0; h < 2; ++h) {
            const int col = 2 * t4 + 8 * (r >> 1) + h;
            const int j = (row * col) & 15;
            const float fr = c16[j];               // cos(2 pi j/16)
            const float fi = -c16[(j + 12) & 15];   // -sin(2 pi j/16) = -cos(2 pi (j - 4)/16)
            tc_split(fr, rh[h], rl[h]);
            tc_split(fi, ih[h], il[h]);
            tc_split(-fi, nih[h], nil[h]);
        }
        A.rh[r] = tc_pack(rh[0], rh[1]);
        A.rl[r] = tc_pack(rl[0], rl[1]);
        A.ih[r] = tc_pack(ih[0], ih[1]);
        A.il[r] = tc_pack(il[0], il[1]);
        A.nih[r] = tc_pack(nih[0], nih[1]);
        A.nil[r] = tc_pack(nil[0], nil[1]);
    }
}

// Power-of-two scale 2^(14 - e) for a butterfly whose largest component is
// amax = f 2^e, f in [0.5, 1); 1 for an all-zero butterfly.
NFFT_HD float tc_scale(float amax) {
    if (!(amax > 0.0f)) return 1.0f;
    int e;
    frexpf(amax, &e);
    int ex = 14 - e;
    if (ex > 126) ex = 126;
    if (ex < -126) ex = -126;
    return ldexpf(1.0f, ex);
}

// B fragments of one lane for its 4 points (k = 2 t4 + {0, 1, 8, 9} of
// column g), already twiddled and scaled.
struct TcB {
    uint32_t rh[2], rl[2], ih[2], il[2];
};
NFFT_HD void tc_make_B(const float2* x, TcB& B) {
    __half rh[4], rl[4], ih[4], il[4];
    for (int p = 0; p < 4; ++p) {
        tc_split(x[p].x, rh[p], rl[p]);
        tc_split(x[p].y, ih[p], il[p]);
    }
    for (int r = 0; r < 2; ++r) {
        B.rh[r] = tc_pack(rh[2 * r], rh[2 * r + 1]);
        B.rl[r] = tc_pack(rl[2 * r], rl[2 * r + 1]);
        B.ih[r] = tc_pack(ih[2 * r], ih[2 * r + 1]);
        B.il[r] = tc_pack(il[2 * r], il[2 * r + 1]);
    }
}

__device__ __forceinline__ void tc_mma(const uint32_t* a, const uint32_t* b, float* d) {
#if defined(__CUDA_ARCH__)
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
#endif
}

// The 12 products of one lane (warp-collective): Yr, Yi fragments (4 floats each).
__device__ __forceinline__ void tc_dft16_mma(const TcA& A, const TcB& B, float* yr, float* yi) {
#pragma unroll
    for (int r = 0; r < 4; ++r) yr[r] = yi[r] = 0.0f;
    // Yr = Fr Xr + (-Fi) Xi
    tc_mma(A.rl, B.rh, yr);
    tc_mma(A.rh, B.rl, yr);
    tc_mma(A.nil, B.ih, yr);
    tc_mma(A.nih, B.il, yr);
    tc_mma(A.rh, B.rh, yr);
    tc_mma(A.nih, B.ih, yr);
    // Yi = Fi Xr + Fr Xi
    tc_mma(A.il, B.rh, yi);
    tc_mma(A.ih, B.rl, yi);
    tc_mma(A.rl, B.ih, yi);
    tc_mma(A.rh, B.il, yi);
    tc_mma(A.ih, B.rh, yi);
    tc_mma(A.rh, B.ih, yi);
}

// Lane read phase of a tensor-core radix-16 sub-stage over a tile of
// 2^logE points in the row layout (spad), for butterfly group q of warp w:
// the lane's 4 points of butterfly 32 w + 8 q + g.
NFFT_HD void tc_read(const float2* sm, int logR, int lns, int w, int q, int lane, float2* x, int& l, int& i) {
    const int lq = logR - 4;
    const int g = lane >> 2, t4 = lane & 3;
    const int b = w * 32 + q * 8 + g;
    l = b >> lq;
    i = b & ((1 << lq) - 1);
    const int base = (l << logR) + i;
    const int ks[4] = {2 * t4, 2 * t4 + 1, 2 * t4 + 8, 2 * t4 + 9};
    for (int p = 0; p < 4; ++p) x[p] = sm[NFFT_SM(spad(base + (ks[p] << lq)))];
    (void)lns;
}

// Twiddle W_{ns 16}^{m k} of the lane's 4 input points (m = 2 t4 + {0,1,8,9}).
NFFT_HD void tc_twiddle(const TwTables<float>* tw, int lns, int i, int lane, float2* x) {
    if (lns == 0) return;
    const int k = i & ((1 << lns) - 1);
    if (!k) return;
    const int t4 = lane & 3;
    const int ks[4] = {2 * t4, 2 * t4 + 1, 2 * t4 + 8, 2 * t4 + 9};
    for (int p = 0; p < 4; ++p) {
        const float2 wv = (lns + 4 <= TW_BITS) ? twiddle_small<float>(tw, (uint32_t)(ks[p] * k), lns + 4)
                                               : twiddle<float>(tw, (uint64_t)(ks[p] * k), lns + 4);
        x[p] = cmul(x[p], wv);
    }
}

// Write phase: the lane's outputs yr/yi (rows g, g+8 of columns 2 t4, 2 t4+1
// of the group, already unscaled) to their Stockham positions.
NFFT_HD void tc_write(float2* sm, int logR, int lns, int w, int q, int lane, const float* yr, const float* yi) {
    const int lq = logR - 4;
    const int g = lane >> 2, t4 = lane & 3;
    for (int r = 0; r < 4; ++r) {
        const int m = g + 8 * (r >> 1);
        const int n = 2 * t4 + (r & 1);
        const int b = w * 32 + q * 8 + n;
        const int l = b >> lq, i = b & ((1 << lq) - 1);
        const int k = i & ((1 << lns) - 1);
        const int o = (l << logR) + ((i >> lns) << (lns + 4)) + k + (m << lns);
        sm[NFFT_SM(spad(o))] = make_float2(yr[r], yi[r]);
    }
}

// Scale 2^(14 - e) from the exponent bits of amax (amax = f 2^e, f in
// [0.5, 1)) and its exact reciprocal; 1 for amax == 0.  Same values as
// tc_scale.
__device__ __forceinline__ void tc_scale_bits(float amax, float& sc, float& inv) {
    const int E = (__float_as_int(amax) >> 23) & 0xff;
    int f = (amax > 0.0f) ? 267 - E : 127;
    f = min(max(f, 1), 253);
    sc = __int_as_float(f << 23);
    inv = __int_as_float((254 - f) << 23);
}

// B fragments with packed f16x2 conversions (bit-identical to tc_make_B).
__device__ __forceinline__ void tc_make_B_fast(const float2* x, TcB& B) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const float2 a = x[2 * r], b = x[2 * r + 1];
        __half2 rh = __floats2half2_rn(a.x, b.x);
        __half2 ih = __floats2half2_rn(a.y, b.y);
        const float2 rb = __half22float2(rh), ib = __half22float2(ih);
        __half2 rl = __floats2half2_rn(a.x - rb.x, b.x - rb.y);
        __half2 il = __floats2half2_rn(a.y - ib.x, b.y - ib.y);
        B.rh[r] = *(uint32_t*)&rh;
        B.ih[r] = *(uint32_t*)&ih;
        B.rl[r] = *(uint32_t*)&rl;
        B.il[r] = *(uint32_t*)&il;
    }
}

// One tensor-core radix-16 sub-stage over a row-layout tile of 2^logE points
// (butterflies = 2^(logE-4) = 8 * 4 * warps; a warp takes 4 groups of 8).
// All four groups' fragments are formed first, then the 48 MMAs run as 16
// independent accumulation chains (hi-hi and cross terms of Yr / Yi per
// group), then the outputs are unscaled and stored.
template <int THREADS>
__device__ __forceinline__ void tc_substage(float2* sm, const TwTables<float>* tw, const TcA& A, int logR, int logE,
                                            int lns, int tid) {
    const int lane = tid & 31, w = tid >> 5;
    const int t4 = lane & 3;
    float2 x[4][4];
    int ls[4], is[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) tc_read(sm, logR, lns, w, q, lane, x[q], ls[q], is[q]);
    __syncthreads();
    TcB B[4];
    float u0[4], u1[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        tc_twiddle(tw, lns, is[q], lane, x[q]);
        float amax = 0.f;
#pragma unroll
        for (int p = 0; p < 4; ++p) amax = fmaxf(amax, fmaxf(fabsf(x[q][p].x), fabsf(x[q][p].y)));
        amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, 1));
        amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, 2));
        float sc, inv;
        tc_scale_bits(amax, sc, inv);
#pragma unroll
        for (int p = 0; p < 4; ++p) x[q][p] = make_float2(x[q][p].x * sc, x[q][p].y * sc);
        tc_make_B_fast(x[q], B[q]);
        // output columns 2 t4, 2 t4 + 1 carry the scales of butterflies held by lanes 8 t4, 8 t4 + 4
        u0[q] = __shfl_sync(0xffffffffu, inv, 8 * t4);
        u1[q] = __shfl_sync(0xffffffffu, inv, 8 * t4 + 4);
    }
    float yr[4][4], yi[4][4], cr[4][4], ci[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) yr[q][r] = yi[q][r] = cr[q][r] = ci[q][r] = 0.f;
    // cross terms (small) and main terms in separate chains, groups interleaved
#pragma unroll
    for (int q = 0; q < 4; ++q) { tc_mma(A.rl, B[q].rh, cr[q]); tc_mma(A.il, B[q].rh, ci[q]); }
#pragma unroll
    for (int q = 0; q < 4; ++q) { tc_mma(A.rh, B[q].rh, yr[q]); tc_mma(A.ih, B[q].rh, yi[q]); }
#pragma unroll
    for (int q = 0; q < 4; ++q) { tc_mma(A.rh, B[q].rl, cr[q]); tc_mma(A.ih, B[q].rl, ci[q]); }
#pragma unroll
    for (int q = 0; q < 4; ++q) { tc_mma(A.nih, B[q].ih, yr[q]); tc_mma(A.rh, B[q].ih, yi[q]); }
#pragma unroll
    for (int q = 0; q < 4; ++q) { tc_mma(A.nil, B[q].ih, cr[q]); tc_mma(A.rl, B[q].ih, ci[q]); }
#pragma unroll
    for (int q = 0; q < 4; ++q) { tc_mma(A.nih, B[q].il, cr[q]); tc_mma(A.rh, B[q].il, ci[q]); }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float orr[4], oi[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const float u = (r & 1) ? u1[q] : u0[q];
            orr[r] = (yr[q][r] + cr[q][r]) * u;
            oi[r] = (yi[q][r] + ci[q][r]) * u;
        }
        tc_write(sm, logR, lns, w, q, lane, orr, oi);
    }
    __syncthreads();
}

}  // namespace nfft

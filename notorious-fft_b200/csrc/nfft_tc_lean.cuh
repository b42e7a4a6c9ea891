// nfft_tc_lean.cuh -- radix-256 Stockham passes of the split tensor-core form
// (float library, NOTORIOUS_FFT_FORM_SPLIT_TC), the specialized kernel.
//
// A CTA owns a tile of 16 Stockham lines x 256 points.  The tile is staged
// through shared memory with coalesced global accesses on both sides; in
// between, every warp turns its lines over entirely in registers:
//
//   radix 256 = 16 x 16:  r = b + 16 a,  r_out = k1 + 16 k2
//   stage 1   Y[k1][b]  = sum_a F[k1][a] X[a][b]            (16 DFT-16s over a)
//   twiddle   U[k1][b]  = Y[k1][b] W_256^{b k1}
//   stage 2   Z[k2][k1] = sum_b F[k2][b] U[b][k1]            (16 DFT-16s over b)
//   output    V[k1 + 16 k2] = Z[k2][k1]
//
// with F[m][k] = W_16^{m k}.  Each stage is one complex 16 x 16 by 16 x 16
// product on the tensor cores, mma.sync.m16n8k16 with FP16 operands and FP32
// accumulation: [Yr; Yi] = [[Fr, -Fi], [Fi, Fr]] [Xr; Xi], both operands split
// into FP16 hi + lo parts and the three leading terms Fhi Xhi + Fhi Xlo +
// Flo Xhi accumulated (~22 significant bits): 2 x 2 x 2 x 3 = 24 MMAs per
// stage per line.  F is the A operand and the data the B operand, so the
// accumulator of stage 1 (rows k1, columns b) already sits in exactly the
// registers that stage 2's B operand (rows b, columns k1) needs: no exchange
// between the stages, only the twiddle and the FP16 split in FP32 registers.
//
// Range: before the split every line is scaled by a power of two so that its
// largest component lies in [2^9, 2^10); stage-1 outputs then stay below
// 16 sqrt(2) 2^10 < 2^15 (FP16 holds up to 65504), and the FP32 stage-2
// outputs are unscaled exactly.  Lo parts below 2^-14 lose relative precision
// as FP16 subnormals, but their absolute error (2^-25) is far below the line's
// rounding level.  Pass pre-twiddles, the internal twiddle and all sums stay
// in FP32 (twiddles from the FP64-generated tables).
//
// Fragment layouts (PTX ISA, mma.m16n8k16, .f16 A/B, .f32 C/D; lane = 4 g + q):
//   A reg i: row g + 8 (i & 1), columns 2q + 8 (i >> 1) + {0, 1}
//   B reg i: rows 2q + 8 i + {0, 1}, column g
//   D reg i: row g + 8 (i >> 1), column 2q + (i & 1)
// So a lane holds the points a = 2q + {0, 1, 8, 9} of butterflies b = g and
// g + 8 going in, and r_out = k1 + 16 k2 for k1 = 2q + {0, 1, 8, 9}, k2 = g,
// g + 8 coming out.
//
// Shared tile: slot (r, l) of line l's point r at r * 16 + (l ^ S(r)), with the
// 4-bit swizzle S(r) = (r0 ^ r4, r1, r2, r3 ^ r5) (r_k: bit k of r).  Every
// access pattern of the kernel -- fragment reads (lanes vary r bits 0-2 and
// 5-6), fragment writes (bits 1-2 and 4-6), column-mode rows (l varies) and
// row-mode runs (bits 0-4) -- touches each of the 16 8-byte bank pairs exactly
// twice per 32 lanes, the minimum of two wavefronts for 256 bytes.
#pragma once

#include <cuda_fp16.h>
#include <string.h>

#include "nfft_tc.cuh"

namespace nfft {

constexpr int TCL_LOGR = 8;
constexpr int TCL_R = 1 << TCL_LOGR;
constexpr int TCL_LOGJ = 4;
constexpr int TCL_J = 1 << TCL_LOGJ;
constexpr int TCL_SLOTS = TCL_R * TCL_J;

NFFT_HD int tcl_slot(int r, int l) {
    const int s = ((r ^ (r >> 4)) & 1) | (r & 6) | ((((r >> 5) ^ (r >> 3)) & 1) << 3);
    return (r << TCL_LOGJ) | (l ^ s);
}

// Two tile buffers, two sets of line offsets, and the per-lane constants
// (F fragments and internal twiddles, 32 lanes; see TcLean::Consts).
constexpr size_t TCL_CONSTS_BYTES = 32 * 176;
template <int THREADS>
constexpr size_t tcl_smem_bytes() {
    return 2 * (sizeof(float2) * (size_t)TCL_SLOTS + sizeof(long long) * 3 * (size_t)TCL_J) + TCL_CONSTS_BYTES;
}

NFFT_HD uint32_t tcl_pack(float lo16, float hi16) {
    // cvt.rn.f16x2.f32 packs its first operand into the upper half
#if defined(__CUDA_ARCH__)
    uint32_t r;
    asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi16), "f"(lo16));
    return r;
#else
    return tc_pack(__float2half_rn(lo16), __float2half_rn(hi16));
#endif
}

// hi / lo FP16 pairs of two FP32 values (x0 in the low half)
NFFT_HD void tcl_split2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
    hi = tcl_pack(x0, x1);
#if defined(__CUDA_ARCH__)
    const __half2 h = *reinterpret_cast<const __half2*>(&hi);
    const float2 hf = __half22float2(h);
#else
    const float2 hf = make_float2(__half2float(__ushort_as_half((unsigned short)(hi & 0xffff))),
                                  __half2float(__ushort_as_half((unsigned short)(hi >> 16))));
#endif
    lo = tcl_pack(x0 - hf.x, x1 - hf.y);
}

NFFT_HD void tcl_mma(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
#if defined(__CUDA_ARCH__)
    asm(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
#else
    (void)d; (void)a; (void)b0; (void)b1;
#endif
}
// d = a b (zero accumulator)
NFFT_HD void tcl_mma0(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
#if defined(__CUDA_ARCH__)
    asm(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%10, %10, %10, %10};"
        : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(0.0f));
#else
    (void)a; (void)b0; (void)b1;
    d[0] = d[1] = d[2] = d[3] = 0.0f;
#endif
}

// The three terms of block (ah, al) times x (small ones first), into d.
NFFT_HD void tcl_terms(float* d, const uint32_t* ah, const uint32_t* al, const uint32_t (&x)[2][2], bool first) {
    if (first) tcl_mma0(d, al, x[0][0], x[0][1]);
    else tcl_mma(d, al, x[0][0], x[0][1]);
    tcl_mma(d, ah, x[1][0], x[1][1]);
    tcl_mma(d, ah, x[0][0], x[0][1]);
}
// One complex 16 x 16 product on the tensor cores: acc[mt][nt][i] =
// ([[Fr, -Fi], [Fi, Fr]] [Xr; Xi]) with B fragments xb[kt][nt][hi/lo][reg],
// walking the A blocks (Fr, then -Fi, then Fi) so that each is read once.
NFFT_HD void tcl_stage(const TcA& A, const uint32_t (&xb)[2][2][2][2], float (&acc)[2][2][4]) {
    {
        uint32_t h[4], l[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) { h[i] = A.rh[i]; l[i] = A.rl[i]; }
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
            tcl_terms(acc[0][nt], h, l, xb[0][nt], true);    // Yr  = Fr Xr
            tcl_terms(acc[1][nt], h, l, xb[1][nt], true);    // Yi  = Fr Xi
        }
    }
    {
        uint32_t h[4], l[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) { h[i] = A.nih[i]; l[i] = A.nil[i]; }
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) tcl_terms(acc[0][nt], h, l, xb[1][nt], false);   // Yr -= Fi Xi
    }
    {
        uint32_t h[4], l[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) { h[i] = A.ih[i]; l[i] = A.il[i]; }
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) tcl_terms(acc[1][nt], h, l, xb[0][nt], false);   // Yi += Fi Xr
    }
}

// W_{2^logP}^q for logP <= 24 from two table levels, without branches
// (T1[0] = 1 exactly): every lane of a warp takes the same path.
template <typename T>
NFFT_HD C2<T> tcl_twiddle(const TwTables<T>* tw, uint64_t q, int logP) {
    const uint64_t u = (q << (36 - logP)) & ((1ull << 36) - 1);
    return cmul(tw_load<T>(tw, 0, (uint32_t)(u >> 24)), tw_load<T>(tw, 1, (uint32_t)(u >> 12) & (TW_SIZE - 1)));
}

// Exponent s with m 2^s in [2^9, 2^10) for the largest component m of a line,
// read from the bits of m; 0 for m = 0, non-finite m or a subnormal m (a line
// that small is below any rounding level of the transform).
NFFT_HD int tcl_scale_exp(float m) {
#if defined(__CUDA_ARCH__)
    const int bits = __float_as_int(m);
#else
    int bits;
    memcpy(&bits, &m, sizeof bits);
#endif
    const int em = (bits >> 23) & 0xff;   // m in [2^(em-127), 2^(em-126))
    if (em == 0 || em == 255) return 0;
    int s = 136 - em;
    return s > 120 ? 120 : (s < -120 ? -120 : s);
}
// 2^s for |s| <= 126, exactly.
NFFT_HD float tcl_pow2(int s) {
    const int bits = (127 + s) << 23;
#if defined(__CUDA_ARCH__)
    return __int_as_float(bits);
#else
    float f;
    memcpy(&f, &bits, sizeof f);
    return f;
#endif
}

// Tile slot e (0 <= e < 16 x 256) of a load or store walk -> (line l, point r):
// lines fastest in column mode (16 adjacent lines make 128-byte rows), points
// fastest in row mode (each line one contiguous run).
NFFT_HD void tcl_walk(int row_mode, int e, int& l, int& r) {
    l = row_mode ? (e >> TCL_LOGR) : (e & (TCL_J - 1));
    r = row_mode ? (e & (TCL_R - 1)) : (e >> TCL_LOGJ);
}
// Element offsets (float2 units) of input point r and output point r of a line
// (bin / bout / j from line_setup): the Stockham pass layout.
NFFT_HD long long tcl_in_off(const PassArgs& a, long long bin, long long j, int r) {
    return bin + j * a.in_estride + (long long)r * (a.in_estride << a.logNj);
}
NFFT_HD long long tcl_out_off(const PassArgs& a, long long bout, long long j, int r) {
    const int logNso = a.logNs_out;
    const long long base = ((j >> logNso) << (logNso + TCL_LOGR)) + (j & ((1ll << logNso) - 1));
    return bout + base * a.out_estride + (long long)r * (a.out_estride << logNso);
}

// p[off] for p pointing into the shared tile sm (the emulator checks the
// absolute slot (p - sm) + off).
template <typename V>
NFFT_HD V& tcl_at(V* sm, V* p, int off) {
    (void)NFFT_SM((int)(p - sm) + off);
    return p[off];
}
template <typename V>
NFFT_HD const V& tcl_at(const V* sm, const V* p, int off) {
    (void)NFFT_SM((int)(p - sm) + off);
    return p[off];
}

// Swizzle of tile row r (see tcl_slot).
NFFT_HD int tcl_swz(int r) { return ((r ^ (r >> 4)) & 1) | (r & 6) | ((((r >> 5) ^ (r >> 3)) & 1) << 3); }

template <int THREADS>
struct TcLean {
    static constexpr int WARPS = THREADS / 32;
    static_assert(TCL_J % WARPS == 0, "lines per warp");
    static constexpr int LPW = TCL_J / WARPS;
    static constexpr int PER_THREAD = TCL_SLOTS / THREADS;

    // Per-lane constants: F fragments and the internal twiddles W_256^{b k1}
    // of the lane's stage-1 outputs (k1 = g + 8 (i >> 1), b = 2q + (i & 1) + 8 nt).
    // The kernel keeps them in shared memory (one copy per CTA, read where
    // used), which leaves registers for a third CTA per SM.
    struct __align__(16) Consts {
        TcA A;
        float2 itw[2][4];
        uint32_t pad[4];   // 176-byte stride (11 x 16): the lanes' 16-byte reads of a
                           // quarter warp fall on 8 distinct bank groups
    };
    static_assert(32 * sizeof(Consts) <= TCL_CONSTS_BYTES, "constants table");

    static NFFT_HD void setup(const TwTables<float>* tw, int lane, Consts& c) {
        tc_make_A(lane, c.A);
        const int g = lane >> 2, q = lane & 3;
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int k1 = g + 8 * (i >> 1), b = 2 * q + (i & 1) + 8 * nt;
                c.itw[nt][i] = twiddle_small<float>(tw, (uint32_t)((k1 * b) & 255), 8);
            }
    }

    // Point r of the lane's B fragment slot: kt-independent; (nt, reg i, half h)
    // -> a = 2q + 8 i + h, b = g + 8 nt.
    static NFFT_HD int in_point(int lane, int nt, int i, int h) {
        const int g = lane >> 2, q = lane & 3;
        return (g + 8 * nt) + 16 * (2 * q + 8 * i + h);
    }
    // Output point of accumulator (nt, i): k2 = g + 8 (i >> 1), k1 = 2q + (i & 1) + 8 nt.
    static NFFT_HD int out_point(int lane, int nt, int i) {
        const int g = lane >> 2, q = lane & 3;
        return (2 * q + (i & 1) + 8 * nt) + 16 * (g + 8 * (i >> 1));
    }

    // A line's registers between the phases below.  The kernel runs the
    // phases in order for one line per warp; the warp-collective steps (the
    // max reduction and the two MMA stages) sit between them, so the CPU
    // emulator can run the same lane phases around its own collectives.
    struct LineRegs {
        float2 x[2][2][2];         // [nt][i][h]: points b = g + 8 nt, a = 2q + 8 i + h
        uint32_t xb[2][2][2][2];   // B fragments [kt: re / im][nt][hi / lo][reg]
        float acc[2][2][4];        // accumulators [mt: re / im][nt][reg]
        int e;                     // scale exponent of the line
    };

    // Shared slots of the lane's fragment points on line l.  With the bits of
    // r_in = b + 16 a (g: bits 0-2, nt: 3, h: 4, q: 5-6, i: 7) the swizzle is
    // S = g ^ h ^ ((nt ^ q0) << 3), so slot = ((g + 32 q) << 4) + (l ^ g ^ (q0 << 3))
    // ^ (h | nt << 3), plus the compile-time row offset ((8 nt + 16 h + 128 i) << 4).
    // Coming out, r_out = k1 + 16 k2 has (i & 1): bit 0, q: 1-2, nt: 3, g: 4-6,
    // i >> 1: 7, so S = (i & 1) ^ g0 ^ (q << 1) ^ ((nt ^ g1) << 3).
    static NFFT_HD int in_slot(int lane, int l, int nt, int i, int h) {
        const int g = lane >> 2, q = lane & 3;
        return (((g + 32 * q) << 4) + (((8 * nt + 16 * h + 128 * i)) << 4)) +
               ((l ^ g ^ ((q & 1) << 3)) ^ (h | (nt << 3)));
    }
    static NFFT_HD int out_slot(int lane, int l, int nt, int i) {
        const int g = lane >> 2, q = lane & 3;
        return (((2 * q + 16 * g) << 4) + (((i & 1) + 8 * nt + 128 * (i >> 1)) << 4)) +
               ((l ^ (g & 1) ^ (q << 1) ^ (((g >> 1) & 1) << 3)) ^ ((i & 1) | (nt << 3)));
    }

    // Phase 1: the lane's 8 points from shared memory (conjugated for an
    // inverse transform's first pass), pass pre-twiddle
    // W_{Ns R}^{r k} (k = j mod Ns, r = b + 16 a: W^{b k} per butterfly times
    // (W^{16 k})^a per point).  Returns the lane's largest component.
    static NFFT_HD float load(const PassArgs& a, const TwTables<float>* tw, const float2* sm, int l, long long j,
                              int lane, LineRegs& s) {
        // slot = base + (lx ^ (h | nt << 3)) + ((8 nt + 16 h + 128 i) << 4): four
        // base pointers per line, the rest compile-time offsets
        const int g = lane >> 2, q = lane & 3;
        const float2* base = sm + ((g + 32 * q) << 4);
        const int lx = l ^ g ^ ((q & 1) << 3);
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float2* p = base + (lx ^ (h | (nt << 3)));
#pragma unroll
                for (int i = 0; i < 2; ++i) s.x[nt][i][h] = tcl_at(sm, p, (8 * nt + 16 * h + 128 * i) << 4);
            }
        if (a.conj_in) {
#pragma unroll
            for (int nt = 0; nt < 2; ++nt)
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int h = 0; h < 2; ++h) s.x[nt][i][h].y = -s.x[nt][i][h].y;
        }
        if (a.logNs > 0) {
            // the per-point factor (W_P^{16 k})^a = W_{P/16}^{a k} (P = Ns R);
            // the per-butterfly factor W_P^{b k} joins the internal twiddle (mid).
            // k < 2^logNs <= 2^16 and a < 16: 32-bit products.
            const uint32_t k = (uint32_t)j & ((1u << a.logNs) - 1);
            const int logQ = a.logNs + 4;
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t e = (uint32_t)(2 * q + 8 * i + h) * k;
                    const float2 v = logQ <= TW_BITS ? twiddle_small<float>(tw, e, logQ)
                                                     : tcl_twiddle<float>(tw, (uint64_t)e, logQ);
                    s.x[0][i][h] = cmul(s.x[0][i][h], v);
                    s.x[1][i][h] = cmul(s.x[1][i][h], v);
                }
        }
        float m = 0.0f;
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int h = 0; h < 2; ++h) m = fmaxf(m, fmaxf(fabsf(s.x[nt][i][h].x), fabsf(s.x[nt][i][h].y)));
        return m;
    }

    // Phase 2: the line's power-of-two scale (m = its largest component) and
    // the split into stage 1's B fragments.  A line whose largest component
    // is already in [1, 2^10) is not scaled: FP16 holds its stage-1 outputs
    // (< 16 sqrt(2) 2^10) and the lo parts keep an absolute floor of 2^-25,
    // far below such a line's rounding level.
    static NFFT_HD void split1(float m, LineRegs& s) {
        s.e = (m >= 1.0f && m < 1024.0f) ? 0 : tcl_scale_exp(m);
        if (s.e != 0) {
            const float sc = tcl_pow2(s.e);
#pragma unroll
            for (int nt = 0; nt < 2; ++nt)
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int h = 0; h < 2; ++h) s.x[nt][i][h] = mkc(s.x[nt][i][h].x * sc, s.x[nt][i][h].y * sc);
        }
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                tcl_split2(s.x[nt][i][0].x, s.x[nt][i][1].x, s.xb[0][nt][0][i], s.xb[0][nt][1][i]);
                tcl_split2(s.x[nt][i][0].y, s.x[nt][i][1].y, s.xb[1][nt][0][i], s.xb[1][nt][1][i]);
            }
    }

    // Phase 3: the twiddle of the stage-1 accumulators, W_256^{b k1} times,
    // after the first pass, the per-butterfly part W_P^{b k} of the pass
    // pre-twiddle (k = j mod Ns, P = Ns R; b = 2q + (i & 1) + 8 nt here), then
    // stage 2's B fragments: B2[kt][nt2] reg 0 = (b = 2q, 2q+1) from n-tile 0,
    // reg 1 = (b = 2q+8, 2q+9) from n-tile 1, both at k1 = g + 8 nt2
    // (accumulator regs 2 nt2 + {0, 1}).
    static NFFT_HD void mid(const PassArgs& a, const TwTables<float>* tw, const Consts& c, long long j, int lane,
                            LineRegs& s) {
        float2 t[2][4];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int i = 0; i < 4; ++i) t[nt][i] = c.itw[nt][i];
        if (a.logNs > 0) {
            const uint32_t k = (uint32_t)j & ((1u << a.logNs) - 1);
            const int logP = a.logNs + TCL_LOGR, q = lane & 3;
            float2 w[2][2];   // W_P^{b k}, b = 2q + h + 8 nt
            w[0][0] = tcl_twiddle<float>(tw, (uint64_t)((uint32_t)(2 * q) * k), logP);
            const float2 s1 = tcl_twiddle<float>(tw, (uint64_t)k, logP);
            const float2 s8 = tcl_twiddle<float>(tw, (uint64_t)(8u * k), logP);
            w[0][1] = cmul(w[0][0], s1);
            w[1][0] = cmul(w[0][0], s8);
            w[1][1] = cmul(w[1][0], s1);
#pragma unroll
            for (int nt = 0; nt < 2; ++nt)
#pragma unroll
                for (int i = 0; i < 4; ++i) t[nt][i] = cmul(t[nt][i], w[nt][i & 1]);
        }
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float2 u = cmul(mkc(s.acc[0][nt][i], s.acc[1][nt][i]), t[nt][i]);
                s.acc[0][nt][i] = u.x;
                s.acc[1][nt][i] = u.y;
            }
#pragma unroll
        for (int kt = 0; kt < 2; ++kt)
#pragma unroll
            for (int nt2 = 0; nt2 < 2; ++nt2)
#pragma unroll
                for (int reg = 0; reg < 2; ++reg)
                    tcl_split2(s.acc[kt][reg][2 * nt2], s.acc[kt][reg][2 * nt2 + 1], s.xb[kt][nt2][0][reg],
                               s.xb[kt][nt2][1][reg]);
    }

    // Phase 4: unscale (with the pass's output factor and conjugation) into
    // the line's shared slots, in place.  slot = base + (lx ^ ((i & 1) | nt << 3))
    // + (((i & 1) + 8 nt + 128 (i >> 1)) << 4).
    static NFFT_HD void store(const PassArgs& a, float2* sm, int l, int lane, const LineRegs& s) {
        const int g = lane >> 2, q = lane & 3;
        float2* base = sm + ((2 * q + 16 * g) << 4);
        const int lx = l ^ (g & 1) ^ (q << 1) ^ (((g >> 1) & 1) << 3);
        const bool plain = s.e == 0 && a.scale == 1.0 && !a.conj_out;
        const float f = (float)a.scale * tcl_pow2(-s.e);
        const float fi = a.conj_out ? -f : f;
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                float2* p = base + (lx ^ (c | (nt << 3)));
#pragma unroll
                for (int hi = 0; hi < 2; ++hi) {
                    const int i = c + 2 * hi;
                    const int off = (c + 8 * nt + 128 * hi) << 4;
                    const float2 v = plain ? mkc(s.acc[0][nt][i], s.acc[1][nt][i])
                                           : mkc(s.acc[0][nt][i] * f, s.acc[1][nt][i] * fi);
                    tcl_at(sm, p, off) = v;
                }
            }
    }

#if defined(__CUDA_ARCH__)
    // One line of the tile (shared slots of line l), in place; the whole warp.
    static __device__ __forceinline__ void line(const PassArgs& a, const TwTables<float>* tw, const Consts& c,
                                                float2* sm, int l, long long j, int lane) {
        LineRegs s;
        float m = load(a, tw, sm, l, j, lane, s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        split1(m, s);
        tcl_stage(c.A, s.xb, s.acc);
        mid(a, tw, c, j, lane, s);
        tcl_stage(c.A, s.xb, s.acc);
        store(a, sm, l, lane, s);
    }
#endif
};


// Store with an L2 policy (one instruction; the policy encodes the pass's
// hint: evict_first for user data, evict_last for kept scratch).
__device__ __forceinline__ void tcl_st(float2* p, float2 v, uint64_t pol) {
#if defined(__CUDA_ARCH__)
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x), "f"(v.y), "l"(pol)
                 : "memory");
#endif
}

// Two adjacent points in one 16-byte store (p 16-byte aligned).
__device__ __forceinline__ void tcl_st2(float2* p, float2 v0, float2 v1, uint64_t pol) {
#if defined(__CUDA_ARCH__)
    asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(v0.x), "f"(v0.y), "f"(v1.x),
                 "f"(v1.y), "l"(pol)
                 : "memory");
#endif
}

// 8-byte asynchronous copy global -> shared (shared-window address dst).
__device__ __forceinline__ void tcl_cp8s(uint32_t dst, const float2* src, uint64_t pol) {
#if defined(__CUDA_ARCH__)
    asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "l"(pol)
                 : "memory");
#endif
}

// The pipeline of a persistent CTA over 16-line tiles, with two shared
// buffers: the copies of tile k+1 are in flight while tile k is transformed
// and written out.
//  lines()    the first 16 threads resolve a tile's lines once: offset of
//             point 0 on each side, or -1 past the last line, and j;
//  prefetch() every thread issues its 16 asynchronous copies.  Column mode
//             (16 adjacent lines make 128-byte rows): thread t copies line
//             t & 15, points (t >> 4) + 16 it.  Row mode (each line one run):
//             thread t copies point t of every line.  Slot (r0 + 16 it, l)
//             sits at (r0 << 4) + (it << 8) + ((l ^ S(r0)) ^ c_it), c_it =
//             (it & 1) | (it & 2) << 2: one XOR per element against a
//             per-thread constant;
//  compute()  every warp transforms its lines in place;
//  writeout() the tile written once with the matching walk of the output side.
template <int THREADS>
struct TcPipe {
    using TL = TcLean<THREADS>;
    static_assert(THREADS == TCL_R, "one thread per point of a line in the row walks");

    static __device__ __forceinline__ void lines(const PassArgs& a, long long tile, long long* lb) {
        const int t = threadIdx.x;
        if (t < TCL_J) {
            long long bin, bout, j;
            const long long lam = (tile << TCL_LOGJ) + t;
            if (a.ndims == 2 && a.jpos == 0 && a.cnt[0] == (1ll << a.logNj) && !a.in_tab && !a.out_tab) {
                // j innermost over the 2^logNj lines of a transform, one batch
                // dimension: shifts instead of the generic divisions
                const long long bt = lam >> a.logNj;
                j = lam < a.nlines ? (lam & (a.cnt[0] - 1)) : -1;
                bin = bt * a.istr[1];
                bout = bt * a.ostr[1];
            } else {
                line_setup(a, lam, 0, TileLines{&bin, &bout, &j});
            }
            const int logNso = a.logNs_out;
            const long long base = ((j >> logNso) << (logNso + TCL_LOGR)) + (j & ((1ll << logNso) - 1));
            lb[t] = j < 0 ? -1 : bin + j * a.in_estride;
            lb[TCL_J + t] = j < 0 ? -1 : bout + base * a.out_estride;
            lb[2 * TCL_J + t] = j;
        }
    }

    static __device__ __forceinline__ void prefetch(const PassArgs& a, const long long* lb, float2* buf, uint64_t pol) {
        const int t = threadIdx.x;
        const float2* in = (const float2*)a.in;
        const long long irs = a.in_estride << a.logNj;
        if (!a.in_row) {
            const int l = t & (TCL_J - 1), r0 = t >> TCL_LOGJ;
            const long long b = lb[l];
            const int sx = l ^ tcl_swz(r0);
            float2* sp = buf + (r0 << TCL_LOGJ);
            if (b < 0) {
#pragma unroll
                for (int k = 0; k < TCL_J; ++k) sp[(k << 8) + (sx ^ ((k & 1) | ((k & 2) << 2)))] = mkc(0.0f, 0.0f);
                return;
            }
            // four shared bases (sx ^ c, c in {0, 1, 8, 9}) plus immediates
            const uint32_t s0 = (uint32_t)__cvta_generic_to_shared(sp);
            const uint32_t sa[4] = {s0 + ((uint32_t)(sx ^ 0) << 3), s0 + ((uint32_t)(sx ^ 1) << 3),
                                    s0 + ((uint32_t)(sx ^ 8) << 3), s0 + ((uint32_t)(sx ^ 9) << 3)};
            const float2* gp = in + b + r0 * irs;
            const long long st = (long long)TCL_J * irs;
#pragma unroll
            for (int k = 0; k < TCL_J; ++k) {
                tcl_cp8s(sa[(k & 1) | (k & 2)] + ((uint32_t)k << 11), gp, pol);
                gp += st;
            }
        } else {
            const int r = t, sr = tcl_swz(r);
            float2* sp = buf + (r << TCL_LOGJ);
            const uint32_t s0 = (uint32_t)__cvta_generic_to_shared(sp);
            const long long roff = r * irs;
#pragma unroll
            for (int k = 0; k < TCL_J; ++k) {
                const long long b = lb[k];
                if (b < 0) sp[k ^ sr] = mkc(0.0f, 0.0f);
                else tcl_cp8s(s0 + ((uint32_t)(k ^ sr) << 3), in + b + roff, pol);
            }
        }
    }

    static __device__ __forceinline__ void compute(const PassArgs& a, const typename TL::Consts& c, const long long* lb,
                                                   float2* buf) {   // c: this lane's constants (shared)
        const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
        const TwTables<float>* tw = (const TwTables<float>*)a.tw;
#pragma unroll 1
        for (int k = 0; k < TL::LPW; ++k) {
            const int l = warp + k * TL::WARPS;
            const long long j = lb[2 * TCL_J + l];
            if (j >= 0) TL::line(a, tw, c, buf, l, j, lane);
        }
    }

    static __device__ __forceinline__ void writeout(const PassArgs& a, const long long* lb, const float2* buf,
                                                    uint64_t pol) {
        const int t = threadIdx.x;
        float2* out = (float2*)a.out;
        const long long ors = a.out_estride << a.logNs_out;
        if (!a.out_row) {
            const int l = t & (TCL_J - 1), r0 = t >> TCL_LOGJ;
            const long long b = lb[TCL_J + l];
            if (b < 0) return;
            const int sx = l ^ tcl_swz(r0);
            const float2* sp = buf + (r0 << TCL_LOGJ);
            const float2* sc[4] = {sp + (sx ^ 0), sp + (sx ^ 1), sp + (sx ^ 8), sp + (sx ^ 9)};
            float2* gp = out + b + r0 * ors;
            const long long st = (long long)TCL_J * ors;
#pragma unroll
            for (int k = 0; k < TCL_J; ++k) {
                tcl_st(gp, sc[(k & 1) | (k & 2)][k << 8], pol);
                gp += st;
            }
        } else {
            // point pairs (2p, 2p + 1) of lines l = (t >> 7) + 2 it: 16-byte
            // stores when the line starts on a pair boundary.  S(2p + 1) = S(2p) ^ 1.
            const int pp = t & 127, r = 2 * pp, s2 = tcl_swz(r);
            const float2* sp0 = buf + (r << TCL_LOGJ);
            const float2* sp1 = sp0 + TCL_J;
#pragma unroll
            for (int it = 0; it < TCL_J / 2; ++it) {
                const int l = (t >> 7) + 2 * it;
                const long long b = lb[TCL_J + l];
                if (b < 0) continue;
                const float2 v0 = sp0[l ^ s2], v1 = sp1[l ^ s2 ^ 1];
                float2* gp = out + b + r * ors;
                if (ors == 1 && (((uintptr_t)gp) & 15) == 0) tcl_st2(gp, v0, v1, pol);
                else {
                    tcl_st(gp, v0, pol);
                    tcl_st(gp + ors, v1, pol);
                }
            }
        }
    }
};

}  // namespace nfft

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

template <int THREADS>
constexpr size_t tcl_smem_bytes() {
    return sizeof(float2) * (size_t)TCL_SLOTS + sizeof(long long) * 3 * (size_t)TCL_J;
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
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
#else
    (void)d; (void)a; (void)b0; (void)b1;
#endif
}

// One complex 16 x 16 product on the tensor cores: acc[mt][nt][i] =
// ([[Fr, -Fi], [Fi, Fr]] [Xr; Xi]) with B fragments xb[kt][nt][hi/lo][reg];
// the three terms of each block with the small ones first.
NFFT_HD void tcl_terms(float* d, const uint32_t* ah, const uint32_t* al, const uint32_t (&x)[2][2]) {
    tcl_mma(d, al, x[0][0], x[0][1]);
    tcl_mma(d, ah, x[1][0], x[1][1]);
    tcl_mma(d, ah, x[0][0], x[0][1]);
}
NFFT_HD void tcl_stage(const TcA& A, const uint32_t (&xb)[2][2][2][2], float (&acc)[2][2][4]) {
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[0][nt][i] = acc[1][nt][i] = 0.0f;
        tcl_terms(acc[0][nt], A.rh, A.rl, xb[0][nt]);     // Yr += Fr Xr
        tcl_terms(acc[0][nt], A.nih, A.nil, xb[1][nt]);   // Yr -= Fi Xi
        tcl_terms(acc[1][nt], A.ih, A.il, xb[0][nt]);     // Yi += Fi Xr
        tcl_terms(acc[1][nt], A.rh, A.rl, xb[1][nt]);     // Yi += Fr Xi
    }
}

// Exponent e with m 2^e in [2^9, 2^10) (m > 0), clamped to keep 2^e and
// 2^-e normal; 0 for m = 0 or non-finite m.
NFFT_HD int tcl_scale_exp(float m) {
    if (!(m > 0.0f) || !(m < 3.0e38f)) return 0;
    int e;
    frexpf(m, &e);   // m = f 2^e, f in [0.5, 1)
    int s = 10 - e;
    if (s > 120) s = 120;
    if (s < -120) s = -120;
    return s;
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

template <int THREADS>
struct TcLean {
    static constexpr int WARPS = THREADS / 32;
    static_assert(TCL_J % WARPS == 0, "lines per warp");
    static constexpr int LPW = TCL_J / WARPS;
    static constexpr int PER_THREAD = TCL_SLOTS / THREADS;

    // Per-lane constants: F fragments and the internal twiddles W_256^{b k1}
    // of the lane's stage-1 outputs (k1 = g + 8 (i >> 1), b = 2q + (i & 1) + 8 nt).
    struct Consts {
        TcA A;
        float2 itw[2][4];
    };

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

    // Phase 1: the lane's 8 points from shared memory, pass pre-twiddle
    // W_{Ns R}^{r k} (k = j mod Ns, r = b + 16 a: W^{b k} per butterfly times
    // (W^{16 k})^a per point).  Returns the lane's largest component.
    static NFFT_HD float load(const PassArgs& a, const TwTables<float>* tw, const float2* sm, int l, long long j,
                              int lane, LineRegs& s) {
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int h = 0; h < 2; ++h) s.x[nt][i][h] = sm[NFFT_SM(tcl_slot(in_point(lane, nt, i, h), l))];
        if (a.logNs > 0) {
            const long long k = j & ((1ll << a.logNs) - 1);
            if (k) {
                const int g = lane >> 2, q = lane & 3;
                const int logP = a.logNs + TCL_LOGR;
                const float2 wb0 = twiddle<float>(tw, (uint64_t)g * (uint64_t)k, logP);
                const float2 w8 = twiddle<float>(tw, (uint64_t)8 * (uint64_t)k, logP);
                const float2 wb1 = cmul(wb0, w8);
                const float2 s1 = twiddle<float>(tw, (uint64_t)16 * (uint64_t)k, logP);
                const float2 va = twiddle<float>(tw, (uint64_t)(32 * q) * (uint64_t)k, logP);
                const float2 s8 = twiddle<float>(tw, (uint64_t)128 * (uint64_t)k, logP);
                float2 v[2][2];
                v[0][0] = va;
                v[0][1] = cmul(va, s1);
                v[1][0] = cmul(va, s8);
                v[1][1] = cmul(v[1][0], s1);
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        s.x[0][i][h] = cmul(s.x[0][i][h], cmul(wb0, v[i][h]));
                        s.x[1][i][h] = cmul(s.x[1][i][h], cmul(wb1, v[i][h]));
                    }
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

    // Phase 2: scale by the line's power of two (m = the line's largest
    // component) and split into stage 1's B fragments.
    static NFFT_HD void split1(float m, LineRegs& s) {
        s.e = tcl_scale_exp(m);
        const float sc = ldexpf(1.0f, s.e);
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                tcl_split2(s.x[nt][i][0].x * sc, s.x[nt][i][1].x * sc, s.xb[0][nt][0][i], s.xb[0][nt][1][i]);
                tcl_split2(s.x[nt][i][0].y * sc, s.x[nt][i][1].y * sc, s.xb[1][nt][0][i], s.xb[1][nt][1][i]);
            }
    }

    // Phase 3: internal twiddle W_256^{b k1} on the stage-1 accumulators, then
    // stage 2's B fragments: B2[kt][nt2] reg 0 = (b = 2q, 2q+1) from n-tile 0,
    // reg 1 = (b = 2q+8, 2q+9) from n-tile 1, both at k1 = g + 8 nt2
    // (accumulator regs 2 nt2 + {0, 1}).
    static NFFT_HD void mid(const Consts& c, LineRegs& s) {
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float2 u = cmul(mkc(s.acc[0][nt][i], s.acc[1][nt][i]), c.itw[nt][i]);
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
    // the line's shared slots, in place.
    static NFFT_HD void store(const PassArgs& a, float2* sm, int l, int lane, const LineRegs& s) {
        const float f = ldexpf((float)a.scale, -s.e);
        const float fi = a.conj_out ? -f : f;
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int i = 0; i < 4; ++i)
                sm[NFFT_SM(tcl_slot(out_point(lane, nt, i), l))] = mkc(s.acc[0][nt][i] * f, s.acc[1][nt][i] * fi);
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
        mid(c, s);
        tcl_stage(c.A, s.xb, s.acc);
        store(a, sm, l, lane, s);
    }
#endif
};

// One tile (16 lines) of a radix-256 split tensor-core pass.  The input is
// read once (coalesced: lines fastest in column mode, points fastest in row
// mode), every warp transforms its lines in shared memory, and the tile is
// written once with the matching mapping of the output side.
template <int THREADS>
__device__ __forceinline__ void tc_lean_tile(const PassArgs& a, const typename TcLean<THREADS>::Consts& c,
                                             long long tile, float2* sm, long long* lin) {
    using TL = TcLean<THREADS>;
    const TwTables<float>* tw = (const TwTables<float>*)a.tw;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    long long* lout = lin + TCL_J;
    long long* lj = lout + TCL_J;
    if (t < TCL_J) line_setup(a, (tile << TCL_LOGJ) + t, t, TileLines{lin, lout, lj});
    __syncthreads();
    // load: a batch of loads in flight before its shared stores
    {
        constexpr int BATCH = TL::PER_THREAD >= 8 ? 8 : TL::PER_THREAD;
#pragma unroll 1
        for (int b0 = 0; b0 < TL::PER_THREAD; b0 += BATCH) {
            float2 buf[BATCH];
#pragma unroll
            for (int it = 0; it < BATCH; ++it) {
                int l, r;
                tcl_walk(a.in_row, t + (b0 + it) * THREADS, l, r);
                const long long j = lj[l];
                if (j < 0) {
                    buf[it] = mkc(0.0f, 0.0f);
                } else {
                    buf[it] = gload((const float2*)a.in + tcl_in_off(a, lin[l], j, r), a.hint_in);
                    if (a.conj_in) buf[it].y = -buf[it].y;
                }
            }
#pragma unroll
            for (int it = 0; it < BATCH; ++it) {
                int l, r;
                tcl_walk(a.in_row, t + (b0 + it) * THREADS, l, r);
                sm[NFFT_SM(tcl_slot(r, l))] = buf[it];
            }
        }
    }
    __syncthreads();
#pragma unroll 1
    for (int k = 0; k < TL::LPW; ++k) {
        const int l = warp + k * TL::WARPS;
        if (lj[l] >= 0) TL::line(a, tw, c, sm, l, lj[l], lane);
    }
    __syncthreads();
    // store
#pragma unroll 4
    for (int it = 0; it < TL::PER_THREAD; ++it) {
        int l, r;
        tcl_walk(a.out_row, t + it * THREADS, l, r);
        const long long j = lj[l];
        if (j < 0) continue;
        gstore((float2*)a.out + tcl_out_off(a, lout[l], j, r), sm[NFFT_SM(tcl_slot(r, l))], a.hint_out);
    }
}

}  // namespace nfft

// nfft_umma.cuh -- layout of the split tensor-core radix-256 pass on the
// sm_100 tensor cores (tcgen05): the tile of 8 Stockham lines x 256 points,
// its shared-memory operands and the index maps of the kernel (nfft_tc.cu).
//
// Both radix-16 stages of the tile are 128 x 32 x 32 real products
//     D = A_hi B_hi + A_lo B_hi + A_hi B_lo      (FP16 operands, FP32 sums)
// issued by one thread as tcgen05.mma with the operands in shared memory and
// the accumulators in tensor memory:
//  * stage 1: row t = 16 l + i holds the 16 points i + 16 m of line l
//    (pass pre-twiddled, scaled by a power of two when out of range), columns
//    (2m, 2m+1) = (re, im); B is the real form of the radix-16 DFT matrix;
//    D row t = y_{l,i}[k1];
//  * the internal twiddles W_256^{i k1}, transposed into stage-2 rows
//    16 l + k1, columns (2i, 2i+1);
//  * stage 2 rows: z_{l,k1}[k2] = output point k1 + 16 k2 of line l.
// A operand layout: K-major, no swizzle: 8-row x 16-byte core matrices at
// row-group stride TCU_SBO and K-chunk stride TCU_LBO (padded so both the
// row-wise stage-1 writes and the transposed stage-2 writes are free of
// bank conflicts).  Input tiles arrive by tensor copy with the 64-byte
// swizzle; outputs leave through the same buffer by tensor store.
#pragma once

#include "nfft_pass.cuh"

namespace nfft {

constexpr int TCU_THREADS = 128;
constexpr int TCU_J = 8;                       // lines per tile
constexpr int TCU_MINB = 5;                    // CTAs per SM the kernel is built for
constexpr int TCU_LBO = 144, TCU_SBO = 672;    // A operand strides (bytes)
constexpr int TCU_AOP = 16 * TCU_SBO;          // one 128-row operand
constexpr int TCU_BLBO = 128, TCU_BSBO = 512;  // B operand (written once per CTA, unpadded)
constexpr int TCU_BOP = 4 * TCU_BSBO;          // one 32-row operand
constexpr int TCU_STAGE = TCU_J * 256 * 8;     // input tile, 64-byte swizzled rows
constexpr int TCU_OFF_AH = TCU_STAGE;
constexpr int TCU_OFF_AL = TCU_OFF_AH + TCU_AOP;
constexpr int TCU_OFF_BH = TCU_OFF_AL + TCU_AOP;
constexpr int TCU_OFF_BL = TCU_OFF_BH + TCU_BOP;
constexpr int TCU_OFF_TW = TCU_OFF_BL + TCU_BOP;   // W_256^{i k1}, stored [k1][i]
constexpr int TCU_OFF_BAR = TCU_OFF_TW + 256 * 8;  // mbarriers and the tensor-memory address
constexpr int TCU_SMEM = TCU_OFF_BAR + 64 + 512;   // + alignment of the stage to 512 bytes
constexpr int TCU_TCOLS = 64;                      // stage-1 and stage-2 accumulators
// Range: a radix-16 output is at most 16 sqrt(2) times the largest input
// component in modulus, so a line whose largest component is below 2^8 keeps
// every stage-1 output, stage-2 operand (< 5800) and FP16 part within FP16
// range; from 1/2 up the lo parts of its large values stay normal FP16
// numbers.  Lines outside [TCU_LO, TCU_HI) are scaled by a power of two into
// [1, 2) before the split and unscaled exactly after stage 2.
constexpr float TCU_LO = 0.5f, TCU_HI = 256.f;

// Where a pass writes: row out (Ns = 1, line j's outputs contiguous), column
// out with j split at Ns (Ns < lines), column out (Ns >= lines).
enum TcuOut { TCU_OUT_ROW = 0, TCU_OUT_COLSPLIT = 1, TCU_OUT_COL = 2 };

struct TcuArgs {
    PassArgs a;
    int out_kind;
    long long tiles_per_tr;    // lines per transform / 8
    long long ntiles;
    long long spin;            // poll limit of every wait
    int withhold;              // failure test: the first input copy is never issued
};

// point (row r, line l) of a 64-byte swizzled tile row (8 lines x 8 bytes)
NFFT_HD int tcu_st_off(int r, int l) { return r * 64 + (((l >> 1) ^ ((r >> 1) & 3)) << 4) + ((l & 1) << 3); }
// byte offset of the (re, im) f16 pair kp of A row `row`
NFFT_HD int tcu_a_off(int row, int kp) { return (row >> 3) * TCU_SBO + (kp >> 2) * TCU_LBO + (row & 7) * 16 + (kp & 3) * 4; }
NFFT_HD int tcu_b_off(int row, int kp) { return (row >> 3) * TCU_BSBO + (kp >> 2) * TCU_BLBO + (row & 7) * 16 + (kp & 3) * 4; }

// Entry (row n, K column c) of the real form of the radix-16 DFT matrix:
// D[2k] = sum_m xr Fr - xi Fi, D[2k+1] = sum_m xr Fi + xi Fr, F = W_16^{mk}.
NFFT_HD float tcu_b_entry(const TwTables<float>* tw, int n, int c) {
    const int k = n >> 1, d = n & 1, m = c >> 1, im = c & 1;
    const C2<float> f = tw->t[0][(m * k * 256) & (TW_SIZE - 1)];
    if (d == 0) return im ? -f.y : f.x;
    return im ? f.x : f.y;
}

// Line j of the tile's row t and the pass pre-twiddle exponent k = j mod Ns.
NFFT_HD void tcu_line(const TcuArgs& u, long long tile, int t, long long& b, int& j) {
    b = tile / u.tiles_per_tr;
    j = (int)(tile - b * u.tiles_per_tr) * TCU_J + (t >> 4);
}

// 2^e as a float (e in [-126, 127]; 0 below)
NFFT_HD float tcu_pow2(int e) {
    if (e < -126) return 0.f;
    if (e > 127) e = 127;
    union { uint32_t u; float f; } v;
    v.u = (uint32_t)(127 + e) << 23;
    return v.f;
}
// E with m 2^-E in [1, 2) for a positive normal m (clamped to +-100); 0 for m = 0
NFFT_HD int tcu_exp(float m) {
    union { float f; uint32_t u; } v;
    v.f = m;
    int e = (int)((v.u >> 23) & 0xff) - 127;
    e = e < -100 ? -100 : (e > 100 ? 100 : e);
    return m > 0.f ? e : 0;
}

}  // namespace nfft

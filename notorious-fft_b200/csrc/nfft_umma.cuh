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
//  * the internal twiddles W_256^{i k1}; stage 2 row (l, k1) column
//    (2i, 2i+1) is the twiddled y_{l,i}[k1], so the stage-2 operand is the
//    stage-1 result transposed per line: it is written M-major (8 rows of
//    one column per 16 bytes), which is a plain row of the thread that holds
//    y_{l,i}, and the product reads it with the A-transpose bit;
//  * stage 2 rows: z_{l,k1}[k2] = output point k1 + 16 k2 of line l.
// A operand layouts, no swizzle, the same two strides:
//  * stage 1, K-major: rows of 8 x 16-byte core matrices, K chunks (8 f16)
//    at TCU_LBO, 8-row groups at TCU_SBO;
//  * stage 2, M-major: 16-byte rows of 8 M values, K rows 16 bytes apart,
//    groups of 8 K rows at TCU_LBO, groups of 8 M at TCU_SBO.
// The 16-byte units of 8 consecutive lanes land in 8 distinct bank groups
// (TCU_LBO / 16 is odd).  Input tiles arrive by tensor copy with the 64-byte
// swizzle; outputs leave through the A region by tensor store.
//
// Thread roles.  Stage 1: thread t holds (line l, row i) with the two lines
// of a warp interleaved in groups of 8 lanes (tcu_role_a), so a half-warp
// reads 2 lines x 8 rows of the swizzled input tile: 16 distinct bank pairs.
// Stage 2 (thread t owns row t of the stage-2 operand, line l, output group
// k1): the same role for column outputs (their staging is the input tile's
// layout), and l = t / 16, k1 = t mod 16 for row outputs (a half-warp writes
// 16 consecutive points of one line).
#pragma once

#include "nfft_pass.cuh"

namespace nfft {

// A CTA holds TCU_TEAMS teams of 128 threads; each team transforms its own
// tiles with its own input stage, operand region, mbarriers, tensor-memory
// columns and named barrier, and the teams share the constant operands.
// One team per CTA at five CTAs per SM is the build: two teams at three CTAs
// per SM (six tiles in flight instead of five) measured 1.5% slower on B200
// (4096 x 2^16: 1.548 vs 1.524 ms; 1024 x 2^16: 0.386 vs 0.379 ms).
constexpr int TCU_TEAMS = 1;
constexpr int TCU_THREADS = 128 * TCU_TEAMS;
constexpr int TCU_J = 8;                       // lines per tile
constexpr int TCU_MINB = TCU_TEAMS == 2 ? 3 : 5;   // CTAs per SM the kernel is built for
constexpr int TCU_LBO = 144, TCU_SBO = 576;    // A operand strides (bytes)
constexpr int TCU_AOP = 16 * TCU_SBO;          // one 128-row operand
constexpr int TCU_BLBO = 128, TCU_BSBO = 512;  // B operand (written once per CTA, unpadded)
constexpr int TCU_BOP = 4 * TCU_BSBO;          // one 32-row operand
constexpr int TCU_STAGE = TCU_J * 256 * 8;     // input tile, 64-byte swizzled rows
// per team: input stage, then the hi and lo A operands (the output staging after stage 2)
constexpr int TCU_TEAM_BYTES = TCU_STAGE + 2 * TCU_AOP;
constexpr int TCU_OFF_AH = TCU_STAGE;          // within a team's region
constexpr int TCU_OFF_AL = TCU_OFF_AH + TCU_AOP;
constexpr int TCU_OFF_BH = TCU_TEAMS * TCU_TEAM_BYTES;
constexpr int TCU_OFF_BL = TCU_OFF_BH + TCU_BOP;
constexpr int TCU_OFF_TW = TCU_OFF_BL + TCU_BOP;   // W_256^{i k1}, stored [k1][i]
constexpr int TCU_OFF_BAR = TCU_OFF_TW + 256 * 8;  // 2 mbarriers per team, then the tensor-memory address
constexpr int TCU_SMEM = TCU_OFF_BAR + 64 + 512;   // + alignment of the stage to 512 bytes
static_assert(TCU_TEAM_BYTES % 512 == 0, "team stages stay 512-byte aligned");
static_assert(16 * TCU_TEAMS + 4 <= 64, "mbarriers and tensor-memory slot");
static_assert(2 * TCU_AOP >= TCU_J * 256 * 8, "output staging fits the A region");
static_assert(4 * TCU_LBO <= TCU_SBO && ((TCU_LBO / 16) & 1), "A operand strides");
constexpr int TCU_TCOLS = 64 * TCU_TEAMS;          // per team: stage-1 and stage-2 accumulators
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
    int log_tpt;               // log2(tiles_per_tr)
    long long ntiles;
    long long spin;            // poll limit of every wait
    int withhold;              // failure test: the first input copy is never issued
};

// point (row r, line l) of a 64-byte swizzled tile row (8 lines x 8 bytes)
NFFT_HD int tcu_st_off(int r, int l) { return r * 64 + (((l >> 1) ^ ((r >> 1) & 3)) << 4) + ((l & 1) << 3); }
// byte offset of the (re, im) f16 pair kp of K-major A row `row`
NFFT_HD int tcu_a_off(int row, int kp) { return (row >> 3) * TCU_SBO + (kp >> 2) * TCU_LBO + (row & 7) * 16 + (kp & 3) * 4; }
// byte offset of the 16-byte unit (rows m0 .. m0 + 7, column k) of M-major A (m0 a multiple of 8)
NFFT_HD int tcu_at_off(int m0, int k) { return (m0 >> 3) * TCU_SBO + (k >> 3) * TCU_LBO + (k & 7) * 16; }
NFFT_HD int tcu_b_off(int row, int kp) { return (row >> 3) * TCU_BSBO + (kp >> 2) * TCU_BLBO + (row & 7) * 16 + (kp & 3) * 4; }

// Entry (row n, K column c) of the real form of the radix-16 DFT matrix:
// D[2k] = sum_m xr Fr - xi Fi, D[2k+1] = sum_m xr Fi + xi Fr, F = W_16^{mk}.
NFFT_HD float tcu_b_entry(const TwTables<float>* tw, int n, int c) {
    const int k = n >> 1, d = n & 1, m = c >> 1, im = c & 1;
    const C2<float> f = tw->t[0][(m * k * 256) & (TW_SIZE - 1)];
    if (d == 0) return im ? -f.y : f.x;
    return im ? f.x : f.y;
}

// Stage-1 role of thread t (line l of the tile, row i) and its inverse.
NFFT_HD void tcu_role_a(int t, int& l, int& i) {
    l = ((t >> 5) << 1) | ((t >> 3) & 1);
    i = (t & 7) | (((t >> 4) & 1) << 3);
}
NFFT_HD int tcu_row_a(int l, int i) { return ((l >> 1) << 5) | ((i >> 3) << 4) | ((l & 1) << 3) | (i & 7); }
// Stage-2 role of thread t (line l, output group k1) and its inverse, by output kind.
NFFT_HD void tcu_role_b(int kind, int t, int& l, int& k1) {
    if (kind == TCU_OUT_ROW) {
        l = t >> 4;
        k1 = t & 15;
    } else {
        tcu_role_a(t, l, k1);
    }
}
NFFT_HD int tcu_row_b(int kind, int l, int k1) { return kind == TCU_OUT_ROW ? 16 * l + k1 : tcu_row_a(l, k1); }

// Transform b and first line j0 of a tile (lines per transform / 8 is a power of two).
NFFT_HD void tcu_tile(const TcuArgs& u, long long tile, long long& b, int& j0) {
    b = tile >> u.log_tpt;
    j0 = (int)(tile & (u.tiles_per_tr - 1)) * TCU_J;
}

NFFT_HD C2<float> tcu_cmul(C2<float> a, C2<float> b) { return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// The passes the kernel takes: lines j of a transform at unit stride (one
// transform, or a batch dimension outside j), plain complex loads and stores,
// distinct 16-byte aligned buffers and batch strides, and an output order it
// can store by tensor map (row out, or column out at Ns >= 8).  Fills the
// tile counts and the output kind; false (and nothing launched) for any
// other pass.
inline bool tcu_shape(const PassArgs& a, TcuArgs& u) {
    if (a.logR != 8 || (a.ndims != 1 && a.ndims != 2) || a.jpos != 0) return false;
    if (a.in_estride != 1 || a.out_estride != 1) return false;
    if (a.in_tab || a.out_tab || a.mid || a.vjp || a.logNj < 3 || a.cnt[0] != (1ll << a.logNj)) return false;
    if (a.logNs_out != 0 && a.logNs_out < 3) return false;
    if (((uintptr_t)a.in & 15) || ((uintptr_t)a.out & 15) || a.in == a.out) return false;
    const long long B = a.ndims == 2 ? a.cnt[1] : 1, Nj = a.cnt[0];
    if (B < 1 || Nj * B != a.nlines) return false;
    if (B > 1 && ((a.istr[1] & 1) || (a.ostr[1] & 1) || a.istr[1] <= 0 || a.ostr[1] <= 0)) return false;
    u.a = a;
    if (a.ndims == 1) {   // one transform: batch stride unused, count 1
        u.a.ndims = 2;
        u.a.cnt[1] = 1;
        u.a.istr[1] = u.a.ostr[1] = 0;
    }
    u.out_kind = a.logNs_out == 0 ? TCU_OUT_ROW : (a.logNs_out < a.logNj ? TCU_OUT_COLSPLIT : TCU_OUT_COL);
    u.tiles_per_tr = Nj / TCU_J;
    u.log_tpt = a.logNj - 3;
    u.ntiles = u.tiles_per_tr * B;
    u.spin = 1ll << 22;
    u.withhold = 0;
    return true;
}

// Element offsets (complex points) of point r of line j of transform b: the
// input, and output point p, as the kernel's tensor maps lay them out.
NFFT_HD long long tcu_in_index(const TcuArgs& u, long long b, int j, int r) {
    return b * u.a.istr[1] + j + (long long)r * u.a.cnt[0];
}
NFFT_HD long long tcu_out_index(const TcuArgs& u, long long b, int j, int p) {
    const int s = u.a.logNs_out;
    const long long base = b * u.a.ostr[1];
    if (u.out_kind == TCU_OUT_ROW) return base + ((long long)j << 8) + p;
    if (u.out_kind == TCU_OUT_COLSPLIT)
        return base + ((long long)(j >> s) << (s + 8)) + (j & ((1 << s) - 1)) + ((long long)p << s);
    return base + j + ((long long)p << s);
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

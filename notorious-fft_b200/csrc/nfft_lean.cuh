// nfft_lean.cuh -- the specialized pass kernel (hot path).
//
// Same Stockham pass semantics as pass_kernel (nfft_pass.cuh), with the pass
// radix R = 2^LOGR and the tile shape fixed at compile time:
//  * the first sub-stage is radix 16 and reads its 16 points per thread
//    straight from global memory (no shared-memory staging), with the pass
//    pre-twiddle W_{Ns R}^{r k} generated per line from two table roots and
//    a depth-4 product tree;
//  * middle sub-stages exchange through shared memory;
//  * the last sub-stage writes its outputs straight to global memory, except
//    for the paired real operators, which need whole lines in shared memory.
// Thread-to-butterfly mappings are chosen per sub-stage so that global
// accesses coalesce: "column" mode walks consecutive lines (J adjacent
// Stockham lines or a unit-stride batch dim), "row" mode walks along a line.
// Column tiles are stored [r][line] with a pitch of J+1 points, row tiles
// [line][r] with one pad point every 16, which keeps both mappings free of
// shared-memory bank conflicts.
#pragma once

#include "nfft_pass.cuh"

namespace nfft {

// Sub-stage radices (log2) of a pass of radix 2^LOGR: radix 16 first.
template <int LOGR> struct LeanSched;
template <> struct LeanSched<4> { static constexpr int n = 1; static constexpr int lr[4] = {4, 0, 0, 0}; };
template <> struct LeanSched<5> { static constexpr int n = 2; static constexpr int lr[4] = {4, 1, 0, 0}; };
template <> struct LeanSched<6> { static constexpr int n = 2; static constexpr int lr[4] = {4, 2, 0, 0}; };
template <> struct LeanSched<7> { static constexpr int n = 2; static constexpr int lr[4] = {4, 3, 0, 0}; };
template <> struct LeanSched<8> { static constexpr int n = 2; static constexpr int lr[4] = {4, 4, 0, 0}; };
template <> struct LeanSched<9> { static constexpr int n = 3; static constexpr int lr[4] = {4, 3, 2, 0}; };
template <> struct LeanSched<10> { static constexpr int n = 3; static constexpr int lr[4] = {4, 4, 2, 0}; };
template <> struct LeanSched<11> { static constexpr int n = 3; static constexpr int lr[4] = {4, 4, 3, 0}; };
template <> struct LeanSched<12> { static constexpr int n = 3; static constexpr int lr[4] = {4, 4, 4, 0}; };
template <> struct LeanSched<13> { static constexpr int n = 4; static constexpr int lr[4] = {4, 4, 3, 2}; };

// Shared-memory index of point r of tile line l.
template <bool COL, int LOGR, int LOGJ>
NFFT_HD int lean_idx(int l, int r) {
    if constexpr (COL) return r * ((1 << LOGJ) + 1) + l;
    else return spad((l << LOGR) + r);
}
template <bool COL, int LOGR, int LOGJ> constexpr int lean_smem_elems() {
    return COL ? (1 << LOGR) * ((1 << LOGJ) + 1) : ((1 << (LOGR + LOGJ)) + (1 << (LOGR + LOGJ - 4)) + 1);
}

// Butterfly b of a sub-stage with B = 2^lb butterflies per line -> (line, i).
// Column mapping: lines fastest; row mapping: butterflies fastest.
template <bool COLMAP, int LOGJ>
NFFT_HD void lean_map(int b, int lb, int& l, int& i) {
    if constexpr (COLMAP) { l = b & ((1 << LOGJ) - 1); i = b >> LOGJ; }
    else { i = b & ((1 << lb) - 1); l = b >> lb; }
}

// x^0 .. x^15 by a depth-4 product tree.
template <typename T>
NFFT_HD void powers16(C2<T> x, C2<T>* p) {
    p[0] = mkc((T)1, (T)0);
    p[1] = x;
    p[2] = cmul(x, x);
    p[3] = cmul(p[2], x);
    p[4] = cmul(p[2], p[2]);
    p[8] = cmul(p[4], p[4]);
    p[12] = cmul(p[8], p[4]);
#pragma unroll
    for (int a = 4; a < 16; a += 4) {
        p[a + 1] = cmul(p[a], x);
        p[a + 2] = cmul(p[a], p[2]);
        p[a + 3] = cmul(p[a], p[3]);
    }
}

// Per-line state held by every thread of the line.
struct LeanLine {
    long long bin, bout, j;
};

// ---- mirror tiles: the last pass of a multi-pass realdft / DCT-2 / DST-2 ------
// The last pass of the packed N/2-point spectrum Z (M = N/2) writes, for line j
// of the ns = M / R lines of a transform, Z[j + r ns], r < R.  Bin k pairs with
// bin M - k, which lives on line ns - j (lines 0 and ns / 2 pair with
// themselves).  A mirror tile therefore holds J/2 "low" lines and their J/2
// partners: tile tt of a transform holds j = tt J/2 + l and ns - (tt J/2 + l)
// for l < J/2, except tile 0, whose first low line is j = 0 and first high line
// j = ns / 2.  The Hermitian unpack then runs inside the tile.
//
// Stockham line of local line l (of J) in tile tt of a transform.
NFFT_HD long long mirror_line(long long tt, int l, int J, long long ns) {
    const int h = J / 2;
    if (l < h) return (tt == 0 && l == 0) ? 0 : tt * h + l;
    const int u = l - h;
    if (tt == 0) return u == 0 ? ns / 2 : ns - u;
    return ns - (tt * h + u);
}
// Local line of Stockham line j in tile tt (inverse of mirror_line).
NFFT_HD int mirror_local(long long tt, long long j, int J, long long ns) {
    const int h = J / 2;
    if (tt == 0) {
        if (j == 0) return 0;
        if (j == ns / 2) return h;
        return j < ns / 2 ? (int)j : (int)(h + (ns - j));
    }
    return j < ns / 2 ? (int)(j - tt * h) : (int)(h + (ns - j - tt * h));
}
// Bin k of unpack item (l < J/2, r < R) of tile tt: every item emits bins k and
// M - k (unpack_pair), the items of a tile cover both lines of each pair.
NFFT_HD long long mirror_item_k(long long tt, int l, int r, int R, long long ns, long long lowj) {
    if (tt == 0 && l == 0) return r < R / 2 ? (long long)r * ns : ns / 2 + (long long)(r - R / 2) * ns;
    return lowj + (long long)r * ns;
}

template <typename T, int LOGR, int LOGT, bool COL_IN, bool COL_OUT, int LOAD, int STORE>
struct Lean {
    static constexpr int THREADS = 1 << LOGT;
    static constexpr int LOGTILE = LOGT + 4;
    static constexpr int LOGJ = LOGTILE - LOGR;
    static constexpr int J = 1 << LOGJ;
    static constexpr int R = 1 << LOGR;
    static constexpr int LOGR_ = LOGR;
    static constexpr bool COL_OUT_ = COL_OUT;
    static constexpr bool PAIRED = (STORE == ST_R || STORE == ST_T2);
    // shared layout: column tiles whenever either side walks lines
    static constexpr bool COLL = COL_IN || COL_OUT;
    static constexpr int NS = LeanSched<LOGR>::n;
    static constexpr int SMEM_ELEMS = lean_smem_elems<COLL, LOGR, LOGJ>();
    static_assert(LOGJ >= 0 && LOGJ <= 8, "tile must hold 1..256 lines");
    // paired stores need whole lines in the tile: row tiles, or mirror tiles
    // (column in and out) for the last pass of a multi-pass transform
    static constexpr bool MIRROR = PAIRED && COL_IN && COL_OUT;
    // row tile of a single-pass DCT-3 / DST-3 or inverse real transform: the
    // input repack runs as a paired phase into shared memory
    // (pair_prepack_thread) and the first sub-stage reads its points from there
    static constexpr bool PREPACK = (LOAD == LD_T3 || LOAD == LD_IR) && !COL_IN;
    static_assert(!(PAIRED && (COL_IN != COL_OUT)), "paired operators need row tiles or mirror tiles");
    static_assert(!MIRROR || LOGJ >= 1, "mirror tiles pair lines");

    // first sub-stage (points from shared memory, then the radix-16 DFT) of PREPACK tiles
    static NFFT_HD void first_smem(const PassArgs& a, const TwTables<T>* tw, const C2<T>* sm, const LeanLine* lines,
                                   int t, C2<T>* v, int& l, int& i) {
        lean_map<false, LOGJ>(t, LOGR - 4, l, i);
        const LeanLine ln = lines[l];
        if (ln.j < 0) {
#pragma unroll
            for (int m = 0; m < 16; ++m) v[m] = mkc((T)0, (T)0);
            return;
        }
#pragma unroll
        for (int m = 0; m < 16; ++m) v[m] = sm[NFFT_SM((lean_idx<false, LOGR, LOGJ>(l, i + (m << (LOGR - 4)))))];
        pre_twiddle_dft(a, tw, ln.j, i, v);
    }

    // ---- first sub-stage: global -> registers -> radix 16 --------------------
    static NFFT_HD void first(const PassArgs& a, const TwTables<T>* tw, const LeanLine* lines, int t, C2<T>* v, int& l,
                              int& i) {
        lean_map<COL_IN, LOGJ>(t, LOGR - 4, l, i);
        const LeanLine ln = lines[l];
        if (ln.j < 0) {
#pragma unroll
            for (int m = 0; m < 16; ++m) v[m] = mkc((T)0, (T)0);
            return;
        }
        if constexpr (LOAD == LD_C) {
            const long long rs = a.in_estride << a.logNj;
            const C2<T>* src = (const C2<T>*)a.in + ln.bin + ln.j * a.in_estride + (long long)i * rs;
            const long long s16 = rs << (LOGR - 4);
            if (a.hint_in == 3) {
#pragma unroll
                for (int m = 0; m < 16; ++m) v[m] = gload(src + m * s16, 3);
            } else if (a.hint_in) {
#pragma unroll
                for (int m = 0; m < 16; ++m) v[m] = gload(src + m * s16, 1);
            } else {
#pragma unroll
                for (int m = 0; m < 16; ++m) v[m] = NFFT_GLD(src + m * s16);
            }
            if (a.conj_in) {
#pragma unroll
                for (int m = 0; m < 16; ++m) v[m].y = -v[m].y;
            }
        } else if constexpr ((LOAD == LD_BLUE || LOAD == LD_FILT) && COL_IN) {
            // first pass of a Bluestein M-point FFT: LD_C's strided addressing
            // plus one table point per point, position p = j + (i + m R/16) Nj
            // (forward: chirp premultiply, zero pad from N on; inverse: conj of
            // the filter product).  All loads issued before any is used.
            const long long rs = a.in_estride << a.logNj;
            const C2<T>* src = (const C2<T>*)a.in + ln.bin + ln.j * a.in_estride + (long long)i * rs;
            const long long s16 = rs << (LOGR - 4);
            const long long p0 = ln.j + ((long long)i << a.logNj), ps = 1ll << (a.logNj + LOGR - 4);
            const C2<T>* tab = (const C2<T>*)(LOAD == LD_BLUE ? a.chirp : a.filt) + p0;
            // two halves of 8 points: 16 loads in flight, as for LD_C
#pragma unroll
            for (int hf = 0; hf < 16; hf += 8) {
                C2<T> c[8];
                if constexpr (LOAD == LD_BLUE) {
#pragma unroll
                    for (int m = hf; m < hf + 8; ++m) {
                        const bool in = p0 + m * ps < a.N;
                        v[m] = in ? gload(src + m * s16, a.hint_in) : mkc((T)0, (T)0);
                        c[m - hf] = in ? gload_keep(tab + m * ps) : mkc((T)0, (T)0);
                    }
#pragma unroll
                    for (int m = hf; m < hf + 8; ++m) {
                        if (a.conj_in) v[m].y = -v[m].y;
                        v[m] = cmul(v[m], c[m - hf]);
                    }
                } else {
#pragma unroll
                    for (int m = hf; m < hf + 8; ++m) {
                        v[m] = gload(src + m * s16, a.hint_in);   // queue: scratch of this launch at L2
                        c[m - hf] = gload_keep(tab + m * ps);
                    }
#pragma unroll
                    for (int m = hf; m < hf + 8; ++m) v[m] = cconj(cmul(v[m], c[m - hf]));
                }
            }
        } else if constexpr (LOAD == LD_T4 && !COL_IN) {
            // row tile of a single-pass DCT-4 / DST-4 (line j = 0): premultiply
            // e^{-i pi p / N} of p = i + m R/16 as a chain of exact steps
            // e^{-i pi (R/16) / N} = W_64 (N = 2R) from one table twiddle
            const T* x = (const T*)a.in + ln.bin;
            if (a.in_estride == 1 && ln.j == 0) {
                const long long N = a.N;
                C2<T> e = twiddle<T>(tw, (uint64_t)i, a.logN + 1);
                const C2<T> st = twiddle<T>(tw, (uint64_t)1, 6);
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    const long long p = i + (m << (LOGR - 4));
                    const T xe = NFFT_GLD(&x[2 * p]), xo = NFFT_GLD(&x[N - 1 - 2 * p]);
                    if (!a.dst) v[m] = mkc(e.x * xe - e.y * xo, e.x * xo + e.y * xe);
                    else v[m] = mkc(-e.x * xe - e.y * xo, e.x * xo - e.y * xe);
                    if (m < 15) e = cmul(e, st);
                }
            } else {
#pragma unroll
                for (int m = 0; m < 16; ++m)
                    v[m] = load_elem<T, LOAD>(a, tw, ln.bin, ln.j + ((long long)(i + (m << (LOGR - 4))) << a.logNj));
            }
        } else if constexpr ((LOAD == LD_R2C || LOAD == LD_T2) && !COL_IN) {
            // row tile of a single-pass real transform (line j = 0): the packed
            // point p = i + m R/16 of the line's N = 2R reals, without the generic
            // operator's per-element branches
            const T* x = (const T*)a.in + ln.bin;
            if (a.in_estride == 1 && ln.j == 0) {
                if constexpr (LOAD == LD_R2C) {
                    if (((uintptr_t)x & (sizeof(C2<T>) - 1)) == 0) {
#pragma unroll
                        for (int m = 0; m < 16; ++m) v[m] = NFFT_GLD((const C2<T>*)x + i + (m << (LOGR - 4)));
                    } else {
#pragma unroll
                        for (int m = 0; m < 16; ++m) {
                            const long long q = 2 * (long long)(i + (m << (LOGR - 4)));
                            v[m] = mkc(NFFT_GLD(&x[q]), NFFT_GLD(&x[q + 1]));
                        }
                    }
                } else {
                    // DCT-2 / DST-2 reorder v[i] = x[2i] (i < N/2), +-x[2N-1-2i]: points
                    // m < 8 lie in the first half of the packed line, m >= 8 in the second
                    const long long N2 = 2 * a.N;
                    const T sg = a.dst ? (T)-1 : (T)1;
#pragma unroll
                    for (int m = 0; m < 16; ++m) {
                        const long long q = 4 * (long long)(i + (m << (LOGR - 4)));
                        if (m < 8) v[m] = mkc(NFFT_GLD(&x[q]), NFFT_GLD(&x[q + 2]));
                        else v[m] = mkc(sg * NFFT_GLD(&x[N2 - 1 - q]), sg * NFFT_GLD(&x[N2 - 3 - q]));
                    }
                }
            } else {
#pragma unroll
                for (int m = 0; m < 16; ++m)
                    v[m] = load_elem<T, LOAD>(a, tw, ln.bin, ln.j + ((long long)(i + (m << (LOGR - 4))) << a.logNj));
            }
        } else {
#pragma unroll
            for (int m = 0; m < 16; ++m)
                v[m] = load_elem<T, LOAD>(a, tw, ln.bin, ln.j + ((long long)(i + (m << (LOGR - 4))) << a.logNj));
        }
        pre_twiddle_dft(a, tw, ln.j, i, v);
    }

    // Pass pre-twiddle W_{Ns R}^{r k} (k = j mod Ns) of the 16 points r = i + m R/16
    // of line j held by this thread, then the first radix-16 DFT.
    static NFFT_HD void pre_twiddle_dft(const PassArgs& a, const TwTables<T>* tw, long long j, int i, C2<T>* v) {
        if (a.logNs > 0) {
            const long long k = j & ((1ll << a.logNs) - 1);
            if (k) {
                // W_{Ns R}^{(i + m R/16) k} = W_{Ns R}^{i k} * (W_{16 Ns}^{k})^m
                if (a.tw_mode == 2) {
#pragma unroll
                    for (int m = 0; m < 16; ++m)
                        v[m] = cmul(v[m], twiddle<T>(tw, (uint64_t)(i + (m << (LOGR - 4))) * (uint64_t)k, a.logNs + LOGR));
                } else if (a.tw_mode == 1) {
                    C2<T> w = twiddle<T>(tw, (uint64_t)i * (uint64_t)k, a.logNs + LOGR);
                    const C2<T> s = twiddle<T>(tw, (uint64_t)k, a.logNs + 4);
                    const C2<T> s4 = cmul(cmul(s, s), cmul(s, s));
                    // four interleaved chains w s^{4c + d}: depth 4 per chain
                    C2<T> c0 = w, c1 = cmul(w, s);
                    C2<T> c2 = cmul(c1, s), c3 = cmul(c2, s);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        v[4 * q + 0] = cmul(v[4 * q + 0], c0);
                        v[4 * q + 1] = cmul(v[4 * q + 1], c1);
                        v[4 * q + 2] = cmul(v[4 * q + 2], c2);
                        v[4 * q + 3] = cmul(v[4 * q + 3], c3);
                        if (q < 3) { c0 = cmul(c0, s4); c1 = cmul(c1, s4); c2 = cmul(c2, s4); c3 = cmul(c3, s4); }
                    }
                } else {
                    C2<T> w0 = twiddle<T>(tw, (uint64_t)i * (uint64_t)k, a.logNs + LOGR);
                    C2<T> s = twiddle<T>(tw, (uint64_t)k, a.logNs + 4);
                    C2<T> p[16];
                    powers16<T>(s, p);
#pragma unroll
                    for (int m = 0; m < 16; ++m) v[m] = cmul(v[m], (m == 0) ? w0 : cmul(w0, p[m]));
                }
            }
        }
        dft16<T>(v);
    }

    // ---- middle / last sub-stage read from shared memory ----------------------
    template <int S, bool COLMAP>
    static NFFT_HD void read(const C2<T>* sm, int t, int q, C2<T>* v, int& l, int& i) {
        constexpr int LR = LeanSched<LOGR>::lr[S];
        constexpr int RHO = 1 << LR;
        constexpr int lq = LOGR - LR;
        lean_map<COLMAP, LOGJ>(t + q * THREADS, lq, l, i);
#pragma unroll
        for (int m = 0; m < RHO; ++m) v[m] = sm[NFFT_SM((lean_idx<COLL, LOGR, LOGJ>(l, i + (m << lq))))];
    }

    // internal twiddles W_{ns RHO}^{m k} and the radix-RHO DFT (ns = 2^lns)
    template <int S>
    static NFFT_HD void twiddle_dft(const TwTables<T>* tw, int i, C2<T>* v) {
        constexpr int LR = LeanSched<LOGR>::lr[S];
        constexpr int RHO = 1 << LR;
        constexpr int lns = lns_of<S>();
        const int k = i & ((1 << lns) - 1);
        if (k) {
            // W^{m k} for m < RHO from the root W^k by a product tree (depth <= 4)
            const C2<T> w1 = (lns + LR <= TW_BITS) ? twiddle_small<T>(tw, (uint32_t)k, lns + LR)
                                                   : twiddle<T>(tw, (uint64_t)k, lns + LR);
            if constexpr (RHO == 16) {
                C2<T> p[16];
                powers16<T>(w1, p);
#pragma unroll
                for (int m = 1; m < 16; ++m) v[m] = cmul(v[m], p[m]);
            } else {
                C2<T> w = w1;
#pragma unroll
                for (int m = 1; m < RHO; ++m) {
                    v[m] = cmul(v[m], w);
                    if (m + 1 < RHO) w = cmul(w, w1);
                }
            }
        }
        dft_radix<T, RHO>(v);
    }

    template <int S> static constexpr int lns_of() {
        int s = 0;
        for (int x = 0; x < S; ++x) s += LeanSched<LOGR>::lr[x];
        return s;
    }

    // Stockham output position of sub-stage S (within the line)
    template <int S>
    static NFFT_HD int out_pos(int i, int m) {
        constexpr int LR = LeanSched<LOGR>::lr[S];
        constexpr int lns = lns_of<S>();
        const int k = i & ((1 << lns) - 1);
        return ((i >> lns) << (lns + LR)) + k + (m << lns);
    }

    template <int S>
    static NFFT_HD void write_smem(C2<T>* sm, int l, int i, const C2<T>* v) {
        constexpr int RHO = 1 << LeanSched<LOGR>::lr[S];
#pragma unroll
        for (int m = 0; m < RHO; ++m) sm[NFFT_SM((lean_idx<COLL, LOGR, LOGJ>(l, out_pos<S>(i, m))))] = v[m];
    }

    // last sub-stage: outputs straight to global memory
    template <int S>
    static NFFT_HD void write_global(const PassArgs& a, const TwTables<T>* tw, const LeanLine* lines, int l, int i,
                                     const C2<T>* v) {
        constexpr int RHO = 1 << LeanSched<LOGR>::lr[S];
        const LeanLine ln = lines[l];
        if (ln.j < 0) return;
        const int logNso = a.logNs_out;
        const long long base = ((ln.j >> logNso) << (logNso + LOGR)) + (ln.j & ((1ll << logNso) - 1));
        if constexpr (STORE == ST_C) {
            const long long rs = a.out_estride << logNso;
            C2<T>* dst = (C2<T>*)a.out + ln.bout + base * a.out_estride + (long long)out_pos<S>(i, 0) * rs;
            constexpr int lns = lns_of<S>();
            const long long sm_ = rs << lns;   // output positions step by 2^lns per m
            C2<T> x[RHO];
            if (a.scale != 1.0) {
                const T f = (T)a.scale;
                const T fi = a.conj_out ? -f : f;
#pragma unroll
                for (int m = 0; m < RHO; ++m) x[m] = mkc(v[m].x * f, v[m].y * fi);
            } else if (a.conj_out) {
#pragma unroll
                for (int m = 0; m < RHO; ++m) x[m] = mkc(v[m].x, -v[m].y);
            } else {
#pragma unroll
                for (int m = 0; m < RHO; ++m) x[m] = v[m];
            }
            if (a.hint_out == 2) {
#pragma unroll
                for (int m = 0; m < RHO; ++m) gstore(dst + m * sm_, x[m], 2);
            } else if (a.hint_out == 1) {
#pragma unroll
                for (int m = 0; m < RHO; ++m) gstore(dst + m * sm_, x[m], 1);
            } else {
#pragma unroll
                for (int m = 0; m < RHO; ++m) NFFT_GST(dst + m * sm_, x[m]);
            }
        } else if constexpr (STORE == ST_C2R) {
            // invrealdft output: each complex point is the real pair (2q, 2q+1);
            // one vector store per point when the line's reals are pair-aligned
            constexpr int lns = lns_of<S>();
            const long long q0 = base + ((long long)out_pos<S>(i, 0) << logNso), qs = 1ll << (lns + logNso);
            T* y = (T*)a.out + ln.bout;
            const T f = (T)a.scale;
            const T fi = a.conj_out ? -f : f;
            if (a.out_estride == 1 && ((uintptr_t)y & (sizeof(C2<T>) - 1)) == 0) {
                C2<T>* dst = (C2<T>*)y + q0;
#pragma unroll
                for (int m = 0; m < RHO; ++m) NFFT_GST(dst + m * qs, mkc(v[m].x * f, v[m].y * fi));
            } else {
#pragma unroll
                for (int m = 0; m < RHO; ++m)
                    store_elem<T, STORE>(a, tw, ln.bout, q0 + m * qs, v[m]);
            }
        } else if constexpr (STORE == ST_BLUE) {
            // last pass of the inverse M-point FFT: window [0, N), back from the
            // conjugated domain, chirp postmultiply, scale; positions q step by
            // 2^(lns + logNso) per m.  Table loads issued before the stores.
            constexpr int lns = lns_of<S>();
            const long long q0 = base + ((long long)out_pos<S>(i, 0) << logNso), qs = 1ll << (lns + logNso);
            const C2<T>* ch = (const C2<T>*)a.chirp + q0;
            C2<T>* dst = (C2<T>*)a.out + ln.bout + q0 * a.out_estride;
            const long long ds = qs * a.out_estride;
            C2<T> c[RHO];
#pragma unroll
            for (int m = 0; m < RHO; ++m) c[m] = q0 + m * qs < a.N ? gload_keep(ch + m * qs) : mkc((T)0, (T)0);
            const T f = (T)a.scale;
            const T fi = a.conj_out ? -f : f;
#pragma unroll
            for (int m = 0; m < RHO; ++m) {
                if (q0 + m * qs >= a.N) continue;
                const C2<T> w = cmul(cconj(v[m]), c[m]);
                NFFT_GST(dst + m * ds, mkc(w.x * f, w.y * fi));
            }
        } else {
#pragma unroll
            for (int m = 0; m < RHO; ++m)
                store_elem<T, STORE>(a, tw, ln.bout, base + ((long long)out_pos<S>(i, m) << logNso), v[m]);
        }
    }
};

template <typename T, int LOGR, int LOGT, bool COL_IN, bool COL_OUT, int LOAD, int STORE>
constexpr size_t lean_smem_bytes() {
    using L = Lean<T, LOGR, LOGT, COL_IN, COL_OUT, LOAD, STORE>;
    return sizeof(C2<T>) * (size_t)L::SMEM_ELEMS + sizeof(LeanLine) * (size_t)L::J;
}

// Mirror tile unpack, the items of thread t: (J/2 low lines) x R items, each
// emitting bins k and M - k; lines fastest, so neighbouring threads write
// neighbouring bins.  A thread's items share one line and step r by
// D = THREADS / (J/2), so k steps by D ns and the twiddles follow exactly
// known ratios: W_N^{k + D ns} = W_N^k W_{2R}^D and e^{-i pi (k + D ns) / 2N} =
// e^{-i pi k / 2N} W_{8R}^D (N = 2 ns R) -- chains of at most 8 products from
// one table twiddle.  The self-paired line 0 of tile 0 (bins r ns, then ns/2 +
// r ns) takes its twiddles from the table.
template <typename L, typename T, int STORE>
NFFT_HD void mirror_unpack_thread(const PassArgs& a, const TwTables<T>* tw, const C2<T>* sm, const LeanLine* lines,
                                  long long tile, int t) {
    using V = C2<T>;
    constexpr int LOGR = L::LOGR_;
    constexpr int R = 1 << LOGR;
    constexpr int H = L::J / 2;
    constexpr int ITEMS = H << LOGR;
    static_assert(L::THREADS % H == 0, "a thread's items share one line");
    constexpr int D = L::THREADS / H;
    const long long ns = 1ll << a.logNj, tpt = ns >> L::LOGJ;
    const long long tt = tile - (tile / tpt) * tpt;
    const long long M = ns << LOGR;
    const int l = t & (H - 1);
    const LeanLine ln = lines[l];
    auto zget = [&](long long q) {
        const long long j = q & (ns - 1);
        const int rr = (int)(q >> a.logNj);
        return sm[NFFT_SM((lean_idx<true, LOGR, L::LOGJ>(mirror_local(tt, j, L::J, ns), rr)))];
    };
    if (tt == 0 && l == 0) {
        for (int w = t; w < ITEMS; w += L::THREADS)
            unpack_pair<T, STORE>(a, tw, ln.bout, mirror_item_k(tt, l, w >> (L::LOGJ - 1), R, ns, ln.j), M, zget);
        return;
    }
    const V ws = twiddle<T>(tw, (uint64_t)D, LOGR + 1);   // W_{2R}^D
    V ts = V{};
    if constexpr (STORE == ST_T2) ts = twiddle<T>(tw, (uint64_t)D, LOGR + 3);   // W_{8R}^D
    // bin k = lowj + r ns is point r of the low line; bin M - k is point
    // R - 1 - r of its partner line ns - lowj: both local lines fixed per thread
    const int loc_lo = mirror_local(tt, ln.j, L::J, ns), loc_hi = mirror_local(tt, ns - ln.j, L::J, ns);
    auto zrow = [&](int line, int rr) { return sm[NFFT_SM((lean_idx<true, LOGR, L::LOGJ>(line, rr)))]; };
    V wk = V{}, tk = V{};
#pragma unroll
    for (int w = t; w < ITEMS; w += L::THREADS) {
        const int r = w >> (L::LOGJ - 1);
        const long long k = ln.j + (long long)r * ns;
        if (w == t) {
            wk = twiddle<T>(tw, (uint64_t)k, a.logN);
            if constexpr (STORE == ST_T2) tk = twiddle<T>(tw, (uint64_t)k, a.logN + 2);
        } else {
            wk = cmul(wk, ws);
            if constexpr (STORE == ST_T2) tk = cmul(tk, ts);
        }
        unpack_pair_tw_z<T, STORE>(a, tw, ln.bout, k, M, zrow(loc_lo, r), zrow(loc_hi, R - 1 - r), wk, tk);
    }
}

// Row-tile paired unpack (whole lines: realdft unpack / DCT-2 post pairs), the
// items of thread t: item w is the bin pair k, R - k (k = w mod (R/2)) of line
// w / (R/2), R the packed spectrum length.  With
// R/2 > THREADS a thread walks one line at a time with k stepping by THREADS
// (twiddles times the exact ratios W_N^THREADS and e^{-i pi THREADS / 2N}, at
// most 8 products per line); otherwise its k is the same on every line and the
// twiddles are reused.  Bin 0 (with bins M and M/2) goes through unpack_pair.
template <typename L, typename T, int STORE>
NFFT_HD void paired_unpack_thread(const PassArgs& a, const TwTables<T>* tw, const C2<T>* sm, const LeanLine* lines,
                                  int t) {
    using V = C2<T>;
    constexpr int LOGR = L::LOGR_;
    constexpr int HALF = LOGR == 0 ? 1 : (1 << (LOGR - 1));
    constexpr int ITEMS = L::J * HALF;
    V ws = V{}, ts = V{};
    if constexpr (HALF > L::THREADS) {
        ws = twiddle<T>(tw, (uint64_t)L::THREADS, a.logN);
        if constexpr (STORE == ST_T2) ts = twiddle<T>(tw, (uint64_t)L::THREADS, a.logN + 2);
    }
    V wk = V{}, tk = V{};
    int prevk = -1;
    for (int w = t; w < ITEMS; w += L::THREADS) {
        const int ll = w / HALF, k = w & (HALF - 1);
        const LeanLine ln = lines[ll];
        if (ln.j < 0) continue;
        auto zget = [&](long long r) { return sm[NFFT_SM((lean_idx<false, LOGR, L::LOGJ>(ll, (int)r)))]; };
        if (k == 0) {
            unpack_pair<T, STORE>(a, tw, ln.bout, 0, (long long)(1 << LOGR), zget);
            continue;
        }
        if (prevk < 0 || k < prevk) {
            wk = twiddle<T>(tw, (uint64_t)k, a.logN);
            if constexpr (STORE == ST_T2) tk = twiddle<T>(tw, (uint64_t)k, a.logN + 2);
        } else if (k != prevk) {
            wk = cmul(wk, ws);
            if constexpr (STORE == ST_T2) tk = cmul(tk, ts);
        }
        prevk = k;
        unpack_pair_tw<T, STORE>(a, tw, ln.bout, k, (long long)(1 << LOGR), zget, wk, tk);
    }
}

// Paired input repack of a row tile (PREPACK): the inverse-real repack
// p -> conj(s + i e^{+2 pi i p/N} d), s / d from the bins z_p and conj z_{M-p},
// for invrealdft (z = the input bins; bins 1 .. M-1 halved for the adjoint of
// realdft) and DCT-3 / DST-3 (z = the pre-twiddled reorder zb of the reals;
// zb_0 doubled for the adjoint of DCT-2 / DST-2).  Item (l, k), k = 0 .. M/2,
// of the tile's lines takes z_k and z_{M-k} once and writes points k and M - k
// of line l (W_N^{M-k} = -conj W_N^k and e^{-i pi (M-k)/2N} = e^{-i pi/4}
// conj e^{-i pi k/2N} exactly), where the generic operators compute both
// members of a pair for each point; items walk k fastest so neighbouring
// threads read neighbouring points.
template <typename L, typename T, int LOAD>
NFFT_HD void pair_prepack_thread(const PassArgs& a, const TwTables<T>* tw, C2<T>* sm, const LeanLine* lines, int t) {
    using V = C2<T>;
    constexpr int LOGR = L::LOGR_;
    constexpr int M = 1 << LOGR;
    constexpr int NI = M / 2 + 1;   // items per line
    const long long N = 2ll * M, es = a.in_estride;
    auto rep = [](V u, V v2, V w2) {
        const V b = cconj(v2);
        const V s2 = cadd(u, b), d = csub(u, b);
        const V od = cmulc(d, w2);
        return cconj(mkc(s2.x - od.y, s2.y + od.x));
    };
    for (int w = t; w < L::J * NI; w += L::THREADS) {
        const int l = w / NI, k = w - l * NI;
        const LeanLine ln = lines[l];
        auto put = [&](int p, V val) { sm[NFFT_SM((lean_idx<false, LOGR, L::LOGJ>(l, p)))] = val; };
        if (ln.j < 0) {
            put(k, mkc((T)0, (T)0));
            if (k > 0 && k < M / 2) put(M - k, mkc((T)0, (T)0));
            continue;
        }
        V zk, zm;
        if constexpr (LOAD == LD_IR) {
            const V* z = (const V*)a.in + ln.bin;
            zk = NFFT_GLD(&z[k * es]);
            zm = NFFT_GLD(&z[(M - k) * es]);
            if (a.vjp && k > 0) {
                zk = cscale(zk, (T)0.5);
                zm = cscale(zm, (T)0.5);
            }
        } else {
            const T* x = (const T*)a.in + ln.bin;
            if (k == 0) {
                zk = mkc(NFFT_GLD(&x[(a.dst ? N - 1 : 0) * es]), (T)0);
                zm = mkc((T)K<T>::r2 * (T)2 * NFFT_GLD(&x[(a.dst ? M - 1 : M) * es]), (T)0);
                if (a.vjp) zk = cscale(zk, (T)2);
            } else {
                const V tk = twiddle<T>(tw, (uint64_t)k, LOGR + 3);   // e^{-i pi k / 2N}
                const V tm = mkc((tk.x - tk.y) * K<T>::r2, -(tk.x + tk.y) * K<T>::r2);
                auto zb = [&](long long q, V tq) -> V {
                    const T xr = a.dst ? NFFT_GLD(&x[(N - q - 1) * es]) : NFFT_GLD(&x[q * es]);
                    const T xi = a.dst ? NFFT_GLD(&x[(q - 1) * es]) : NFFT_GLD(&x[(N - q) * es]);
                    return mkc(xr * tq.x - xi * tq.y, -xr * tq.y - xi * tq.x);
                };
                zk = zb(k, tk);
                zm = zb(M - k, tm);
            }
        }
        if (k == 0) {
            put(0, cconj(mkc(zk.x + zm.x, zk.x - zm.x)));
            continue;
        }
        const V wk = twiddle<T>(tw, (uint64_t)k, LOGR + 1);   // W_N^k
        put(k, rep(zk, zm, wk));
        if (k < M / 2) put(M - k, rep(zm, zk, mkc(-wk.x, wk.y)));
    }
}

// One tile of a specialized pass (all threads of the CTA call it; uniform
// early exit past the last line).
template <typename T, int LOGR, int LOGT, bool COL_IN, bool COL_OUT, int LOAD, int STORE>
__device__ __forceinline__ void lean_tile(const PassArgs& a, long long tile, unsigned char* smraw) {
    using L = Lean<T, LOGR, LOGT, COL_IN, COL_OUT, LOAD, STORE>;
    using V = C2<T>;
    V* sm = (V*)smraw;
    LeanLine* lines = (LeanLine*)(sm + L::SMEM_ELEMS);
    const TwTables<T>* tw = (const TwTables<T>*)a.tw;
    const int t = threadIdx.x;
    const long long line0 = tile << L::LOGJ;
    if (line0 >= a.nlines) return;
    if (t < L::J) {
        long long tmp[3];
        TileLines tl{&tmp[0], &tmp[1], &tmp[2]};
        if constexpr (L::MIRROR) {
            const long long ns = 1ll << a.logNj, tpt = ns >> L::LOGJ;   // lines, tiles per transform
            const long long tr = tile / tpt, tt = tile - tr * tpt;
            line_setup(a, tr * ns + mirror_line(tt, t, L::J, ns), 0, tl);
        } else {
            line_setup(a, line0 + t, 0, tl);
        }
        lines[t] = LeanLine{tmp[0], tmp[1], tmp[2]};
    }
    __syncthreads();

    V v[16];
    int l, i;
    if constexpr (L::PREPACK) {
        pair_prepack_thread<L, T, LOAD>(a, tw, sm, lines, t);
        __syncthreads();
        L::first_smem(a, tw, sm, lines, t, v, l, i);
        __syncthreads();   // every point read before the sub-stage writes
    } else {
        L::first(a, tw, lines, t, v, l, i);
    }
    if constexpr (L::NS == 1) {
        // single radix-16 sub-stage: the same thread stores its outputs
        if constexpr (L::PAIRED) {
            L::template write_smem<0>(sm, l, i, v);
        } else {
            L::template write_global<0>(a, tw, lines, l, i, v);
        }
    } else {
        L::template write_smem<0>(sm, l, i, v);
        __syncthreads();
        if constexpr (LOAD == LD_C && COL_IN && !L::MIRROR) {   // mirror tiles: lines are not one address run
            // every load of the tile has completed: drop the scratch lines just read
            constexpr int PER_LINE = 128 / (int)sizeof(V);
            if (a.discard_in && L::J >= PER_LINE && (l % PER_LINE) == 0) {
                const LeanLine ln = lines[l];
                if (ln.j >= 0) {
                    const V* src = (const V*)a.in + ln.bin + ln.j * a.in_estride;
                    const long long rs = a.in_estride << a.logNj;
#pragma unroll
                    for (int m = 0; m < 16; ++m) discard_l2(&src[(long long)(i + (m << (LOGR - 4))) * rs]);
                }
            }
        }
        // middle sub-stages (compile-time unrolled)
        if constexpr (L::NS >= 3) {
            constexpr int S = 1;
            constexpr int RHO = 1 << LeanSched<LOGR>::lr[S];
            V w[16];
            int ls[16 / RHO], is[16 / RHO];
#pragma unroll
            for (int q = 0; q < 16 / RHO; ++q) L::template read<S, L::COLL>(sm, t, q, &w[q * RHO], ls[q], is[q]);
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 16 / RHO; ++q) {
                L::template twiddle_dft<S>(tw, is[q], &w[q * RHO]);
                L::template write_smem<S>(sm, ls[q], is[q], &w[q * RHO]);
            }
            __syncthreads();
        }
        if constexpr (L::NS >= 4) {
            constexpr int S = 2;
            constexpr int RHO = 1 << LeanSched<LOGR>::lr[S];
            V w[16];
            int ls[16 / RHO], is[16 / RHO];
#pragma unroll
            for (int q = 0; q < 16 / RHO; ++q) L::template read<S, L::COLL>(sm, t, q, &w[q * RHO], ls[q], is[q]);
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 16 / RHO; ++q) {
                L::template twiddle_dft<S>(tw, is[q], &w[q * RHO]);
                L::template write_smem<S>(sm, ls[q], is[q], &w[q * RHO]);
            }
            __syncthreads();
        }
        // last sub-stage
        {
            constexpr int S = L::NS - 1;
            constexpr int RHO = 1 << LeanSched<LOGR>::lr[S];
            V w[16];
            int ls[16 / RHO], is[16 / RHO];
#pragma unroll
            for (int q = 0; q < 16 / RHO; ++q) L::template read<S, COL_OUT>(sm, t, q, &w[q * RHO], ls[q], is[q]);
            if constexpr (L::PAIRED) __syncthreads();
#pragma unroll
            for (int q = 0; q < 16 / RHO; ++q) {
                L::template twiddle_dft<S>(tw, is[q], &w[q * RHO]);
                if constexpr (L::PAIRED) L::template write_smem<S>(sm, ls[q], is[q], &w[q * RHO]);
                else L::template write_global<S>(a, tw, lines, ls[q], is[q], &w[q * RHO]);
            }
        }
    }
    if constexpr (L::MIRROR) {
        __syncthreads();
        mirror_unpack_thread<L, T, STORE>(a, tw, sm, lines, tile, t);
    } else if constexpr (L::PAIRED) {
        __syncthreads();
        paired_unpack_thread<L, T, STORE>(a, tw, sm, lines, t);
    }
}

// Minimum CTAs per SM the specialized kernels are compiled for (register
// budget 65536 / (threads x CTAs)).  The passes are latency-bound, so warps per
// SM matter: the float kernels fit in 64 registers and run 8 CTAs of 128
// threads per SM (measured on B200: +11% at 2^16, +29% at 4096 over 4 CTAs);
// the double kernels need their 128.
#ifndef NFFT_LEAN_MINB_T7_F64
#define NFFT_LEAN_MINB_T7_F64 4
#endif
#ifndef NFFT_LEAN_MINB_T7_F32
#define NFFT_LEAN_MINB_T7_F32 8
#endif
#ifndef NFFT_LEAN_MINB_T8_F64
#define NFFT_LEAN_MINB_T8_F64 2
#endif
#ifndef NFFT_LEAN_MINB_T8_F32
#define NFFT_LEAN_MINB_T8_F32 4
#endif
#ifndef NFFT_LEAN_MINB_T9_F32
#define NFFT_LEAN_MINB_T9_F32 2
#endif
template <typename T, int LOGT>
constexpr int lean_min_blocks() {
    return LOGT <= 7 ? (sizeof(T) == 4 ? NFFT_LEAN_MINB_T7_F32 : NFFT_LEAN_MINB_T7_F64)
                     : (LOGT == 8 ? (sizeof(T) == 4 ? NFFT_LEAN_MINB_T8_F32 : NFFT_LEAN_MINB_T8_F64)
                                  : (sizeof(T) == 4 ? NFFT_LEAN_MINB_T9_F32 : 1));
}

// Tile order of a standalone Bluestein filter-product pass (LD_FILT): the
// batch's transforms fastest, so the filter points one tile reads are read by
// the other transforms' tiles right after it (L2 hits instead of one filter
// sweep per transform).  A permutation of [0, tiles); identity for one
// transform or other line layouts.
NFFT_HD long long lean_batch_inner(const PassArgs& a, long long tile, int logJ) {
    if (a.ndims != 2 || a.jpos != 0 || a.cnt[1] <= 1) return tile;
    const long long tpt = a.cnt[0] >> logJ, B = a.cnt[1];
    if ((tpt << logJ) != a.cnt[0] || tile >= tpt * B) return tile;
    return (tile % B) * tpt + tile / B;
}

template <typename T, int LOGR, int LOGT, bool COL_IN, bool COL_OUT, int LOAD, int STORE>
__global__ void __launch_bounds__(1 << LOGT, (lean_min_blocks<T, LOGT>()))
lean_pass_kernel(const PassArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    long long tile = (long long)blockIdx.x + (long long)blockIdx.y * gridDim.x;
    if constexpr (LOAD == LD_FILT) tile = lean_batch_inner(a, tile, Lean<T, LOGR, LOGT, COL_IN, COL_OUT, LOAD, STORE>::LOGJ);
    lean_tile<T, LOGR, LOGT, COL_IN, COL_OUT, LOAD, STORE>(a, tile, smraw);
}

}  // namespace nfft

// nfft_pass.cuh -- the generic Stockham pass kernel.
//
// Every transform in the library is a sequence of passes.  A pass takes a
// power-of-two axis of length L = 2^logL, factored as L = Ns * R * Q, and
// performs radix-R "super-butterflies" of the self-sorting (Stockham, DIT)
// formulation for every line j in [0, L/R):
//
//     k  = j mod Ns
//     v_r = in[j + r (L/R)] * W_{Ns R}^{r k}          r in [0, R)
//     V  = DFT_R(v)
//     out[(j / Ns) Ns R + k + r Ns] = V_r
//
// Passes with Ns = 1, R1, R1 R2, ... compose to the full DFT with the output
// in natural order.  A CTA processes a tile of J lines x R elements: it loads
// the tile from global memory (applying the pass's pre-twiddle and the
// transform's fused input operator), runs the radix-R DFT as radix-16/8/4/2
// sub-stages in shared memory (each thread holds 16 points in registers per
// sub-stage), and stores the tile (applying the fused output operator).
// Lines are either J consecutive j of one axis (column mode: consecutive
// threads touch consecutive addresses across lines) or whole contiguous
// transforms (row mode: consecutive threads walk along a line).
#pragma once

#include "nfft_common.cuh"

namespace nfft {

// Fused input operators (how element p of the complex sequence is produced).
enum LoadOp : int {
    LD_C = 0,     // complex element, optional conjugation
    LD_T2 = 1,    // DCT-2/DST-2: even / reversed-odd reorder of N reals, packed as N/2 complex
    LD_T3 = 2,    // DCT-3/DST-3: pre-twiddle + inverse-real repack (conjugated for the inverse FFT)
    LD_IR = 3,    // invrealdft: repack of N/2+1 bins into N/2 complex (conjugated)
    LD_T4 = 4,    // DCT-4/DST-4: premultiply (x[2n] +- i x[N-1-2n]) by e^{-i pi n/N}
    LD_BLUE = 5,  // Bluestein: chirp premultiply, zero pad beyond N
    LD_R2C = 6,   // realdft: N reals read pairwise as N/2 complex (any alignment / stride)
    LD_BLUE_R = 7,   // Bluestein of N reals (realdft of any N): (x_p, 0) times the chirp
    LD_BLUE_T2 = 8,  // Bluestein DCT-2 of any N: even / reversed-odd reorder of N reals, times the chirp
    LD_FILT = 9,     // Bluestein: conj(spectrum * filter), the input of the inverse M-point FFT
};
// Fused output operators.
enum StoreOp : int {
    ST_C = 0,     // complex element, optional conjugation and scale
    ST_R = 1,     // realdft unpack (pairs k, M-k; whole line in the tile)
    ST_T2 = 2,    // DCT-2/DST-2 post-twiddle (pairs; whole line in the tile)
    ST_T3 = 3,    // DCT-3/DST-3 un-reorder of the real output
    ST_T4 = 4,    // DCT-4/DST-4 postmultiply
    ST_BLUE = 5,  // Bluestein: window [0, N), chirp postmultiply, scale
    ST_C2R = 6,   // invrealdft: complex element written as two reals (any alignment / stride)
    ST_BLUE_R = 7,   // Bluestein realdft of any N: bins 0 .. N/2 of the windowed, chirped output
    ST_BLUE_T2 = 8,  // Bluestein DCT-2 of any N: y_q = 2 Re(e^{-i pi q/2N} V_q), q < N
};
constexpr int NUM_LOAD_OPS = 10, NUM_STORE_OPS = 9;

constexpr int MAX_LINE_DIMS = 4;
constexpr int MAX_SUB = 4;
constexpr int MAX_J = 256;

struct PassArgs {
    const void* in;
    void* out;
    const void* tw;          // TwTables<T>*
    int logR, logNs, logNj;  // pass radix R, product of earlier radices, L/R
    int logNs_out;           // Ns used for the output position (0 after a fused middle FFT)
    int logJ;                // lines per tile
    int nsub;                // sub-stage count
    int sublog[MAX_SUB];     // log2 of each sub-stage radix
    int in_row, out_row;     // 1: walk along lines (contiguous elements) when loading / storing
    int ndims, jpos;         // line dims (innermost first); which one is j (-1: none)
    long long cnt[MAX_LINE_DIMS];
    long long istr[MAX_LINE_DIMS], ostr[MAX_LINE_DIMS];
    long long nlines;
    long long in_estride, out_estride;  // element stride along the axis (elements of the array type)
    int conj_in, conj_out;
    double scale;
    long long N;             // real length (real ops) or Bluestein length
    int logN;                // log2 N for the real operators
    int dst;                 // 1: the DST variant of the operator
    const void* chirp;       // Bluestein chirp e^{-i pi k^2/N}, k < N (C2<T>)
    const void* filt;        // Bluestein filter spectrum / M, natural order (C2<T>)
    int mid;                 // Bluestein middle pass: x filter, conj, second FFT
    int logM;                // log2 of the axis length for the fused middle pass
    int vjp;                 // adjoint weights (see the operators below)
    int hint_in, hint_out;   // L2 policy of the complex input / output (gload / gstore)
    int discard_in;          // input is scratch read for the last time: drop its L2 lines
    int tw_mode;             // pass pre-twiddles: 0 product tree, 1 chained products, 2 table lookups
    // Ragged batches: line dim tab_dim takes its input / output offset from a
    // per-index table (elements of the array type) instead of index * stride.
    const long long* in_tab;
    const long long* out_tab;
    int tab_dim;
    const void* post;        // Bluestein DCT-2 post-twiddle e^{-i pi q / 2N}, q < N (C2<T>)
};

// Shared-memory index with one padding element every 16 (breaks the
// power-of-two strides of the sub-stage writes across banks).
NFFT_HD int spad(int i) { return i + (i >> 4); }

template <typename T, int OP>
NFFT_HD C2<T> load_elem(const PassArgs& a, const TwTables<T>* tw, long long base, long long p) {
    using V = C2<T>;
    if constexpr (OP == LD_C) {
        V v = NFFT_GLD(&((const V*)a.in)[base + p * a.in_estride]);
        if (a.conj_in) v.y = -v.y;
        return v;
    } else if constexpr (OP == LD_BLUE) {
        if (p >= a.N) return mkc((T)0, (T)0);
        V v = NFFT_GLD(&((const V*)a.in)[base + p * a.in_estride]);
        if (a.conj_in) v.y = -v.y;
        return cmul(v, gload_keep(&((const V*)a.chirp)[p]));
    } else if constexpr (OP == LD_BLUE_R || OP == LD_BLUE_T2) {
        if (p >= a.N) return mkc((T)0, (T)0);
        const T* x = (const T*)a.in + base;
        const long long es = a.in_estride;
        T r;
        if constexpr (OP == LD_BLUE_R) r = NFFT_GLD(&x[p * es]);
        else r = (p < (a.N + 1) / 2) ? NFFT_GLD(&x[(2 * p) * es]) : NFFT_GLD(&x[(2 * a.N - 1 - 2 * p) * es]);
        return cscale(gload_keep(&((const V*)a.chirp)[p]), r);
    } else if constexpr (OP == LD_FILT) {
        const V v = NFFT_GLD(&((const V*)a.in)[base + p * a.in_estride]);
        return cconj(cmul(v, gload_keep(&((const V*)a.filt)[p])));
    } else if constexpr (OP == LD_R2C) {
        const T* x = (const T*)a.in + base;
        const long long es = a.in_estride;
        return mkc(NFFT_GLD(&x[(2 * p) * es]), NFFT_GLD(&x[(2 * p + 1) * es]));
    } else if constexpr (OP == LD_T2) {
        // z[p] = (v[2p], v[2p+1]),  v[i] = x[2i] (i < N/2),  v[i] = s x[2N-1-2i] otherwise
        const T* x = (const T*)a.in + base;
        const long long es = a.in_estride, N = a.N;
        auto vget = [&](long long i) -> T {
            if (i < N / 2) return NFFT_GLD(&x[(2 * i) * es]);
            T t = NFFT_GLD(&x[(2 * N - 1 - 2 * i) * es]);
            return a.dst ? -t : t;
        };
        return mkc(vget(2 * p), vget(2 * p + 1));
    } else if constexpr (OP == LD_T4) {
        const T* x = (const T*)a.in + base;
        const long long es = a.in_estride, N = a.N;
        T xe = NFFT_GLD(&x[(2 * p) * es]), xo = NFFT_GLD(&x[(N - 1 - 2 * p) * es]);
        V e = twiddle<T>(tw, (uint64_t)p, a.logN + 1);   // e^{-i pi p / N}
        if (!a.dst) return mkc(e.x * xe - e.y * xo, e.x * xo + e.y * xe);
        return mkc(-e.x * xe - e.y * xo, e.x * xo - e.y * xe);
    } else {
        // LD_IR / LD_T3: inverse-real repack of bins z[p], z[M-p] (M = N/2):
        //   ibuf_0 = (Re z_0 + Re z_M) + i (Re z_0 - Re z_M)
        //   ibuf_k = s + i e^{+2 pi i k/N} d,  s = z_k + conj z_{M-k},  d = z_k - conj z_{M-k}
        // returned conjugated (the N/2-point inverse FFT runs as conj(FFT(conj .))).
        const long long N = a.N, M = N / 2;
        V zk, zm;
        if constexpr (OP == LD_IR) {
            const V* z = (const V*)a.in + base;
            const long long es = a.in_estride;
            zk = NFFT_GLD(&z[p * es]);
            zm = NFFT_GLD(&z[(M - p) * es]);
            if (a.vjp) {
                // adjoint of realdft = invrealdft of the cotangent with bins 1..M-1 halved
                if (p > 0 && p < M) zk = cscale(zk, (T)0.5);
                if (M - p > 0 && M - p < M) zm = cscale(zm, (T)0.5);
            }
        } else {
            // DCT-3/DST-3 pre-twiddle: zb_k = (xr tw.re - xi tw.im, -xr tw.im - xi tw.re),
            // tw = e^{-i pi k / 2N};  zb_0 = (x_0, 0), zb_M = (sqrt2 x_M, 0)  (DST reads x reversed)
            const T* x = (const T*)a.in + base;
            const long long es = a.in_estride;
            auto zb = [&](long long k) -> V {
                if (k == 0) return mkc(NFFT_GLD(&x[(a.dst ? N - 1 : 0) * es]), (T)0);
                if (k == M) return mkc((T)K<T>::r2 * (T)2 * NFFT_GLD(&x[(a.dst ? M - 1 : M) * es]), (T)0);
                T xr = a.dst ? NFFT_GLD(&x[(N - k - 1) * es]) : NFFT_GLD(&x[k * es]);
                T xi = a.dst ? NFFT_GLD(&x[(k - 1) * es]) : NFFT_GLD(&x[(N - k) * es]);
                V t = twiddle<T>(tw, (uint64_t)k, a.logN + 2);
                return mkc(xr * t.x - xi * t.y, -xr * t.y - xi * t.x);
            };
            zk = zb(p);
            zm = zb(M - p);
            if (a.vjp) {
                // adjoint of DCT-2 / DST-2 = DCT-3 / DST-3 of the cotangent with x_0 (x_{N-1}) doubled
                if (p == 0) zk = cscale(zk, (T)2);
                if (M - p == 0) zm = cscale(zm, (T)2);
            }
        }
        V r;
        if (p == 0) {
            r = mkc(zk.x + zm.x, zk.x - zm.x);
        } else {
            V b = cconj(zm);
            V s = cadd(zk, b), d = csub(zk, b);
            V od = cmulc(d, twiddle<T>(tw, (uint64_t)p, a.logN));   // d * e^{+2 pi i p/N}
            r = mkc(s.x - od.y, s.y + od.x);
        }
        return cconj(r);
    }
}

// Element-wise output operators (ST_C, ST_T3, ST_T4, ST_BLUE).  q is the
// element's position along the complex output sequence.
template <typename T, int OP>
NFFT_HD void store_elem(const PassArgs& a, const TwTables<T>* tw, long long base, long long q, C2<T> v) {
    using V = C2<T>;
    if constexpr (OP == ST_C) {
        if (a.conj_out) v.y = -v.y;
        if (a.scale != 1.0) v = cscale(v, (T)a.scale);
        NFFT_GST(&((V*)a.out)[base + q * a.out_estride], v);
    } else if constexpr (OP == ST_C2R) {
        if (a.conj_out) v.y = -v.y;
        if (a.scale != 1.0) v = cscale(v, (T)a.scale);
        T* y = (T*)a.out + base;
        NFFT_GST(&y[(2 * q) * a.out_estride], v.x);
        NFFT_GST(&y[(2 * q + 1) * a.out_estride], v.y);
    } else if constexpr (OP == ST_BLUE) {
        if (q >= a.N) return;
        v = cconj(v);                                  // leave the conjugated inverse-FFT domain
        v = cmul(v, gload_keep(&((const V*)a.chirp)[q]));
        if (a.conj_out) v.y = -v.y;
        if (a.scale != 1.0) v = cscale(v, (T)a.scale);
        NFFT_GST(&((V*)a.out)[base + q * a.out_estride], v);
    } else if constexpr (OP == ST_BLUE_R) {
        if (q > a.N / 2) return;
        v = cmul(cconj(v), gload_keep(&((const V*)a.chirp)[q]));
        if (a.scale != 1.0) v = cscale(v, (T)a.scale);
        NFFT_GST(&((V*)a.out)[base + q * a.out_estride], v);
    } else if constexpr (OP == ST_BLUE_T2) {
        if (q >= a.N) return;
        v = cmul(cconj(v), gload_keep(&((const V*)a.chirp)[q]));
        const V w = NFFT_GLD(&((const V*)a.post)[q]);
        T y = (T)2 * (v.x * w.x - v.y * w.y);
        if (a.scale != 1.0) y = (T)(y * a.scale);
        NFFT_GST(&((T*)a.out)[base + q * a.out_estride], y);
    } else if constexpr (OP == ST_T3) {
        // real output t[2q], t[2q+1] of the inverse FFT -> y[2i] = t_i, y[N-1-2i] = +-t_{N/2+i}
        v = cconj(v);
        T* y = (T*)a.out + base;
        const long long es = a.out_estride, N = a.N;
        T vals[2] = {v.x, v.y};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            long long t = 2 * q + h;
            if (t < N / 2) NFFT_GST(&y[(2 * t) * es], vals[h]);
            else NFFT_GST(&y[(2 * N - 1 - 2 * t) * es], a.dst ? -vals[h] : vals[h]);
        }
    } else if constexpr (OP == ST_T4) {
        // y[2q] = 2 Re(f(2q) t_q), y[N-1-2q] = 2 Re(f(N-1-2q) conj t_q), f(n) = e^{-i pi (2n+1)/4N}
        // (Im instead of Re for DST-4)
        T* y = (T*)a.out + base;
        const long long es = a.out_estride, N = a.N;
        V f0 = twiddle<T>(tw, (uint64_t)(4 * q + 1), a.logN + 3);
        // f(N-1-2q) = e^{-i pi / 2} conj f(2q) exactly
        V f1 = mkc(-f0.y, -f0.x);
        V c = cconj(v);
        T y0, y1;
        if (!a.dst) {
            y0 = (T)2 * (f0.x * v.x - f0.y * v.y);
            y1 = (T)2 * (f1.x * c.x - f1.y * c.y);
        } else {
            y0 = (T)2 * (f0.x * v.y + f0.y * v.x);
            y1 = (T)2 * (f1.x * c.y + f1.y * c.x);
        }
        NFFT_GST(&y[(2 * q) * es], y0);
        NFFT_GST(&y[(N - 1 - 2 * q) * es], y1);
    }
}

// realdft bin from the packed N/2-point spectrum: X_k = s + (-i) W_N^k d,
// s = (a + conj b)/2, d = (a - conj b)/2, a = Z_k, b = Z_{M-k}.
template <typename T>
NFFT_HD C2<T> real_unpack(C2<T> a, C2<T> b, C2<T> w) {
    C2<T> bb = cconj(b);
    C2<T> s = cscale(cadd(a, bb), (T)0.5), d = cscale(csub(a, bb), (T)0.5);
    C2<T> od = cmul(d, w);
    return mkc(s.x + od.y, s.y - od.x);
}

// Emit realdft bin k (0 <= k <= M) as ST_R (complex bin) or ST_T2 (DCT-2 /
// DST-2 outputs derived from the bin; t = e^{-i pi k / 2N} for 0 < k < M).
template <typename T, int OP>
NFFT_HD void emit_bin(const PassArgs& a, const TwTables<T>* tw, long long base, long long k, C2<T> X,
                      C2<T> t = C2<T>{}) {
    using V = C2<T>;
    const long long N = a.N, M = N / 2;
    if constexpr (OP == ST_R) {
        // adjoint of invrealdft = realdft of the cotangent with bins 1..M-1 doubled
        if (a.vjp && k > 0 && k < M) X = cscale(X, (T)2);
        NFFT_GST(&((V*)a.out)[base + k * a.out_estride], X);
    } else {
        T* y = (T*)a.out + base;
        const long long es = a.out_estride;
        if (k == 0) {
            // adjoint of DCT-3 / DST-3 = DCT-2 / DST-2 with output 0 (N-1) halved
            NFFT_GST(&y[(a.dst ? N - 1 : 0) * es], a.vjp ? X.x : (T)2 * X.x);
        } else if (k == M) {
            NFFT_GST(&y[(a.dst ? M - 1 : M) * es], (T)2 * K<T>::r2 * X.x);
        } else {
            (void)tw;
            T c = (T)2 * (X.x * t.x - X.y * t.y);
            T s = (T)-2 * (X.x * t.y + X.y * t.x);
            if (!a.dst) { NFFT_GST(&y[k * es], c); NFFT_GST(&y[(N - k) * es], s); }
            else { NFFT_GST(&y[(k - 1) * es], s); NFFT_GST(&y[(N - k - 1) * es], c); }
        }
    }
}

// Bins k and M - k (0 < k < M/2... M - 1) from their twiddles: w = W_N^k and,
// for ST_T2, t = e^{-i pi k / 2N}.  W_N^{M-k} = -conj(W_N^k) exactly (W_N^M =
// -1) and e^{-i pi (M-k) / 2N} = e^{-i pi / 4} conj(t): one twiddle per pair.
template <typename T, int OP>
NFFT_HD void unpack_pair_tw_z(const PassArgs& a, const TwTables<T>* tw, long long base, long long k, long long M,
                              C2<T> zk, C2<T> zm, C2<T> w, C2<T> t) {
    using V = C2<T>;
    const V wm = mkc(-w.x, w.y);
    V tm = V{};
    if constexpr (OP == ST_T2) tm = mkc((t.x - t.y) * K<T>::r2, -(t.x + t.y) * K<T>::r2);
    emit_bin<T, OP>(a, tw, base, k, real_unpack<T>(zk, zm, w), t);
    emit_bin<T, OP>(a, tw, base, M - k, real_unpack<T>(zm, zk, wm), tm);
}
template <typename T, int OP, typename Get>
NFFT_HD void unpack_pair_tw(const PassArgs& a, const TwTables<T>* tw, long long base, long long k, long long M,
                            Get zget, C2<T> w, C2<T> t) {
    unpack_pair_tw_z<T, OP>(a, tw, base, k, M, zget(k), zget(M - k), w, t);
}

// Paired unpack of one line's packed spectrum Z (M = N/2 complex values read
// through zget(i)) for work item k in [0, M/2): bins k and M-k (k = 0 also
// emits bins M and M/2).
template <typename T, int OP, typename Get>
NFFT_HD void unpack_pair(const PassArgs& a, const TwTables<T>* tw, long long base, long long k, long long M, Get zget) {
    using V = C2<T>;
    if (k == 0) {
        V z0 = zget(0);
        emit_bin<T, OP>(a, tw, base, 0, mkc(z0.x + z0.y, (T)0));
        emit_bin<T, OP>(a, tw, base, M, mkc(z0.x - z0.y, (T)0));
        if (M >= 2) {
            V zh = zget(M / 2);
            // bin M/2 = N/4: post-twiddle e^{-i pi / 8}
            emit_bin<T, OP>(a, tw, base, M / 2, mkc(zh.x, -zh.y), mkc(K<T>::c8, -K<T>::s8));
        }
    } else {
        const V w = twiddle<T>(tw, (uint64_t)k, a.logN);
        V t = V{};
        if constexpr (OP == ST_T2) t = twiddle<T>(tw, (uint64_t)k, a.logN + 2);
        unpack_pair_tw<T, OP>(a, tw, base, k, M, zget, w, t);
    }
}

// ---------------------------------------------------------------------------
// Per-thread phases of the pass kernel.  Each is a host+device function of
// (tile state, thread or slot index) so the kernel below and the test-only
// CPU emulator execute the same index arithmetic; the kernel separates the
// phases with __syncthreads, the emulator runs each phase for every thread
// before the next.
// ---------------------------------------------------------------------------
#ifdef NFFT_EMULATE
__host__ __device__ void nfft_emu_smem_check(int idx);
#define NFFT_SM(i) (nfft_emu_smem_check(i), (i))
#else
#define NFFT_SM(i) (i)
#endif

struct TileLines {
    long long* in;   // batch offset of each line in the input (elements)
    long long* out;  // batch offset in the output
    long long* j;    // Stockham line index along the axis, -1 past the end
};

// Decompose global line lam over the line dims.
NFFT_HD void line_setup(const PassArgs& a, long long lam, int l, TileLines tl) {
    long long bin = 0, bout = 0, j = 0;
    if (lam < a.nlines) {
        long long rem = lam;
        for (int d = 0; d < a.ndims; ++d) {
            long long c = rem % a.cnt[d];
            rem /= a.cnt[d];
            if (d == a.jpos) {
                j = c;
            } else {
                bin += (d == a.tab_dim && a.in_tab) ? NFFT_GLD(&a.in_tab[c]) : c * a.istr[d];
                bout += (d == a.tab_dim && a.out_tab) ? NFFT_GLD(&a.out_tab[c]) : c * a.ostr[d];
            }
        }
    } else {
        j = -1;
    }
    tl.in[l] = bin;
    tl.out[l] = bout;
    tl.j[l] = j;
}

// Load of tile slot e (0 <= e < J R): the fused input operator's value.  The
// kernel issues the loads of all its slots before consuming any of them.
template <typename T, int LOAD>
NFFT_HD C2<T> load_slot_value(const PassArgs& a, const TwTables<T>* tw, TileLines tl, int e) {
    const int logR = a.logR, logJ = a.logJ;
    int l, r;
    if (a.in_row) { l = e >> logR; r = e & ((1 << logR) - 1); }
    else { l = e & ((1 << logJ) - 1); r = e >> logJ; }
    long long j = tl.j[l];
    if (j < 0) return mkc((T)0, (T)0);
    long long p = j + ((long long)r << a.logNj);
    return load_elem<T, LOAD>(a, tw, tl.in[l], p);
}

// Pass pre-twiddle W_{Ns R}^{r k} of slot e and its store into shared memory.
template <typename T>
NFFT_HD void load_slot_commit(const PassArgs& a, const TwTables<T>* tw, C2<T>* sm, TileLines tl, int e, C2<T> v) {
    const int logR = a.logR, logJ = a.logJ;
    int l, r;
    if (a.in_row) { l = e >> logR; r = e & ((1 << logR) - 1); }
    else { l = e & ((1 << logJ) - 1); r = e >> logJ; }
    if (a.logNs > 0) {
        long long j = tl.j[l];
        long long k = j & ((1ll << a.logNs) - 1);
        if (j >= 0 && k) v = cmul(v, twiddle<T>(tw, (uint64_t)r * (uint64_t)k, a.logNs + logR));
    }
    sm[NFFT_SM(spad((l << logR) + r))] = v;
}

// Sub-stage of radix RHO = 2^LR: read phase (16 points per thread into v).
template <typename T, int THREADS, int RHO, int LR>
NFFT_HD void substage_read(const C2<T>* sm, C2<T>* v, int logR, int logE, int tid) {
    constexpr int NB = 16 / RHO;
    const int nbf = 1 << (logE - LR);
    const int lq = logR - LR;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        int b = tid + q * THREADS;
        if (b < nbf) {
            int l = b >> lq, i = b & ((1 << lq) - 1);
            int base = (l << logR) + i;
#pragma unroll
            for (int m = 0; m < RHO; ++m) v[q * RHO + m] = sm[NFFT_SM(spad(base + (m << lq)))];
        }
    }
}

// Sub-stage write phase: twiddle W_{ns RHO}^{m k}, radix-RHO DFT, Stockham store.
template <typename T, int THREADS, int RHO, int LR>
NFFT_HD void substage_write(C2<T>* sm, C2<T>* v, const TwTables<T>* tw, int logR, int logE, int lns, int tid) {
    constexpr int NB = 16 / RHO;
    const int nbf = 1 << (logE - LR);
    const int lq = logR - LR;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        int b = tid + q * THREADS;
        if (b < nbf) {
            int l = b >> lq, i = b & ((1 << lq) - 1);
            int k = i & ((1 << lns) - 1);
            if (lns > 0) {
#pragma unroll
                for (int m = 1; m < RHO; ++m) {
                    C2<T> w = (lns + LR <= TW_BITS) ? twiddle_small<T>(tw, (uint32_t)(m * k), lns + LR)
                                                    : twiddle<T>(tw, (uint64_t)(m * k), lns + LR);
                    v[q * RHO + m] = cmul(v[q * RHO + m], w);
                }
            }
            dft_radix<T, RHO>(&v[q * RHO]);
            int o = (l << logR) + ((i >> lns) << (lns + LR)) + k;
#pragma unroll
            for (int m = 0; m < RHO; ++m) sm[NFFT_SM(spad(o + (m << lns)))] = v[q * RHO + m];
        }
    }
}

// Bluestein middle step for slot e: multiply by the filter spectrum at the
// forward output position, conjugate (the inverse FFT runs as conj(FFT(conj))).
template <typename T>
NFFT_HD void mid_slot(const PassArgs& a, C2<T>* sm, TileLines tl, int e) {
    const int logR = a.logR, logNs = a.logNs;
    int l = e >> logR, r = e & ((1 << logR) - 1);
    long long j = tl.j[l];
    if (j < 0) return;
    long long q = ((j >> logNs) << (logNs + logR)) + (j & ((1ll << logNs) - 1)) + ((long long)r << logNs);
    C2<T> v = sm[NFFT_SM(spad(e))];
    sm[NFFT_SM(spad(e))] = cconj(cmul(v, gload_keep(&((const C2<T>*)a.filt)[q])));
}

// Store tile slot e with an element-wise output operator.
template <typename T, int STORE>
NFFT_HD void store_slot(const PassArgs& a, const TwTables<T>* tw, const C2<T>* sm, TileLines tl, int e) {
    const int logR = a.logR, logJ = a.logJ, logNso = a.logNs_out;
    int l, r;
    if (a.out_row) { l = e >> logR; r = e & ((1 << logR) - 1); }
    else { l = e & ((1 << logJ) - 1); r = e >> logJ; }
    long long j = tl.j[l];
    if (j < 0) return;
    C2<T> v = sm[NFFT_SM(spad((l << logR) + r))];
    long long q = ((j >> logNso) << (logNso + logR)) + (j & ((1ll << logNso) - 1)) + ((long long)r << logNso);
    store_elem<T, STORE>(a, tw, tl.out[l], q, v);
}

// Paired store (realdft unpack / DCT-2 post) of work item w; whole lines.
template <typename T, int STORE>
NFFT_HD void paired_slot(const PassArgs& a, const TwTables<T>* tw, const C2<T>* sm, TileLines tl, int w) {
    const int logR = a.logR, R = 1 << logR;
    int l, k;
    if (R == 1) { l = w; k = 0; }
    else { l = w >> (logR - 1); k = w & ((R >> 1) - 1); }
    if (tl.j[l] < 0) return;
    const int lb = l << logR;
    unpack_pair<T, STORE>(a, tw, tl.out[l], k, (long long)R, [&](long long i) { return sm[NFFT_SM(spad(lb + (int)i))]; });
}

NFFT_HD int paired_items(const PassArgs& a) {
    return a.logR == 0 ? (1 << a.logJ) : (1 << (a.logJ + a.logR - 1));
}

template <typename T, int THREADS>
__device__ __forceinline__ void tile_fft(C2<T>* sm, const TwTables<T>* tw, const PassArgs& a, int logE, int tid) {
    int lns = 0;
    C2<T> v[16];
    for (int s = 0; s < a.nsub; ++s) {
        int lr = a.sublog[s];
        switch (lr) {
        case 4: substage_read<T, THREADS, 16, 4>(sm, v, a.logR, logE, tid); break;
        case 3: substage_read<T, THREADS, 8, 3>(sm, v, a.logR, logE, tid); break;
        case 2: substage_read<T, THREADS, 4, 2>(sm, v, a.logR, logE, tid); break;
        default: substage_read<T, THREADS, 2, 1>(sm, v, a.logR, logE, tid); break;
        }
        __syncthreads();
        switch (lr) {
        case 4: substage_write<T, THREADS, 16, 4>(sm, v, tw, a.logR, logE, lns, tid); break;
        case 3: substage_write<T, THREADS, 8, 3>(sm, v, tw, a.logR, logE, lns, tid); break;
        case 2: substage_write<T, THREADS, 4, 2>(sm, v, tw, a.logR, logE, lns, tid); break;
        default: substage_write<T, THREADS, 2, 1>(sm, v, tw, a.logR, logE, lns, tid); break;
        }
        __syncthreads();
        lns += lr;
    }
}

// Shared memory of a pass kernel with a tile of 2^log_tile points: the padded
// tile plus three per-line arrays of MAX_J entries.
template <typename T> constexpr size_t pass_smem_elems(int log_tile) {
    return (size_t)((1 << log_tile) + (1 << (log_tile - 4)) + 1);
}
template <typename T> constexpr size_t pass_smem_bytes(int log_tile) {
    return sizeof(C2<T>) * pass_smem_elems<T>(log_tile) + (size_t)MAX_J * 3 * sizeof(long long);
}

// One tile of the generic pass (all threads of the CTA call it; uniform early
// exit past the last line).
template <typename T, int LOG_TILE, int LOAD, int STORE>
__device__ __forceinline__ void pass_tile(const PassArgs& a, long long tile, unsigned char* smraw) {
    using V = C2<T>;
    constexpr int THREADS = (1 << LOG_TILE) / 16;
    V* sm = (V*)smraw;
    TileLines tl;
    tl.in = (long long*)(sm + pass_smem_elems<T>(LOG_TILE));
    tl.out = tl.in + MAX_J;
    tl.j = tl.out + MAX_J;
    const TwTables<T>* tw = (const TwTables<T>*)a.tw;

    const int tid = threadIdx.x;
    const int logE = a.logR + a.logJ;
    const int J = 1 << a.logJ, E = 1 << logE;
    const long long line0 = tile << a.logJ;
    if (line0 >= a.nlines) return;

    for (int l = tid; l < J; l += THREADS) line_setup(a, line0 + l, l, tl);
    __syncthreads();
    {
        // all global loads of the slot set in flight before any is consumed
        V buf[16];
#pragma unroll
        for (int it = 0; it < 16; ++it) {
            int e = tid + it * THREADS;
            if (e < E) buf[it] = load_slot_value<T, LOAD>(a, tw, tl, e);
        }
#pragma unroll
        for (int it = 0; it < 16; ++it) {
            int e = tid + it * THREADS;
            if (e < E) load_slot_commit<T>(a, tw, sm, tl, e, buf[it]);
        }
    }
    __syncthreads();
    tile_fft<T, THREADS>(sm, tw, a, logE, tid);
    if (a.mid) {
        for (int it = 0; it < 16; ++it) {
            int e = tid + it * THREADS;
            if (e >= E) break;
            mid_slot<T>(a, sm, tl, e);
        }
        __syncthreads();
        tile_fft<T, THREADS>(sm, tw, a, logE, tid);
    }
    if constexpr (STORE == ST_R || STORE == ST_T2) {
        const int items = paired_items(a);
        for (int w = tid; w < items; w += THREADS) paired_slot<T, STORE>(a, tw, sm, tl, w);
    } else {
#pragma unroll
        for (int it = 0; it < 16; ++it) {
            int e = tid + it * THREADS;
            if (e < E) store_slot<T, STORE>(a, tw, sm, tl, e);
        }
    }
}

template <typename T, int LOG_TILE, int LOAD, int STORE>
__global__ void __launch_bounds__((1 << LOG_TILE) / 16)
pass_kernel(const PassArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    pass_tile<T, LOG_TILE, LOAD, STORE>(a, (long long)blockIdx.x + (long long)blockIdx.y * gridDim.x, smraw);
}

// Paired-unpack epilogue for transforms whose packed spectrum needed more
// than one pass: reads Z (M complex per line, contiguous, line distance zdist)
// and writes realdft bins or DCT-2/DST-2 outputs.
// Per-item body of the unpack epilogue (host+device, see the pass kernel).
template <typename T, int STORE>
NFFT_HD void unpack_item(const PassArgs& a, const TwTables<T>* tw, const C2<T>* Z, long long zdist, long long w) {
    const long long M = a.N / 2;
    const long long per = M >= 2 ? M / 2 : 1;
    long long line = w / per, k = w - line * per;
    long long rem = line, bout = 0;
    for (int d = 0; d < a.ndims; ++d) {
        long long c = rem % a.cnt[d];
        rem /= a.cnt[d];
        bout += (d == a.tab_dim && a.out_tab) ? NFFT_GLD(&a.out_tab[c]) : c * a.ostr[d];
    }
    const C2<T>* zl = Z + line * zdist;
    unpack_pair<T, STORE>(a, tw, bout, k, M, [&](long long i) { return NFFT_GLD(&zl[i]); });
}

// Work items of one unpack tile: chunk `chunk` (UNPACK_TILE items) of one line.
constexpr int UNPACK_TILE = 2048;
NFFT_HD long long unpack_per_line(const PassArgs& a) { return (a.N / 2) >= 2 ? a.N / 4 : 1; }
NFFT_HD long long unpack_tiles_per_line(const PassArgs& a) {
    return (unpack_per_line(a) + UNPACK_TILE - 1) / UNPACK_TILE;
}
NFFT_HD void unpack_tile_range(const PassArgs& a, long long tile, long long& w0, long long& w1) {
    const long long per = unpack_per_line(a), tpl = unpack_tiles_per_line(a);
    const long long line = tile / tpl, chunk = tile - line * tpl;
    w0 = line * per + chunk * UNPACK_TILE;
    w1 = w0 + UNPACK_TILE;
    if (w1 > (line + 1) * per) w1 = (line + 1) * per;
}

template <typename T, int STORE>
__global__ void unpack_kernel(const PassArgs a, const C2<T>* Z, long long zdist, long long nlines) {
    const TwTables<T>* tw = (const TwTables<T>*)a.tw;
    const long long M = a.N / 2;
    const long long per = M >= 2 ? M / 2 : 1;
    const long long total = per * nlines;
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x)
        unpack_item<T, STORE>(a, tw, Z, zdist, w);
}

// Size-1 transforms of the real families (the reference's N = 1 special
// cases, src/07_legacy.h:164-167, 241-244, 759-761, 869, 958, 1014, 1300-1303):
// y = factor * x0, written as a complex (x0, 0) for realdft or a real value.
template <typename T>
__global__ void tiny_kernel(const T* x, T* y, long long howmany, long long inner, long long idist, long long odist,
                            int in_cplx, int out_cplx, double factor) {
    const long long total = howmany * inner;
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
        long long b = w / inner, i = w - b * inner;
        T v = x[(b * idist + i) * (in_cplx ? 2 : 1)];
        T r = (T)(factor * (double)v);
        if (out_cplx) {
            y[(b * odist + i) * 2] = r;
            y[(b * odist + i) * 2 + 1] = (T)0;
        } else {
            y[b * odist + i] = r;
        }
    }
}

}  // namespace nfft

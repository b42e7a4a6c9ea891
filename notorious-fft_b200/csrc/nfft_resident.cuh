// nfft_resident.cuh -- batched power-of-two complex DFT of two Stockham passes
// in ONE persistent launch, with the inter-pass scratch kept in L2.
//
// Separate launches of pass 1 and pass 2 move every point through HBM four
// times (input, scratch write, scratch read, output).  Here both passes run in
// one kernel: the work order interleaves the pass-1 tiles of transform t with
// the pass-2 tiles of transform t - lag, so a transform's scratch is read back
// a few tens of MB of traffic after it was written -- while it is still in L2
// (written with evict_last priority, read at L2 and then discarded, so it is
// never written back).  DRAM then carries only the input and the output.
//
// Work item g (one tile of one pass of one transform, decoded by
// resident_decode) is claimed in order with an atomic counter, the claim of the
// next item in flight while the current one runs.  A pass-2 tile of transform t
// waits (bounded) until all pass-1 tiles of t have been published on t's
// counter; pass-1 tiles of t always precede pass-2 tiles of t in the order, so
// a claimed item always makes progress.  The tile bodies are the specialized
// pass bodies of nfft_lean.cuh (pass 1: column in / row out, pass 2: column in
// / column out), inlined with compile-time radices.
#pragma once

#include "nfft_lean.cuh"

namespace nfft {

struct ResidentArgs {
    long long B;          // transforms in this launch
    long long lag;        // transforms between the pass-1 and pass-2 tiles of a transform
    int log_tiles;        // log2 tiles per transform per pass
    unsigned* ctr;        // [0] next item, [1] abort flag, [2 + t] pass-1 tiles of t done
    int* status;          // item + 1 of the first wait that gave up; 0 when none did
    long long spin_limit;
};

// Item g -> (pass 1 or 2, transform, tile).  Order: pass 1 of transforms
// 0 .. lag-1; then for s = lag .. B-1 pass 1 of s followed by pass 2 of s - lag;
// then pass 2 of B - lag .. B - 1.
NFFT_HD void resident_decode(long long g, long long B, long long lag, int lt, int& pass, long long& tr,
                             long long& tile) {
    const long long T = 1ll << lt;
    const long long a = lag << lt;
    if (g < a) {
        pass = 1;
        tr = g >> lt;
        tile = g & (T - 1);
        return;
    }
    g -= a;
    const long long b = (B - lag) << (lt + 1);
    if (g < b) {
        const long long s = g >> (lt + 1), w = g & (2 * T - 1);
        if (w < T) {
            pass = 1;
            tr = lag + s;
            tile = w;
        } else {
            pass = 2;
            tr = s;
            tile = w - T;
        }
        return;
    }
    g -= b;
    pass = 2;
    tr = (B - lag) + (g >> lt);
    tile = g & (T - 1);
}

// Line of thread t in global tile g of a resident pass with radix 2^logR and
// 2^logJ lines per tile (column mapping; the lines of a transform are its
// 2^logNj Stockham lines, the batch dim outermost): the line's offsets and
// Stockham index, and the thread's butterfly index i.  Equivalent to
// line_setup for these passes, with shifts instead of divisions.
NFFT_HD void resident_line(const PassArgs& a, int logJ, int logR, long long g, int t, long long& bin, long long& bout,
                           long long& j, int& i) {
    const int l = t & ((1 << logJ) - 1);
    i = t >> logJ;
    (void)logR;
    const long long lam = (g << logJ) + l;
    const long long b = lam >> a.logNj;
    j = lam & ((1ll << a.logNj) - 1);
    bin = a.ndims > 1 ? b * a.istr[1] : 0;
    bout = a.ndims > 1 ? b * a.ostr[1] : 0;
}

#if defined(__CUDACC__)
__device__ __forceinline__ unsigned res_ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned res_ld_relaxed(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded wait of thread 0; 1: satisfied, 0: the launch is abandoned.
static __device__ __noinline__ int resident_wait(const ResidentArgs& r, long long tr, unsigned target, long long item) {
    unsigned ns = 32;
    for (long long n = 0;; ++n) {
        if (res_ld_acquire(&r.ctr[2 + tr]) >= target) return 1;
        if (res_ld_relaxed(&r.ctr[1])) return 0;
        if (n >= r.spin_limit) {
            atomicExch(&r.ctr[1], 1u);
            atomicCAS(r.status, 0, (int)(item + 1));
            return 0;
        }
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
}

template <typename T, int R1, int R2, int LOGT>
constexpr size_t resident_smem_bytes() {
    constexpr size_t s1 = lean_smem_bytes<T, R1, LOGT, true, false, LD_C, ST_C>();
    constexpr size_t s2 = lean_smem_bytes<T, R2, LOGT, true, true, LD_C, ST_C>();
    return s1 > s2 ? s1 : s2;
}

// a1: pass 1 (input -> scratch), a2: pass 2 (scratch -> output); both with the
// batch dim outermost, so tile k of transform t is line tile t * 2^lt + k.
template <typename T, int R1, int R2, int LOGT>
__global__ void __launch_bounds__(1 << LOGT, (LOGT <= 7 ? 4 : (LOGT == 8 ? 2 : 1)))
resident_kernel(const PassArgs a1, const PassArgs a2, const ResidentArgs r) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ long long s_item;
    __shared__ int s_go;
    const int t = threadIdx.x;
    const long long nitems = r.B << (r.log_tiles + 1);
    unsigned long long claim = 0;
    if (t == 0) claim = atomicAdd(&r.ctr[0], 1u);
    for (;;) {
        if (t == 0) {
            s_item = (long long)claim;
            s_go = ((long long)claim < nitems) && !res_ld_relaxed(&r.ctr[1]);
            if (s_go) claim = atomicAdd(&r.ctr[0], 1u);   // next claim in flight during this item
        }
        __syncthreads();
        if (!s_go) break;
        const long long item = s_item;
        int pass;
        long long tr, tile;
        resident_decode(item, r.B, r.lag, r.log_tiles, pass, tr, tile);
        if (pass == 2) {
            if (t == 0) s_go = resident_wait(r, tr, 1u << r.log_tiles, item);
            __syncthreads();
            if (!s_go) break;
            lean_tile<T, R2, LOGT, true, true, LD_C, ST_C>(a2, (tr << r.log_tiles) + tile, smraw);
            __syncthreads();
        } else {
            lean_tile<T, R1, LOGT, true, false, LD_C, ST_C>(a1, (tr << r.log_tiles) + tile, smraw);
            __syncthreads();
            if (t == 0) {
                __threadfence();
                atomicAdd(&r.ctr[2 + tr], 1u);
            }
        }
    }
}

// ---- software-pipelined variant ---------------------------------------------
// While a CTA computes tile k, the inputs of tile k+1 are already on their way
// into a shared-memory staging buffer (cp.async, 16 points per thread in slots
// private to the thread, so the staged data needs no barrier): the first
// sub-stage of every tile reads shared memory instead of waiting on global
// latency.  The next item is claimed one item ahead; its prefetch is issued
// right after the current tile's first barrier -- for a pass-2 tile only when
// one poll shows its transform's pass 1 complete, otherwise the tile is loaded
// (after a bounded wait) once the current tile is published.

template <typename T>
__device__ __forceinline__ void res_cp_async(C2<T>* dst, const C2<T>* src) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(C2<T>) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(src) : "memory");
}
__device__ __forceinline__ void res_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void res_cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Issue the loads of global tile g of the pass L (arguments a) into the
// staging slots of this thread; threads t < J also record the tile's lines.
template <typename L, typename T>
__device__ __forceinline__ void res_prefetch(const PassArgs& a, long long g, C2<T>* stage, LeanLine* lines) {
    const int t = threadIdx.x;
    long long bin, bout, j;
    int i;
    resident_line(a, L::LOGJ, L::LOGR_, g, t, bin, bout, j, i);
    if (t < L::J) lines[t] = LeanLine{bin, bout, j};
    const long long rs = a.in_estride << a.logNj;
    const C2<T>* src = (const C2<T>*)a.in + bin + j * a.in_estride + (long long)i * rs;
    const long long s16 = rs << (L::LOGR_ - 4);
#pragma unroll
    for (int m = 0; m < 16; ++m) res_cp_async<T>(&stage[m * L::THREADS + t], src + m * s16);
    res_cp_commit();
}

// One tile of pass L from the staging buffer.  pre(): run by every thread just
// before the first barrier; post(): just after it.
template <typename L, typename T, typename Pre, typename Post>
__device__ __forceinline__ void res_pf_tile(const PassArgs& a, const TwTables<T>* tw, C2<T>* sm, const C2<T>* stage,
                                            const LeanLine* lines, Pre pre, Post post) {
    using V = C2<T>;
    const int t = threadIdx.x;
    int l, i;
    lean_map<true, L::LOGJ>(t, L::LOGR_ - 4, l, i);
    const long long j = lines[l].j;
    V v[16];
    res_cp_wait_all();
#pragma unroll
    for (int m = 0; m < 16; ++m) v[m] = stage[m * L::THREADS + t];
    if (a.conj_in) {
#pragma unroll
        for (int m = 0; m < 16; ++m) v[m].y = -v[m].y;
    }
    L::pre_twiddle_dft(a, tw, j, i, v);
    L::template write_smem<0>(sm, l, i, v);
    pre();
    __syncthreads();
    if (a.discard_in) {
        // every load of the tile has completed: drop the scratch lines just read
        constexpr int PER_LINE = 128 / (int)sizeof(V);
        if (L::J >= PER_LINE && (l % PER_LINE) == 0) {
            const LeanLine ln = lines[l];
            const V* src = (const V*)a.in + ln.bin + ln.j * a.in_estride;
            const long long rs = a.in_estride << a.logNj;
#pragma unroll
            for (int m = 0; m < 16; ++m) discard_l2(&src[(long long)(i + (m << (L::LOGR_ - 4))) * rs]);
        }
    }
    post();
    if constexpr (L::NS >= 3) {
        constexpr int S = 1;
        constexpr int RHO = 1 << LeanSched<L::LOGR_>::lr[S];
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
    {
        constexpr int S = L::NS - 1;
        constexpr int RHO = 1 << LeanSched<L::LOGR_>::lr[S];
        V w[16];
        int ls[16 / RHO], is[16 / RHO];
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) L::template read<S, true>(sm, t, q, &w[q * RHO], ls[q], is[q]);
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) {
            L::template twiddle_dft<S>(tw, is[q], &w[q * RHO]);
            L::template write_global<S>(a, tw, lines, ls[q], is[q], &w[q * RHO]);
        }
    }
}

template <typename T, int R1, int R2, int LOGT>
constexpr size_t resident_pf_smem_bytes() {
    using L1 = Lean<T, R1, LOGT, true, false, LD_C, ST_C>;
    using L2 = Lean<T, R2, LOGT, true, true, LD_C, ST_C>;
    constexpr int ex = L1::SMEM_ELEMS > L2::SMEM_ELEMS ? L1::SMEM_ELEMS : L2::SMEM_ELEMS;
    constexpr int jm = L1::J > L2::J ? L1::J : L2::J;
    return sizeof(C2<T>) * ((size_t)ex + 16 * (size_t)(1 << LOGT)) + 2 * sizeof(LeanLine) * (size_t)jm;
}
// CTAs per SM the shared memory allows (227 KB per CTA at most, 228 KB per SM).
template <typename T, int R1, int R2, int LOGT>
constexpr int resident_pf_min_blocks() {
    constexpr size_t per = resident_pf_smem_bytes<T, R1, R2, LOGT>() + 1024;
    constexpr int by_smem = (int)((228u * 1024u) / per);
    constexpr int by_regs = LOGT <= 7 ? 4 : (LOGT == 8 ? 2 : 1);
    return by_smem < 1 ? 1 : (by_smem < by_regs ? by_smem : by_regs);
}

template <typename T, int R1, int R2, int LOGT>
__global__ void __launch_bounds__(1 << LOGT, (resident_pf_min_blocks<T, R1, R2, LOGT>()))
resident_pf_kernel(const PassArgs a1, const PassArgs a2, const ResidentArgs r) {
    using L1 = Lean<T, R1, LOGT, true, false, LD_C, ST_C>;
    using L2 = Lean<T, R2, LOGT, true, true, LD_C, ST_C>;
    using V = C2<T>;
    constexpr int TH = 1 << LOGT;
    constexpr int EX = L1::SMEM_ELEMS > L2::SMEM_ELEMS ? L1::SMEM_ELEMS : L2::SMEM_ELEMS;
    constexpr int JM = L1::J > L2::J ? L1::J : L2::J;
    extern __shared__ __align__(16) unsigned char smraw[];
    V* sm = (V*)smraw;
    V* stage = sm + EX;
    LeanLine* lbuf = (LeanLine*)(stage + 16 * TH);
    // [c]: the current item of a tile of parity c; [c ^ 1]: written by thread 0
    // during that tile (the next item), so the two never race
    __shared__ long long s_next[2];   // item, -1: none
    __shared__ int s_pf[2];           // its loads are already in flight
    __shared__ int s_go;
    const TwTables<T>* tw = (const TwTables<T>*)a1.tw;
    const int t = threadIdx.x;
    const int lt = r.log_tiles;
    const long long nitems = r.B << (lt + 1);
    unsigned long long claim = 0;   // thread 0: the item after s_next, in flight
    if (t == 0) {
        const long long c0 = atomicAdd(&r.ctr[0], 1u);
        s_next[0] = c0 < nitems ? c0 : -1;
        if (s_next[0] >= 0) claim = atomicAdd(&r.ctr[0], 1u);
        s_pf[0] = 0;
    }
    __syncthreads();
    int cur_buf = 0;
    for (;;) {
        const long long item = s_next[cur_buf];
        const int prefetched = s_pf[cur_buf];
        if (item < 0) break;
        int pass;
        long long tr, tile;
        resident_decode(item, r.B, r.lag, lt, pass, tr, tile);
        LeanLine* lines = lbuf + cur_buf * JM;
        if (!prefetched) {
            // not prefetched: wait for its dependency, then load it now
            if (t == 0) s_go = (pass == 2) ? resident_wait(r, tr, 1u << lt, item) : !res_ld_relaxed(&r.ctr[1]);
            __syncthreads();
            if (!s_go) break;
            if (pass == 1) res_prefetch<L1, T>(a1, (tr << lt) + tile, stage, lines);
            else res_prefetch<L2, T>(a2, (tr << lt) + tile, stage, lines);
            __syncthreads();   // lines of the tile
        }
        LeanLine* nlines = lbuf + (cur_buf ^ 1) * JM;
        // thread 0, before the tile's first barrier: take the next claim, and
        // check (one poll) whether its loads may start now
        const int nb = cur_buf ^ 1;
        auto pre = [&]() {
            if (t == 0) {
                const long long c = (long long)claim;
                const long long nx = (c < nitems && !res_ld_relaxed(&r.ctr[1])) ? c : -1;
                int pf = 0;
                if (nx >= 0) {
                    claim = atomicAdd(&r.ctr[0], 1u);
                    int p2;
                    long long tr2, tile2;
                    resident_decode(nx, r.B, r.lag, lt, p2, tr2, tile2);
                    pf = (p2 == 1) || res_ld_acquire(&r.ctr[2 + tr2]) >= (1u << lt);
                }
                s_next[nb] = nx;
                s_pf[nb] = pf;
            }
        };
        auto post = [&]() {
            if (s_pf[nb]) {
                int p2;
                long long tr2, tile2;
                resident_decode(s_next[nb], r.B, r.lag, lt, p2, tr2, tile2);
                if (p2 == 1) res_prefetch<L1, T>(a1, (tr2 << lt) + tile2, stage, nlines);
                else res_prefetch<L2, T>(a2, (tr2 << lt) + tile2, stage, nlines);
            }
        };
        if (pass == 1) res_pf_tile<L1, T>(a1, tw, sm, stage, lines, pre, post);
        else res_pf_tile<L2, T>(a2, tw, sm, stage, lines, pre, post);
        __syncthreads();
        if (pass == 1 && t == 0) {
            __threadfence();
            atomicAdd(&r.ctr[2 + tr], 1u);
        }
        cur_buf ^= 1;
    }
    res_cp_wait_all();
}
#endif

}  // namespace nfft

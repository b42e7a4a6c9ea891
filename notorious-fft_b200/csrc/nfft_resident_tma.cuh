// nfft_resident_tma.cuh -- the resident two-pass batched complex DFT with its
// tile loads moved off the critical path: a producer warp streams every tile
// into shared memory with the Tensor Memory Accelerator while consumer warp
// groups compute earlier tiles.
//
// Same work as resident_kernel (nfft_resident.cuh): both Stockham passes of a
// batch of transforms in one persistent launch, the pass-1 tiles of transform
// t interleaved with the pass-2 tiles of transform t - lag, the inter-pass
// scratch written with evict_last priority and read back from L2.  The plain
// resident kernel loads each tile with 16 global loads per thread and stalls
// on them (long-scoreboard and barrier stalls; it moves only the algorithmic
// DRAM bytes but no faster than two separate launches).  Here:
//  * one CTA per SM holds NG groups of 2^LOGT threads; every group owns two
//    stage buffers and claims its own work items in order (atomic counter);
//  * thread 0 of a group issues the next item's tile as ONE tensor copy
//    (cp.async.bulk.tensor, 3-D box: reals of the tile's J lines x the pass
//    radix R x one transform) into the group's other stage, completing on
//    that stage's mbarrier, BEFORE the group computes the current tile -- so
//    the copy of tile k+1 overlaps the arithmetic of tile k.  A pass-2 tile
//    whose transform's pass 1 is not complete at that moment is loaded after
//    the current tile has been published instead (bounded wait), so a group
//    never waits on an item behind its own current tile;
//  * the group reads its 16 points per thread from the dense [r][line] box,
//    runs the pass pre-twiddle and radix 16, then the sub-stage exchanges of
//    the specialized pass (nfft_lean.cuh) in place in the same stage buffer
//    (padded layout), and stores its outputs straight to global memory.
//    Pass-1 tiles publish on their transform's counter (barrier, fence,
//    atomicAdd); pass-2 tiles drop the scratch lines they loaded (discard, no
//    write-back).
// No producer warp: 12 warps per SM leave 168 registers per thread, enough
// for the pass bodies without spills (a 13th warp caps every thread at 128
// registers -- 16K registers per SM sub-partition, one of which then holds 4
// warps -- and the spilled lines miss the small L1 left beside the stages).
// Every wait is bounded: a wait that gives up raises the launch's abort flag
// and records the status word, and a group leaves only after its issued
// copies have landed (bounded), so no copy is in flight into the shared
// memory of a finished CTA.
#pragma once

#include <cuda.h>

#include "nfft_resident.cuh"

namespace nfft {

// Tile geometry of a pass for the tensor copy: the pass input seen as a 3-D
// array of reals [transform][r][2 * line] (lines contiguous, r at stride
// 2^logNj complex elements, transforms at the batch stride).  A tile is the
// box {2 J, R, 1} at (2 j0, 0, b); radices above 2^8 take R / 256 boxes of
// 256 rows (a box dimension holds at most 256 elements).
struct TmaPassGeom {
    unsigned long long dim[3];          // reals, r rows, transforms
    unsigned long long stride_bytes[2]; // of dims 1 and 2
    unsigned box[3];                    // 2 J, rows per box, 1
    int nbox;                           // boxes per tile
};

NFFT_HD TmaPassGeom tma_pass_geom(int logNj, int logR, int logJ, long long B, long long batch_stride_elems,
                                  size_t cplx_bytes) {
    TmaPassGeom g;
    g.dim[0] = 2ull << logNj;
    g.dim[1] = 1ull << logR;
    g.dim[2] = (unsigned long long)B;
    g.stride_bytes[0] = (unsigned long long)cplx_bytes << logNj;
    g.stride_bytes[1] = (unsigned long long)batch_stride_elems * cplx_bytes;
    const int rows = logR > 8 ? 256 : (1 << logR);
    g.box[0] = 2u << logJ;
    g.box[1] = (unsigned)rows;
    g.box[2] = 1;
    g.nbox = (1 << logR) / rows;
    return g;
}

// Box coordinates of global tile gt (2^logJ lines per tile, 2^logNj lines per
// transform, batch dim outermost).
NFFT_HD void tma_tile_coords(long long gt, int logJ, int logNj, int& x, int& z) {
    const long long lam0 = gt << logJ;
    z = (int)(lam0 >> logNj);
    x = (int)(2 * (lam0 & ((1ll << logNj) - 1)));
}

// Thread tt's 16 first-sub-stage points from a tile's dense [r][line] box
// (line l, butterfly i), conjugated for inverse transforms.
template <typename L, typename V>
NFFT_HD void tma_stage_read(const PassArgs& a, const V* st, int tt, V* v, int& l, int& i) {
    lean_map<true, L::LOGJ>(tt, L::LOGR_ - 4, l, i);
#pragma unroll
    for (int m = 0; m < 16; ++m) v[m] = st[NFFT_SM((((i + (m << (L::LOGR_ - 4))) << L::LOGJ) + l))];
    if (a.conj_in) {
#pragma unroll
        for (int m = 0; m < 16; ++m) v[m].y = -v[m].y;
    }
}

// 128-byte L2 line w (w < (J sizeof(V) / 128) R) of the scratch rows of
// global tile gt, when a tile row is a whole number of lines (else NULL).
template <typename L, typename V>
NFFT_HD const void* tma_discard_line(const PassArgs& a, long long gt, int w) {
    constexpr int ROW = L::J * (int)sizeof(V);
    if constexpr (ROW % 128 != 0) {
        (void)a, (void)gt, (void)w;
        return nullptr;
    }
    constexpr int PER_ROW = ROW / 128 > 0 ? ROW / 128 : 1;
    const long long lam0 = gt << L::LOGJ;
    const long long b = lam0 >> a.logNj, j0 = lam0 & ((1ll << a.logNj) - 1);
    const V* base = (const V*)a.in + (a.ndims > 1 ? b * a.istr[1] : 0) + j0;
    return (const unsigned char*)(base + ((long long)(w / PER_ROW) << a.logNj)) + 128 * (w % PER_ROW);
}

template <typename T, int R1, int R2, int LOGT>
struct TmaRes {
    using L1 = Lean<T, R1, LOGT, true, false, LD_C, ST_C>;
    using L2 = Lean<T, R2, LOGT, true, true, LD_C, ST_C>;
    static constexpr int THREADS = 1 << LOGT;
    static constexpr size_t TILE_BYTES = sizeof(C2<T>) << (LOGT + 4);
    static constexpr size_t PAD1 = sizeof(C2<T>) * (size_t)L1::SMEM_ELEMS;
    static constexpr size_t PAD2 = sizeof(C2<T>) * (size_t)L2::SMEM_ELEMS;
    static constexpr size_t RAW = TILE_BYTES > PAD1 ? (TILE_BYTES > PAD2 ? TILE_BYTES : PAD2) : (PAD1 > PAD2 ? PAD1 : PAD2);
    static constexpr size_t STAGE = (RAW + 127) / 128 * 128;
    static constexpr int JMAX = L1::J > L2::J ? L1::J : L2::J;
    // per group: two stages and their mbarriers, a state word block, a line table
    static constexpr size_t GROUP_EXTRA = 2 * 8 + 64 + JMAX * sizeof(LeanLine);
    static constexpr size_t SMEM_MAX = 232448;   // opt-in dynamic shared memory per CTA
    static constexpr size_t smem_bytes(int ng) { return (size_t)ng * (2 * STAGE + GROUP_EXTRA); }
    static constexpr int stages(int ng) { return 2 * ng; }
};

#if defined(__CUDACC__)
__device__ __forceinline__ unsigned tma_smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tma_smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tma_smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tma_smem_u32(b)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ int mbar_try(unsigned long long* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(tma_smem_u32(b)), "r"(parity)
        : "memory");
    return (int)ok;
}
// Bounded wait for the completion of the phase of parity `parity`; 1: done.
__device__ __forceinline__ int mbar_wait(unsigned long long* b, unsigned parity, long long limit) {
    for (long long n = 0; n < limit; ++n)
        if (mbar_try(b, parity)) return 1;
    return 0;
}
__device__ __forceinline__ void tma_group_bar(int id, int threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}
__device__ __forceinline__ void tma_load_box(void* dst, const CUtensorMap* map, int x, int y, int z,
                                             unsigned long long* bar, unsigned long long pol) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3, %4}], [%5], %6;" ::"r"(tma_smem_u32(dst)),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(tma_smem_u32(bar)), "l"(pol)
        : "memory");
}

// resident_wait, inlined (a call would make the kernel save live registers
// to local memory around it).
__device__ __forceinline__ int tma_dep_wait(const ResidentArgs& r, long long tr, unsigned target, long long item) {
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

// A wait of this launch gave up: raise the abort flag, record the status.
__device__ __forceinline__ void tma_res_fail(const ResidentArgs& r, long long code) {
    atomicExch(&r.ctr[1], 1u);
    atomicCAS(r.status, 0, (int)code);
}

// One tile of pass L from stage buffer `st` by group thread tt (2^LOGT
// threads, named barrier `bar`).  The stage is free for the next tensor copy
// once every thread has passed the barrier after the last shared read.
template <typename L, typename T>
__device__ __forceinline__ void tma_res_tile(const PassArgs& a, long long gt, C2<T>* st, LeanLine* lines, int tt,
                                             int bar) {
    using V = C2<T>;
    constexpr int TH = L::THREADS;
    constexpr int LOGR = L::LOGR_;
    const TwTables<T>* tw = (const TwTables<T>*)a.tw;
    if (tt < L::J) {
        long long bin, bout, j;
        int i_;
        resident_line(a, L::LOGJ, LOGR, gt, tt, bin, bout, j, i_);
        lines[tt] = LeanLine{bin, bout, j};
    }
    if (a.discard_in && (L::J * (int)sizeof(V)) % 128 == 0) {
        // the tile's scratch rows are in shared memory now: drop their L2 lines
        constexpr int LINES = (L::J * (int)sizeof(V) / 128) << LOGR;
        for (int w = tt; w < LINES; w += TH) discard_l2(tma_discard_line<L, V>(a, gt, w));
    }
    int l, i;
    V v[16];
    tma_stage_read<L, V>(a, st, tt, v, l, i);
    const long long j = ((gt << L::LOGJ) + l) & ((1ll << a.logNj) - 1);
    tma_group_bar(bar, TH);   // the dense box is read; lines[] written
    L::pre_twiddle_dft(a, tw, j, i, v);
    L::template write_smem<0>(st, l, i, v);
    tma_group_bar(bar, TH);
    if constexpr (L::NS >= 3) {
        constexpr int S = 1;
        constexpr int RHO = 1 << LeanSched<LOGR>::lr[S];
        V w[16];
        int ls[16 / RHO], is[16 / RHO];
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) L::template read<S, L::COLL>(st, tt, q, &w[q * RHO], ls[q], is[q]);
        tma_group_bar(bar, TH);
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) {
            L::template twiddle_dft<S>(tw, is[q], &w[q * RHO]);
            L::template write_smem<S>(st, ls[q], is[q], &w[q * RHO]);
        }
        tma_group_bar(bar, TH);
    }
    if constexpr (L::NS >= 4) {
        constexpr int S = 2;
        constexpr int RHO = 1 << LeanSched<LOGR>::lr[S];
        V w[16];
        int ls[16 / RHO], is[16 / RHO];
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) L::template read<S, L::COLL>(st, tt, q, &w[q * RHO], ls[q], is[q]);
        tma_group_bar(bar, TH);
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) {
            L::template twiddle_dft<S>(tw, is[q], &w[q * RHO]);
            L::template write_smem<S>(st, ls[q], is[q], &w[q * RHO]);
        }
        tma_group_bar(bar, TH);
    }
    {
        constexpr int S = L::NS - 1;
        constexpr int RHO = 1 << LeanSched<LOGR>::lr[S];
        V w[16];
        int ls[16 / RHO], is[16 / RHO];
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) L::template read<S, L::COL_OUT_>(st, tt, q, &w[q * RHO], ls[q], is[q]);
        // every generic access of the stage precedes the next tensor copy into it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tma_group_bar(bar, TH);
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) {
            L::template twiddle_dft<S>(tw, is[q], &w[q * RHO]);
            L::template write_global<S>(a, tw, lines, ls[q], is[q], &w[q * RHO]);
        }
    }
}

// State of a group in shared memory (its thread 0 keeps it there rather than
// in registers, which would stay live -- and spill -- across the tile body).
struct TmaGroupState {
    long long cur;       // item of this iteration (-1: done)
    long long nxt;       // item to run in the next iteration (-1: none)
    long long ahead;     // item claimed one iteration early (-1: none)
    int ok;              // this iteration's copy landed
    int pend;            // nxt is a pass-2 tile not yet ready: load it after this tile
    int issued[2];       // copies issued into each stage
    int waited[2];       // copies waited for
};

// Thread 0 of a group: the copy of item g (decoded) into stage buffer dst.
template <int R1, int R2, int LOGT, size_t TILE_BYTES, typename V>
__device__ __forceinline__ void tma_res_issue(const CUtensorMap* m1, const CUtensorMap* m2, const PassArgs& a1,
                                              const PassArgs& a2, const ResidentArgs& r, int pass, long long tr,
                                              long long tile, V* dst, unsigned long long* full,
                                              unsigned long long pol) {
    const long long gt = (tr << r.log_tiles) + tile;
    const int logR = pass == 1 ? R1 : R2;
    const int logJ = LOGT + 4 - logR;
    int x, z;
    tma_tile_coords(gt, logJ, pass == 1 ? a1.logNj : a2.logNj, x, z);
    if (pass == 2) asm volatile("fence.proxy.async.global;" ::: "memory");   // other CTAs' pass-1 stores
    mbar_arrive_tx(full, (unsigned)TILE_BYTES);
    const int rows = logR > 8 ? 256 : (1 << logR);
    for (int k = 0; k < (1 << logR) / rows; ++k)
        tma_load_box(dst + ((size_t)(k * rows) << logJ), pass == 1 ? m1 : m2, x, k * rows, z, full, pol);
}

// m1 / m2: tensor maps of the pass-1 input and of the scratch (tma_pass_geom);
// a1 / a2 and r as for resident_kernel.
template <typename T, int R1, int R2, int LOGT, int NG>
__global__ void __launch_bounds__(NG << LOGT, 1)
tma_resident_kernel(const __grid_constant__ CUtensorMap m1, const __grid_constant__ CUtensorMap m2, const PassArgs a1,
                    const PassArgs a2, const ResidentArgs r) {
    using G = TmaRes<T, R1, R2, LOGT>;
    using V = C2<T>;
    constexpr int TH = G::THREADS;
    static_assert(G::smem_bytes(NG) <= G::SMEM_MAX, "two stages per group must fit in shared memory");
    extern __shared__ __align__(128) unsigned char tma_smraw[];
    const int t = threadIdx.x, c = t >> LOGT, tt = t & (TH - 1), bar = 1 + c;
    unsigned char* const stage0 = tma_smraw + (size_t)(2 * c) * G::STAGE;   // stage b at stage0 + b STAGE
    unsigned long long* full = (unsigned long long*)(tma_smraw + (size_t)(2 * NG) * G::STAGE) + 2 * c;
    TmaGroupState* gs = (TmaGroupState*)(tma_smraw + (size_t)(2 * NG) * G::STAGE + 16 * NG) + c;
    LeanLine* lines = (LeanLine*)(tma_smraw + (size_t)(2 * NG) * G::STAGE + 16 * NG + 64 * NG) + c * G::JMAX;
    const long long nitems = r.B << (r.log_tiles + 1);
    const unsigned tiles1 = 1u << r.log_tiles;
    auto claim = [&]() -> long long {
        if (res_ld_relaxed(&r.ctr[1])) return -1;
        const long long g = (long long)atomicAdd(&r.ctr[0], 1u);
        return g < nitems ? g : -1;
    };
    auto policy = []() {
        unsigned long long pol;
        asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
        return pol;
    };
    if (tt == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        gs->issued[0] = gs->issued[1] = gs->waited[0] = gs->waited[1] = 0;
        long long cur = claim();
        if (cur >= 0) {
            int pass;
            long long tr, tile;
            resident_decode(cur, r.B, r.lag, r.log_tiles, pass, tr, tile);
            if (pass == 2 && !tma_dep_wait(r, tr, tiles1, cur)) {
                cur = -1;
            } else {
                tma_res_issue<R1, R2, LOGT, G::TILE_BYTES>(&m1, &m2, a1, a2, r, pass, tr, tile, (V*)stage0, &full[0],
                                                           policy());
                gs->issued[0] = 1;
            }
        }
        gs->cur = cur;
        gs->ahead = cur >= 0 ? claim() : -1;
    }
    for (int k = 0;; ++k) {
        const int b = k & 1;
        if (tt == 0) {
            // the next item's copy goes out before this tile's arithmetic
            const long long cur = gs->cur;
            const long long nxt = cur >= 0 ? gs->ahead : -1;
            int pend = 0;
            if (nxt >= 0) {
                int pn;
                long long ntr, ntile;
                resident_decode(nxt, r.B, r.lag, r.log_tiles, pn, ntr, ntile);
                if (pn == 1 || res_ld_acquire(&r.ctr[2 + ntr]) >= tiles1) {
                    tma_res_issue<R1, R2, LOGT, G::TILE_BYTES>(&m1, &m2, a1, a2, r, pn, ntr, ntile,
                                                               (V*)(stage0 + (size_t)(b ^ 1) * G::STAGE), &full[b ^ 1],
                                                               policy());
                    gs->issued[b ^ 1]++;
                } else {
                    pend = 1;
                }
            }
            int ok = 1;
            if (cur >= 0) {
                ok = mbar_wait(&full[b], (unsigned)(k >> 1) & 1u, r.spin_limit);
                if (ok) gs->waited[b]++;
                else tma_res_fail(r, -2);
            }
            gs->nxt = nxt;
            gs->pend = pend;
            gs->ok = ok;
        }
        // claim of the item after next: the atomic's round trip overlaps this tile
        long long ahead = -1;
        if (tt == 0 && gs->nxt >= 0) ahead = claim();
        tma_group_bar(bar, TH);
        const long long g = gs->cur;
        if (g < 0 || !gs->ok) break;
        if (tt != 0) mbar_wait(&full[b], (unsigned)(k >> 1) & 1u, r.spin_limit);   // acquire; the phase is complete
        int pass;
        long long tr, tile;
        resident_decode(g, r.B, r.lag, r.log_tiles, pass, tr, tile);
        const long long gt = (tr << r.log_tiles) + tile;
        if (pass == 1) {
            tma_res_tile<typename G::L1, T>(a1, gt, (V*)(stage0 + (size_t)b * G::STAGE), lines, tt, bar);
            tma_group_bar(bar, TH);
            if (tt == 0) {
                __threadfence();
                atomicAdd(&r.ctr[2 + tr], 1u);
            }
        } else {
            tma_res_tile<typename G::L2, T>(a2, gt, (V*)(stage0 + (size_t)b * G::STAGE), lines, tt, bar);
        }
        if (tt == 0) {
            long long nxt = gs->nxt;
            if (gs->pend) {
                // published above: now the pass-2 tile whose transform was not ready
                int pn;
                long long ntr, ntile;
                resident_decode(nxt, r.B, r.lag, r.log_tiles, pn, ntr, ntile);
                if (tma_dep_wait(r, ntr, tiles1, nxt)) {
                    tma_res_issue<R1, R2, LOGT, G::TILE_BYTES>(&m1, &m2, a1, a2, r, pn, ntr, ntile,
                                                               (V*)(stage0 + (size_t)(b ^ 1) * G::STAGE),
                                                               &full[b ^ 1], policy());
                    gs->issued[b ^ 1]++;
                } else {
                    nxt = -1;
                }
            }
            gs->cur = nxt;
            gs->ahead = ahead;
        }
    }
    // no copy may still be landing in this CTA's shared memory when it exits
    if (tt == 0)
        for (int b = 0; b < 2; ++b)
            if (gs->issued[b] > gs->waited[b] &&
                !mbar_wait(&full[b], (unsigned)((gs->issued[b] - 1) & 1), r.spin_limit))
                tma_res_fail(r, -3);
}
#endif

}  // namespace nfft

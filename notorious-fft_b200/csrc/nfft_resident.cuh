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
#endif

}  // namespace nfft

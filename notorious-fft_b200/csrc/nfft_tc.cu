// nfft_tc.cu -- the split-tensor-core pass kernels of the float library
// (NOTORIOUS_FFT_FORM_SPLIT_TC):
//  * tc_lean_kernel: radix-256 passes, both radix-16 stages of a line as FP16
//    hi + lo tensor-core products in registers (nfft_tc_lean.cuh), persistent
//    CTAs over 16-line tiles -- every radix-256 pass of the form;
//  * tc_pass_kernel: the generic Stockham pass (nfft_pass.cuh) with its
//    radix-16 sub-stages computed by tc_substage (nfft_tc.cuh) -- the other
//    pass radices.
#include <stdlib.h>

#include <algorithm>

#include "nfft_engine.h"
#include "nfft_tc.cuh"
#include "nfft_tc_lean.cuh"

namespace nfft {

#if NFFT_REAL_IS_FLOAT

template <int LOG_TILE>
__global__ void __launch_bounds__((1 << LOG_TILE) / 16) tc_pass_kernel(const PassArgs a) {
    constexpr int TILE = 1 << LOG_TILE;
    constexpr int THREADS = TILE / 16;
    extern __shared__ __align__(16) unsigned char smraw[];
    float2* sm = (float2*)smraw;
    TileLines tl;
    tl.in = (long long*)(sm + pass_smem_elems<float>(LOG_TILE));
    tl.out = tl.in + MAX_J;
    tl.j = tl.out + MAX_J;
    const TwTables<float>* tw = (const TwTables<float>*)a.tw;
    const int tid = threadIdx.x;
    const int logE = a.logR + a.logJ;
    const int J = 1 << a.logJ, E = 1 << logE;
    const long long tile = (long long)blockIdx.x + (long long)blockIdx.y * gridDim.x;
    const long long line0 = tile << a.logJ;
    if (line0 >= a.nlines) return;
    TcA A;
    tc_make_A(tid & 31, A);
    for (int l = tid; l < J; l += THREADS) line_setup(a, line0 + l, l, tl);
    __syncthreads();
    {
        float2 buf[16];
#pragma unroll
        for (int it = 0; it < 16; ++it) {
            int e = tid + it * THREADS;
            if (e < E) buf[it] = load_slot_value<float, LD_C>(a, tw, tl, e);
        }
#pragma unroll
        for (int it = 0; it < 16; ++it) {
            int e = tid + it * THREADS;
            if (e < E) load_slot_commit<float>(a, tw, sm, tl, e, buf[it]);
        }
    }
    __syncthreads();
    int lns = 0;
    float2 v[16];
    for (int s = 0; s < a.nsub; ++s) {
        const int lr = a.sublog[s];
        if (lr == 4) {
            tc_substage<THREADS>(sm, tw, A, a.logR, logE, lns, tid);
        } else {
            switch (lr) {
            case 3: substage_read<float, THREADS, 8, 3>(sm, v, a.logR, logE, tid); break;
            case 2: substage_read<float, THREADS, 4, 2>(sm, v, a.logR, logE, tid); break;
            default: substage_read<float, THREADS, 2, 1>(sm, v, a.logR, logE, tid); break;
            }
            __syncthreads();
            switch (lr) {
            case 3: substage_write<float, THREADS, 8, 3>(sm, v, tw, a.logR, logE, lns, tid); break;
            case 2: substage_write<float, THREADS, 4, 2>(sm, v, tw, a.logR, logE, lns, tid); break;
            default: substage_write<float, THREADS, 2, 1>(sm, v, tw, a.logR, logE, lns, tid); break;
            }
            __syncthreads();
        }
        lns += lr;
    }
#pragma unroll
    for (int it = 0; it < 16; ++it) {
        int e = tid + it * THREADS;
        if (e < E) store_slot<float, ST_C>(a, tw, sm, tl, e);
    }
}

constexpr int TCL_THREADS = 256;

// Persistent CTAs: the per-lane constants (F fragments, internal twiddles) are
// set up once per CTA and reused for every tile it takes; the copies of the
// next tile overlap the transform and the write-out of the current one.
template <int MINB>
__global__ void __launch_bounds__(TCL_THREADS, MINB) tc_lean_kernel(const PassArgs a) {
    using P = TcPipe<TCL_THREADS>;
    using TL = TcLean<TCL_THREADS>;
    extern __shared__ __align__(16) unsigned char smraw[];
    float2* const buf0 = (float2*)smraw;                              // buffers: buf0 + b TCL_SLOTS
    long long* const lb0 = (long long*)(buf0 + 2 * TCL_SLOTS);        // line offsets: lb0 + b 3 TCL_J
    typename TL::Consts* const tab = (typename TL::Consts*)(lb0 + 6 * TCL_J);
    auto buf = [&](int b) { return buf0 + b * TCL_SLOTS; };
    auto lb = [&](int b) { return lb0 + b * 3 * TCL_J; };
    if (threadIdx.x < 32) TL::setup((const TwTables<float>*)a.tw, threadIdx.x, tab[threadIdx.x]);
    const typename TL::Consts& c = tab[threadIdx.x & 31];
    uint64_t pol_in, pol_out;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol_in));
    if (a.hint_out >= 2) asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol_out));
    else asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol_out));
    const long long ntiles = (a.nlines + TCL_J - 1) >> TCL_LOGJ;
    long long tile = blockIdx.x;
    if (tile >= ntiles) return;
    P::lines(a, tile, lb(0));
    __syncthreads();
    P::prefetch(a, lb(0), buf(0), pol_in);
    asm volatile("cp.async.commit_group;" ::: "memory");
    for (int k = 0; tile < ntiles; tile += gridDim.x, ++k) {
        const int cur = k & 1, nxt = cur ^ 1;
        const long long next = tile + gridDim.x;
        // the buffer and line offsets of `nxt` were last read before the
        // barrier that ended the previous write-out
        if (next < ntiles) P::lines(a, next, lb(nxt));
        __syncthreads();
        if (next < ntiles) P::prefetch(a, lb(nxt), buf(nxt), pol_in);
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        __syncthreads();
        P::compute(a, c, lb(cur), buf(cur));
        __syncthreads();
        P::writeout(a, lb(cur), buf(cur), pol_out);
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

bool tc_lean_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("NOTORIOUS_FFT_TC_LEAN");
        v = e ? atoi(e) : 1;
    }
    return v != 0;
}

// CTAs per SM the kernel is compiled for: 2 (default, 128 registers) or 3
// (NOTORIOUS_FFT_TC_CTAS=3: 80 registers with a few spills; measured slower
// on B200, 1339 vs 1552 GB/s on 2^16 x 2048).
static int tc_lean_ctas() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("NOTORIOUS_FFT_TC_CTAS");
        v = (e && atoi(e) == 3) ? 3 : 2;
    }
    return v;
}

bool launch_tc_lean(const PassArgs& a, int sm_count, cudaStream_t s) {
    static int per_sm = 0;
    const int minb = tc_lean_ctas();
    const void* fn = minb == 2 ? (const void*)tc_lean_kernel<2> : (const void*)tc_lean_kernel<3>;
    const size_t smem = tcl_smem_bytes<TCL_THREADS>();
    if (!per_sm) {
        if (!cuda_ok(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                     "cudaFuncSetAttribute(tc lean)"))
            return false;
        int n = 0;
        if (!cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, TCL_THREADS, smem),
                     "cudaOccupancyMaxActiveBlocksPerMultiprocessor(tc lean)"))
            return false;
        per_sm = n > 0 ? n : 1;
    }
    const long long ntiles = (a.nlines + TCL_J - 1) >> TCL_LOGJ;
    if (ntiles <= 0) return true;
    const long long grid = std::min<long long>(ntiles, (long long)std::max(sm_count, 1) * per_sm);
    if (minb == 2) tc_lean_kernel<2><<<(unsigned)grid, TCL_THREADS, smem, s>>>(a);
    else tc_lean_kernel<3><<<(unsigned)grid, TCL_THREADS, smem, s>>>(a);
    note_launch();
    return cuda_ok(cudaGetLastError(), "tensor-core radix-256 pass launch");
}

bool launch_tc_pass(const PassArgs& a, int log_tile, long long ntiles, cudaStream_t s) {
    static bool attr = false;
    const size_t smem = pass_smem_bytes<float>(log_tile);
    if (log_tile != 12) {
        set_error(6, "tensor-core pass tile 2^%d not built", log_tile);
        return false;
    }
    if (!attr) {
        if (!cuda_ok(cudaFuncSetAttribute((const void*)tc_pass_kernel<12>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem),
                     "cudaFuncSetAttribute(tc pass)"))
            return false;
        attr = true;
    }
    if (ntiles <= 0) return true;
    tc_pass_kernel<12><<<(unsigned)ntiles, (1 << 12) / 16, smem, s>>>(a);
    note_launch();
    return cuda_ok(cudaGetLastError(), "tensor-core pass launch");
}

#else

bool tc_lean_enabled() { return false; }

bool launch_tc_lean(const PassArgs&, int, cudaStream_t) {
    set_error(6, "the split tensor-core form exists in the float library only");
    return false;
}

bool launch_tc_pass(const PassArgs&, int, long long, cudaStream_t) {
    set_error(6, "the split tensor-core form exists in the float library only");
    return false;
}

#endif

}  // namespace nfft

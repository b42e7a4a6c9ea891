// nfft_tc.cu -- the split-tensor-core pass kernels of the float library
// (NOTORIOUS_FFT_FORM_SPLIT_TC):
//  * tc_umma_kernel: radix-256 passes on the sm_100 tensor cores (tcgen05
//    products from shared memory into tensor memory, tensor copies in and
//    out; nfft_umma.cuh) -- every radix-256 pass over unit-stride lines with
//    16-byte aligned buffers and strides;
//  * tc_lean_kernel: the other radix-256 passes, both radix-16 stages of a
//    line as FP16 hi + lo warp-level products in registers
//    (nfft_tc_lean.cuh), persistent CTAs over 16-line tiles;
//  * tc_pass_kernel: the generic Stockham pass (nfft_pass.cuh) with its
//    radix-16 sub-stages computed by tc_substage (nfft_tc.cuh) -- the other
//    pass radices.
#include <stdlib.h>

#include <algorithm>

#include <cuda.h>

#include "nfft_engine.h"
#include "nfft_tc.cuh"
#include "nfft_tc_lean.cuh"
#include "nfft_umma.cuh"

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

// ---------------------------------------------------------------------------
// Radix-256 passes on tcgen05 (layout: nfft_umma.cuh).  Persistent CTAs of
// TCU_TEAMS teams of 128 threads; a team transforms one tile (8 lines) at a
// time, the next tile's input copy running while the current one is
// transformed; thread t of a team owns stage-1 row t and stage-2 row t, one
// thread of the team issues its products.  Every wait
// polls at most TcuArgs::spin times and at most 2 s; a wait that gives up
// records its kind (1: input copy, 2 / 3: stage-1 / stage-2 products) in
// g_tcu_status, lets the copies and products in flight finish (bounded),
// frees the tensor memory and leaves.
// ---------------------------------------------------------------------------
__device__ unsigned g_tcu_status;
static bool s_tcu_used = false;   // a tcgen05 pass was launched in this process

__device__ __forceinline__ uint32_t tcu_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// shared-memory matrix descriptor (sm_100): start, LBO, SBO (16-byte units), version 1, no swizzle
__device__ __forceinline__ uint64_t tcu_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           ((uint64_t)1 << 46);
}
__device__ __forceinline__ bool tcu_try(uint64_t* m, unsigned parity) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(tcu_smem(m)), "r"(parity)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t tcu_now() {
    uint64_t v;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
    return v;
}
// At most `spin` polls and at most 2 s (a poll may suspend the thread for a
// system-dependent time).
__device__ __forceinline__ bool tcu_wait(uint64_t* m, unsigned parity, long long spin) {
    if (tcu_try(m, parity)) return true;
    const uint64_t t0 = tcu_now();
    for (long long n = 1; n < spin; ++n) {
        if (tcu_try(m, parity)) return true;
        if ((n & 255) == 0 && tcu_now() - t0 > 2000000000ull) return false;
    }
    return false;
}
__device__ __forceinline__ void tcu_load(const CUtensorMap* map, void* dst, uint64_t* bar, int c0, int c2) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tcu_smem(bar)), "r"(TCU_STAGE)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(tcu_smem(dst)),
        "l"((uint64_t)map), "r"(c0), "r"(0), "r"(c2), "r"(tcu_smem(bar))
        : "memory");
}
// D = Ah Bh + Al Bh + Ah Bl; K = 32 as two steps of 16 (two K chunks / K-row groups each)
__device__ __forceinline__ void tcu_mma6(uint32_t d, uint32_t ah, uint32_t al, uint32_t bh, uint32_t bl, bool a_mmajor) {
    // instruction descriptor: FP32 accumulators, FP16 A and B, B K-major, A K- or M-major, N = 32, M = 128
    const uint32_t idesc = (1u << 4) | (a_mmajor ? (1u << 15) : 0u) | ((uint32_t)(32 >> 3) << 17) |
                           ((uint32_t)(128 >> 4) << 24);
    const uint32_t as[3] = {ah, al, ah}, bs[3] = {bh, bh, bl};
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            const uint64_t ad = tcu_desc(as[q] + ks * 2 * TCU_LBO, TCU_LBO, TCU_SBO);
            const uint64_t bd = tcu_desc(bs[q] + ks * 2 * TCU_BLBO, TCU_BLBO, TCU_BSBO);
            const uint32_t acc = (q | ks) ? 1u : 0u;
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d),
                "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                : "memory");
        }
}
__device__ __forceinline__ void tcu_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(tcu_smem(bar))
                 : "memory");
}
// the 32 accumulator columns of this thread's row (warp w reads lanes 32 w ..)
__device__ __forceinline__ void tcu_ld32(uint32_t taddr, float* v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]), "=f"(v[8]),
          "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15]), "=f"(v[16]),
          "=f"(v[17]), "=f"(v[18]), "=f"(v[19]), "=f"(v[20]), "=f"(v[21]), "=f"(v[22]), "=f"(v[23]), "=f"(v[24]),
          "=f"(v[25]), "=f"(v[26]), "=f"(v[27]), "=f"(v[28]), "=f"(v[29]), "=f"(v[30]), "=f"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
// named barrier of team 0 (id 1) or team 1 (id 2) over its 128 threads, plain
// and with an AND vote (immediate ids: the kernel reserves three barriers)
__device__ __forceinline__ void tcu_team_sync(int team) {
    if (team) asm volatile("bar.sync 2, 128;" ::: "memory");
    else asm volatile("bar.sync 1, 128;" ::: "memory");
}
__device__ __forceinline__ bool tcu_team_and(int team, bool p) {
    unsigned r;
    if (team)
        asm volatile("{\n .reg .pred q, o;\n setp.ne.u32 q, %1, 0;\n bar.red.and.pred o, 2, 128, q;\n"
                     " selp.u32 %0, 1, 0, o;\n}"
                     : "=r"(r)
                     : "r"((unsigned)p)
                     : "memory");
    else
        asm volatile("{\n .reg .pred q, o;\n setp.ne.u32 q, %1, 0;\n bar.red.and.pred o, 1, 128, q;\n"
                     " selp.u32 %0, 1, 0, o;\n}"
                     : "=r"(r)
                     : "r"((unsigned)p)
                     : "memory");
    return r != 0;
}
__device__ __forceinline__ uint32_t tcu_h2(float re, float im) {
    const __half2 h = __floats2half2_rn(re, im);
    return *(const uint32_t*)&h;
}
// hi / lo FP16 parts of 4 complex points, one 16-byte store each
__device__ __forceinline__ void tcu_split4(unsigned char* hi, unsigned char* lo, int off, const float2* x) {
    uint32_t hh[4], ll[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float re = x[q].x, im = x[q].y;
        const __half2 h = __floats2half2_rn(re, im);
        const float2 hf = __half22float2(h);
        hh[q] = *(const uint32_t*)&h;
        ll[q] = tcu_h2(re - hf.x, im - hf.y);
    }
    *(uint4*)(hi + off) = make_uint4(hh[0], hh[1], hh[2], hh[3]);
    *(uint4*)(lo + off) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
}

__global__ void __launch_bounds__(TCU_THREADS, TCU_MINB)
    tc_umma_kernel(const TcuArgs u, const __grid_constant__ CUtensorMap imap, const __grid_constant__ CUtensorMap omap) {
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char* sm = smraw + ((512 - (tcu_smem(smraw) & 511)) & 511);
    const int t = threadIdx.x, team = t >> 7, tt = t & 127, w = tt >> 5;
    unsigned char* stg = sm + team * TCU_TEAM_BYTES;       // the team's input stage
    uint64_t* bar = (uint64_t*)(sm + TCU_OFF_BAR) + 2 * team;   // [0] input tile, [1] products
    uint32_t* tslot = (uint32_t*)(sm + TCU_OFF_BAR + 16 * TCU_TEAMS);
    const PassArgs& a = u.a;
    const TwTables<float>* tw = (const TwTables<float>*)a.tw;
    int l, i, l2, k2r;
    tcu_role_a(tt, l, i);
    tcu_role_b(u.out_kind, tt, l2, k2r);
    const bool rowk = u.out_kind == TCU_OUT_ROW;
    const long long G = (long long)gridDim.x * TCU_TEAMS;
    const long long first = (long long)blockIdx.x * TCU_TEAMS + team;
    unsigned char* Ah = stg + TCU_OFF_AH;
    unsigned char* Al = stg + TCU_OFF_AL;
    // constants: the DFT matrix operands and the internal twiddles (with 2^-5)
    for (int q = t; q < 32 * 32; q += TCU_THREADS) {
        const int n = q >> 5, c = q & 31;
        const float v = tcu_b_entry(tw, n, c);
        const __half h = __float2half_rn(v);
        const __half lo = __float2half_rn(v - __half2float(h));
        const int off = tcu_b_off(n, c >> 1) + (c & 1) * 2;
        *(__half*)(sm + TCU_OFF_BH + off) = h;
        *(__half*)(sm + TCU_OFF_BL + off) = lo;
    }
    for (int q = t; q < 256; q += TCU_THREADS) {
        const int ii = q >> 4, k1 = q & 15;
        const C2<float> c = tw->t[0][(ii * k1 * 16) & (TW_SIZE - 1)];
        ((float2*)(sm + TCU_OFF_TW))[k1 * 16 + ii] = make_float2(c.x, c.y);
    }
    if (tt == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tcu_smem(&bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tcu_smem(&bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (t < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tcu_smem(tslot)),
                     "r"(TCU_TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = *tslot;
    const uint32_t d1 = tbase + 64 * team, d2 = d1 + 32, lane_addr = (uint32_t)(32 * w) << 16;
    const uint32_t ah = tcu_smem(Ah), al = tcu_smem(Al), bh = tcu_smem(sm + TCU_OFF_BH), bl = tcu_smem(sm + TCU_OFF_BL);
    const float2* twt = (const float2*)(sm + TCU_OFF_TW);
    const int logNs = a.logNs;
    const float fscale = (float)a.scale;
    bool pending = false;      // the team's issuer: an input copy in flight
    bool mma_out = false;      // products whose completion was not observed (abandoned launch)
    unsigned in_par = 0, mma_par = 0;
    if (tt == 0 && first < u.ntiles && !u.withhold) {
        long long b;
        int j0;
        tcu_tile(u, first, b, j0);
        tcu_load(&imap, stg, &bar[0], j0, (int)b);
        pending = true;
    }
    for (long long tile = first; tile < u.ntiles; tile += G) {
        const bool got = tcu_wait(&bar[0], in_par, u.spin);
        // the previous tile's output store has read its staging area
        if (tt == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        if (!tcu_team_and(team, got)) {
            if (tt == 0) atomicCAS(&g_tcu_status, 0u, 1u);
            break;
        }
        in_par ^= 1;
        if (tt == 0) pending = false;
        long long b;
        int j0;
        tcu_tile(u, tile, b, j0);
        const int j = j0 + l;
        // ---- stage 1: row t = points i + 16 m of line l ----
        float2 x[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = *(const float2*)(stg + tcu_st_off(i + 16 * m, l));
        if (a.conj_in) {
#pragma unroll
            for (int m = 0; m < 16; ++m) x[m].y = -x[m].y;
        }
        if (logNs > 0) {
            const long long k = j & ((1ll << logNs) - 1);
            if (k) {
                // W_{256 Ns}^{(i + 16 m) k} = W_{256 Ns}^{i k} (W_{16 Ns}^k)^m, powers by a depth-4 tree
                const C2<float> wb0 = twiddle<float>(tw, (uint64_t)i * (uint64_t)k, logNs + 8);
                const C2<float> st0 = twiddle<float>(tw, (uint64_t)k, logNs + 4);
                const float2 wb = make_float2(wb0.x, wb0.y), s1 = make_float2(st0.x, st0.y);
                float2 pw[16];
                pw[0] = wb;
                pw[1] = tcu_cmul(wb, s1);
                const float2 s2 = tcu_cmul(s1, s1), s4 = tcu_cmul(s2, s2), s8 = tcu_cmul(s4, s4);
                pw[2] = tcu_cmul(wb, s2);
                pw[3] = tcu_cmul(pw[1], s2);
#pragma unroll
                for (int m = 4; m < 8; ++m) pw[m] = tcu_cmul(pw[m - 4], s4);
#pragma unroll
                for (int m = 8; m < 16; ++m) pw[m] = tcu_cmul(pw[m - 8], s8);
#pragma unroll
                for (int m = 0; m < 16; ++m) x[m] = tcu_cmul(x[m], pw[m]);
            }
        }
        // one power-of-two scale per line (its 16 rows are 16 lanes of one warp),
        // none when the line's largest component is already in the unscaled range
        float mx = 0.f;
#pragma unroll
        for (int m = 0; m < 16; ++m) mx = fmaxf(mx, fmaxf(fabsf(x[m].x), fabsf(x[m].y)));
        // (a line's 16 rows are lanes 8 (l & 1) + {0..7, 16..23} of the warp)
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 4));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 16));
        const int e1 = (mx >= TCU_LO && mx < TCU_HI) ? 0 : tcu_exp(mx);
        // the exponent of this thread's stage-2 line (held by lane 8 (l2 & 1) in stage 1)
        const int e2 = rowk ? __shfl_sync(0xffffffffu, e1, (l2 & 1) << 3) : e1;
        if (e1 == 0) {
#pragma unroll
            for (int c = 0; c < 4; ++c) tcu_split4(Ah, Al, tcu_a_off(tt, 4 * c), &x[4 * c]);
        } else {
            const float s_in = tcu_pow2(-e1);
#pragma unroll
            for (int m = 0; m < 16; ++m) x[m] = make_float2(x[m].x * s_in, x[m].y * s_in);
#pragma unroll
            for (int c = 0; c < 4; ++c) tcu_split4(Ah, Al, tcu_a_off(tt, 4 * c), &x[4 * c]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        tcu_team_sync(team);   // tile read, stage-1 operand written
        if (tt == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const long long next = tile + G;
            if (next < u.ntiles) {
                long long nb;
                int nj0;
                tcu_tile(u, next, nb, nj0);
                tcu_load(&imap, stg, &bar[0], nj0, (int)nb);
                pending = true;
            }
            tcu_mma6(d1, ah, al, bh, bl, false);
            tcu_commit(&bar[1]);
        }
        // Each thread's own wait orders its tensor-memory reads and operand
        // writes after the products; whether every wait succeeded is decided
        // at the next barrier.  A warp with a wait that gave up touches
        // nothing (warp-uniform: the tensor-memory loads are .sync.aligned).
        const bool ok1 = __all_sync(0xffffffffu, tcu_wait(&bar[1], mma_par, u.spin));
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // ---- stage-1 outputs y[k1] of row t: twiddle; column (2i, 2i+1) of the
        //      M-major stage-2 rows of (l, k1), 8 k1 per 16-byte unit ----
        float v[32];
        if (ok1) {
            tcu_ld32(d1 + lane_addr, v);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const float2 c = twt[q * 16 + i];
                const float re = v[2 * q] * c.x - v[2 * q + 1] * c.y;
                const float im = v[2 * q] * c.y + v[2 * q + 1] * c.x;
                v[2 * q] = re;
                v[2 * q + 1] = im;
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int off = tcu_at_off(tcu_row_b(u.out_kind, l, 8 * h), 2 * i);
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    uint32_t hh[4], ll[4];
#pragma unroll
                    for (int p = 0; p < 4; ++p) {
                        const float x0 = v[2 * (8 * h + 2 * p) + c], x1 = v[2 * (8 * h + 2 * p + 1) + c];
                        const __half2 hv = __floats2half2_rn(x0, x1);
                        const float2 hf = __half22float2(hv);
                        hh[p] = *(const uint32_t*)&hv;
                        ll[p] = tcu_h2(x0 - hf.x, x1 - hf.y);
                    }
                    *(uint4*)(Ah + off + 16 * c) = make_uint4(hh[0], hh[1], hh[2], hh[3]);
                    *(uint4*)(Al + off + 16 * c) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
                }
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        if (!tcu_team_and(team, ok1)) {
            mma_out = true;
            if (tt == 0) atomicCAS(&g_tcu_status, 0u, 2u);
            break;
        }
        mma_par ^= 1;
        if (tt == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            tcu_mma6(d2, ah, al, bh, bl, true);
            tcu_commit(&bar[1]);
        }
        const bool ok2 = __all_sync(0xffffffffu, tcu_wait(&bar[1], mma_par, u.spin));
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // ---- stage-2 row t (line l2, group k1): outputs k1 + 16 k2, staged in the A region ----
        unsigned char* ob = Ah;
        if (ok2) {
            tcu_ld32(d2 + lane_addr, v);
            const float g = tcu_pow2(e2) * fscale;
            const float gi = a.conj_out ? -g : g;
            if (g != 1.f || gi != 1.f) {
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    v[2 * q] *= g;
                    v[2 * q + 1] *= gi;
                }
            }
            if (rowk) {
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    *(float2*)(ob + l2 * 2048 + (k2r + 16 * q) * 8) = make_float2(v[2 * q], v[2 * q + 1]);
            } else {
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    *(float2*)(ob + tcu_st_off(k2r + 16 * q, l2)) = make_float2(v[2 * q], v[2 * q + 1]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        if (!tcu_team_and(team, ok2)) {
            mma_out = true;
            if (tt == 0) atomicCAS(&g_tcu_status, 0u, 3u);
            break;
        }
        mma_par ^= 1;
        if (tt == 0) {
            if (u.out_kind == TCU_OUT_ROW) {
                asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                                 (uint64_t)&omap),
                             "r"(0), "r"(j0), "r"((int)b), "r"(tcu_smem(ob))
                             : "memory");
            } else if (u.out_kind == TCU_OUT_COLSPLIT) {
                const int lo = a.logNs_out;
                asm volatile(
                    "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                        (uint64_t)&omap),
                    "r"(j0 & ((1 << lo) - 1)), "r"(0), "r"(j0 >> lo), "r"((int)b), "r"(tcu_smem(ob))
                    : "memory");
            } else {
                asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                                 (uint64_t)&omap),
                             "r"(j0), "r"(0), "r"((int)b), "r"(tcu_smem(ob))
                             : "memory");
            }
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
    }
    if (tt == 0) {   // the team's own copies and products
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
        if (mma_out) tcu_wait(&bar[1], mma_par, u.spin);   // abandoned launch: products still running
        if (pending) tcu_wait(&bar[0], in_par, u.spin);    // abandoned launch: a copy still in flight
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (t < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TCU_TCOLS) : "memory");
}

bool tc_umma_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("NOTORIOUS_FFT_TC_UMMA");
        v = e ? atoi(e) : 1;
    }
    return v != 0;
}

typedef CUresult (*TcuEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static TcuEncodeFn tcu_encoder() {
    static TcuEncodeFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (TcuEncodeFn)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// Tensor map of 8-byte elements (one complex float); strides in bytes.
static bool tcu_map(CUtensorMap* m, const void* base, int rank, const cuuint64_t* dims, const cuuint64_t* strides,
                    const cuuint32_t* box, CUtensorMapSwizzle sw) {
    TcuEncodeFn enc = tcu_encoder();
    if (!enc) return false;
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, (cuuint32_t)rank, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool try_launch_tc_umma(const PassArgs& a, int sm_count, cudaStream_t s, bool& launched) {
    launched = false;
    TcuArgs u;
    if (!tcu_shape(a, u)) return true;
    const long long B = u.a.cnt[1], Nj = u.a.cnt[0];
    const long long istr = B > 1 ? u.a.istr[1] * 8 : Nj * 256 * 8;
    const long long ostr = B > 1 ? u.a.ostr[1] * 8 : Nj * 256 * 8;
    CUtensorMap imap, omap;
    {
        const cuuint64_t dims[3] = {(cuuint64_t)Nj, 256, (cuuint64_t)B};
        const cuuint64_t strides[2] = {(cuuint64_t)(Nj * 8), (cuuint64_t)istr};
        const cuuint32_t box[3] = {TCU_J, 256, 1};
        if (!tcu_map(&imap, a.in, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_64B)) return true;
    }
    const int so = a.logNs_out;
    if (u.out_kind == TCU_OUT_ROW) {
        const cuuint64_t dims[3] = {256, (cuuint64_t)Nj, (cuuint64_t)B};
        const cuuint64_t strides[2] = {2048, (cuuint64_t)ostr};
        const cuuint32_t box[3] = {256, TCU_J, 1};
        if (!tcu_map(&omap, a.out, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_NONE)) return true;
    } else if (u.out_kind == TCU_OUT_COLSPLIT) {
        const cuuint64_t dims[4] = {(cuuint64_t)1 << so, 256, (cuuint64_t)(Nj >> so), (cuuint64_t)B};
        const cuuint64_t strides[3] = {(cuuint64_t)8 << so, (cuuint64_t)8 << (so + 8), (cuuint64_t)ostr};
        const cuuint32_t box[4] = {TCU_J, 256, 1, 1};
        if (!tcu_map(&omap, a.out, 4, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_64B)) return true;
    } else {
        const cuuint64_t dims[3] = {(cuuint64_t)Nj, 256, (cuuint64_t)B};
        const cuuint64_t strides[2] = {(cuuint64_t)8 << so, (cuuint64_t)ostr};
        const cuuint32_t box[3] = {TCU_J, 256, 1};
        if (!tcu_map(&omap, a.out, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_64B)) return true;
    }
    static bool attr = false;
    if (!attr) {
        if (!cuda_ok(cudaFuncSetAttribute((const void*)tc_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          TCU_SMEM),
                     "cudaFuncSetAttribute(tc umma)"))
            return false;
        if (!cuda_ok(cudaFuncSetAttribute((const void*)tc_umma_kernel,
                                          cudaFuncAttributePreferredSharedMemoryCarveout, 100),
                     "cudaFuncSetAttribute(tc umma carveout)"))
            return false;
        attr = true;
    }
    // NOTORIOUS_FFT_TC_UMMA_SPIN / _WITHHOLD: the failure test's short poll limit
    // and a first input copy that is never issued (every CTA's first wait runs out)
    static const long long spin = [] {
        const char* e = getenv("NOTORIOUS_FFT_TC_UMMA_SPIN");
        const long long v = e ? atoll(e) : 0;
        return v > 0 ? v : (1ll << 22);
    }();
    static const int withhold = [] {
        const char* e = getenv("NOTORIOUS_FFT_TC_UMMA_WITHHOLD");
        return e ? atoi(e) : 0;
    }();
    u.spin = spin;
    u.withhold = withhold;
    // resident CTAs: shared memory and registers allow TCU_MINB per SM
    // (the occupancy query does not count kernels that allocate tensor memory)
    const long long grid = std::min<long long>((u.ntiles + TCU_TEAMS - 1) / TCU_TEAMS,
                                               (long long)std::max(sm_count, 1) * TCU_MINB);
    if (grid <= 0) {
        launched = true;
        return true;
    }
    tc_umma_kernel<<<(unsigned)grid, TCU_THREADS, TCU_SMEM, s>>>(u, imap, omap);
    note_launch();
    s_tcu_used = true;
    launched = true;
    return cuda_ok(cudaGetLastError(), "tensor-core (tcgen05) radix-256 pass launch");
}

unsigned tc_umma_take_status() {
    if (!s_tcu_used) return 0;
    unsigned v = 0, z = 0;
    if (cudaMemcpyFromSymbol(&v, g_tcu_status, sizeof v) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (v) cudaMemcpyToSymbol(g_tcu_status, &z, sizeof z);
    return v;
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

bool tc_umma_enabled() { return false; }

bool try_launch_tc_umma(const PassArgs&, int, cudaStream_t, bool& launched) {
    launched = false;
    return true;
}

unsigned tc_umma_take_status() { return 0; }

bool launch_tc_pass(const PassArgs&, int, long long, cudaStream_t) {
    set_error(6, "the split tensor-core form exists in the float library only");
    return false;
}

#endif

}  // namespace nfft

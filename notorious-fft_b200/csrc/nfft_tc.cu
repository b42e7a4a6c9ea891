// nfft_tc.cu -- the split-tensor-core pass kernel of the float library
// (NOTORIOUS_FFT_FORM_SPLIT_TC): the generic Stockham pass (nfft_pass.cuh)
// with its radix-16 sub-stages computed by tc_substage (nfft_tc.cuh).
#include "nfft_engine.h"
#include "nfft_tc.cuh"

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

bool launch_tc_pass(const PassArgs&, int, long long, cudaStream_t) {
    set_error(6, "the split tensor-core form exists in the float library only");
    return false;
}

#endif

}  // namespace nfft

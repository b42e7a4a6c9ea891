// nfft_queue_branches.cuh -- the branches of the persistent queue kernel
// (nfft_queue_kernel.cu).  Each branch runs all tiles of one queue item with
// the same tile bodies as the standalone pass kernels.  The branches are
// separate, non-inlined device functions, instantiated in the translation
// units nfft_queue_b0..b4.cu (compiled in parallel as relocatable device code
// with the kernel's register budget) and reached through the kernel's
// dispatcher by the device linker.
#pragma once

#include "nfft_lean.cuh"
#include "nfft_queue.h"

namespace nfft {

template <typename T, int ST>
__device__ __forceinline__ void unpack_tile(const QDesc& d, long long tile) {
    const PassArgs& a = d.a;
    const TwTables<T>* tw = (const TwTables<T>*)a.tw;
    long long w0, w1;
    unpack_tile_range(a, tile, w0, w1);
    for (long long w = w0 + threadIdx.x; w < w1; w += QUEUE_THREADS)
        unpack_item<T, ST>(a, tw, (const C2<T>*)d.z, d.zdist, w);
}

template <typename T>
__device__ __forceinline__ void scalar_tile(const PassArgs& a, long long tile) {
    const long long i0 = tile * SCALAR_TILE;
    long long i1 = i0 + SCALAR_TILE;
    if (i1 > a.nlines) i1 = a.nlines;
    for (long long i = i0 + threadIdx.x; i < i1; i += QUEUE_THREADS) {
        const T* x = (const T*)a.in + a.in_tab[i];
        T* y = (T*)a.out + a.out_tab[i];
        const T re = (T)(a.scale * (double)x[0]);
        const T im = (a.conj_in && a.dst) ? (T)(a.scale * (double)x[1]) : (T)0;
        y[0] = re;
        if (a.conj_out) y[1] = im;
    }
}

template <typename T, int R, int CI, int CO, int LD, int ST>
__device__ __noinline__ void qb_lean(const QDesc* d, long long tile0, int ntiles, unsigned char* smraw) {
    for (int k = 0; k < ntiles; ++k) {
        lean_tile<T, R, QUEUE_LOGT, CI != 0, CO != 0, LD, ST>(d->a, tile0 + k, smraw);
        __syncthreads();
    }
}
template <typename T, int LD, int ST>
__device__ __noinline__ void qb_gen(const QDesc* d, long long tile0, int ntiles, unsigned char* smraw) {
    for (int k = 0; k < ntiles; ++k) {
        pass_tile<T, QUEUE_LOG_TILE, LD, ST>(d->a, tile0 + k, smraw);
        __syncthreads();
    }
}
template <typename T, int ST>
__device__ __noinline__ void qb_unpack(const QDesc* d, long long tile0, int ntiles) {
    for (int k = 0; k < ntiles; ++k) unpack_tile<T, ST>(*d, tile0 + k);
    __syncthreads();
}
template <typename T>
__device__ __noinline__ void qb_scalar(const QDesc* d, long long tile0, int ntiles) {
    for (int k = 0; k < ntiles; ++k) scalar_tile<T>(d->a, tile0 + k);
    __syncthreads();
}

}  // namespace nfft

// nfft_queue_kernel.cu -- the persistent kernel of the ragged-batch queue.
//
// One launch runs every item of a queue (nfft_queue.h).  Each CTA (256
// threads) loops: claim the next item with an atomic counter (the claim for
// the following item is issued before the current one runs, so its latency
// hides behind the work), copy the item's pass descriptor to shared memory,
// wait until the item's dependency counter is published, run the item's tiles
// through the branch its op names (the same tile bodies as the standalone
// pass kernels), then publish the tiles.
//
// Coherence: data read here may have been written earlier in the same launch
// by another SM, so this file is compiled with -Xptxas -dlcm=cg (global loads
// are served by L2, never by a stale L1 line) and scratch reads use the L2
// load hint.  Twiddle tables are read-only for the whole launch (ld.global.nc).
// Publishing is __syncthreads + __threadfence + atomicAdd; waiting is an
// acquire load of the counter followed by __syncthreads.
//
// Waits are bounded: after spin_limit polls the CTA raises the abort flag and
// records the item in the status word; every CTA checks the flag between
// items and in its own waits, so an abandoned launch drains quickly and the
// context stays usable.
#include "nfft_engine.h"
#include "nfft_lean.cuh"
#include "nfft_queue.h"

namespace nfft {

template <typename T>
constexpr size_t queue_tile_smem() {
    size_t m = pass_smem_bytes<T>(QUEUE_LOG_TILE);
#define X(R, CI, CO, LD, ST)                                                             \
    if (lean_smem_bytes<T, R, QUEUE_LOGT, CI != 0, CO != 0, LD, ST>() > m)              \
        m = lean_smem_bytes<T, R, QUEUE_LOGT, CI != 0, CO != 0, LD, ST>();
    NFFT_QUEUE_LEAN(X)
#undef X
    return (m + 15) / 16 * 16;
}
constexpr size_t QUEUE_TILE_SMEM = queue_tile_smem<real_t>();
constexpr size_t QUEUE_SMEM = QUEUE_TILE_SMEM + sizeof(QDesc);

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded wait of thread 0 for the item's dependency.  1: satisfied; 0: the
// launch is abandoned (this wait gave up, or another CTA's did).
__device__ __noinline__ int queue_wait(const QueueArgs& q, int wait, unsigned target, long long item) {
    unsigned ns = 32;
    for (long long n = 0;; ++n) {
        if (ld_acquire_u32(&q.ctr[wait]) >= target) return 1;
        if (ld_relaxed_u32(&q.ctr[QCTR_ABORT])) return 0;
        if (n >= q.spin_limit) {
            atomicExch(&q.ctr[QCTR_ABORT], 1u);
            atomicCAS(q.status, 0, (int)(item + 1));
            return 0;
        }
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
}

// Branch functions (nfft_queue_branches.cuh), compiled in the translation
// units nfft_queue_b0..b4.cu and linked as relocatable device code.
template <typename T, int R, int CI, int CO, int LD, int ST>
__device__ void qb_lean(const QDesc* d, long long tile0, int ntiles, unsigned char* smraw);
template <typename T, int LD, int ST>
__device__ void qb_gen(const QDesc* d, long long tile0, int ntiles, unsigned char* smraw);
template <typename T, int ST>
__device__ void qb_unpack(const QDesc* d, long long tile0, int ntiles);
template <typename T>
__device__ void qb_scalar(const QDesc* d, long long tile0, int ntiles);

template <typename T>
__device__ __forceinline__ void queue_run_item(int op, const QDesc* d, long long tile0, int ntiles,
                                               unsigned char* smraw) {
    switch (op) {
#define X(R, CI, CO, LD, ST)                                                                  \
    case qop_lean(R, CI, CO, LD, ST): qb_lean<T, R, CI, CO, LD, ST>(d, tile0, ntiles, smraw); break;
        NFFT_QUEUE_LEAN(X)
#undef X
#define X(LD, ST)                                                                             \
    case qop_gen(LD, ST): qb_gen<T, LD, ST>(d, tile0, ntiles, smraw); break;
        NFFT_QUEUE_GENERIC(X)
#undef X
    case qop_unpack(ST_R): qb_unpack<T, ST_R>(d, tile0, ntiles); break;
    case qop_unpack(ST_T2): qb_unpack<T, ST_T2>(d, tile0, ntiles); break;
    case QOP_SCALAR: qb_scalar<T>(d, tile0, ntiles); break;
    default: __syncthreads(); break;
    }
}

template <typename T>
__global__ void __launch_bounds__(QUEUE_THREADS, 2) queue_kernel(const QueueArgs q) {
    extern __shared__ __align__(16) unsigned char smraw[];
    QDesc* sd = (QDesc*)(smraw + QUEUE_TILE_SMEM);
    __shared__ long long s_item;
    __shared__ int s_go;
    const int t = threadIdx.x;
    unsigned claim = 0;
    if (t == 0) claim = atomicAdd(&q.ctr[QCTR_NEXT], 1u);
    for (;;) {
        if (t == 0) {
            s_item = claim;
            s_go = ((long long)claim < q.nitems) && !ld_relaxed_u32(&q.ctr[QCTR_ABORT]);
            if (s_go) claim = atomicAdd(&q.ctr[QCTR_NEXT], 1u);   // next claim in flight during this item
        }
        __syncthreads();
        if (!s_go) break;
        const long long item = s_item;
        const QItem it = q.items[item];
        {
            const int* src = (const int*)&q.descs[it.desc];
            int* dst = (int*)sd;
            for (int w = t; w < (int)(sizeof(QDesc) / sizeof(int)); w += QUEUE_THREADS) dst[w] = src[w];
        }
        __syncthreads();
        if (t == 0) {
            if (sd->flags & QD_IN_USER) sd->a.in = (const char*)q.user_in + (size_t)sd->a.in;
            if (sd->flags & QD_OUT_USER) sd->a.out = (char*)q.user_out + (size_t)sd->a.out;
            s_go = it.wait >= 0 ? queue_wait(q, it.wait, (unsigned)it.target, item) : 1;
        }
        __syncthreads();
        if (!s_go) break;
        queue_run_item<T>(it.op, sd, it.tile0, it.ntiles, smraw);   // ends with __syncthreads
        if (t == 0 && it.done >= 0) {
            __threadfence();
            atomicAdd(&q.ctr[it.done], (unsigned)it.ntiles);
        }
    }
}

size_t queue_smem_bytes() { return QUEUE_SMEM; }

// Resident CTAs of the queue kernel on this device (the persistent grid).
int queue_grid(const DeviceCtx* c) {
    static int attr_set[64] = {};
    const int dev = c->device;
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        if (!cuda_ok(cudaFuncSetAttribute((const void*)queue_kernel<real_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)QUEUE_SMEM),
                     "cudaFuncSetAttribute(queue kernel)"))
            return 0;
        attr_set[dev] = 1;
    }
    int per_sm = 0;
    if (!cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, queue_kernel<real_t>, QUEUE_THREADS, QUEUE_SMEM),
                 "queue kernel occupancy"))
        return 0;
    if (per_sm < 1) {
        set_error(4, "the queue kernel does not fit on an SM");
        return 0;
    }
    return per_sm * c->sm_count;
}

bool launch_queue(const QueueArgs& q, int grid, cudaStream_t s) {
    queue_kernel<real_t><<<grid, QUEUE_THREADS, QUEUE_SMEM, s>>>(q);
    return cuda_ok(cudaGetLastError(), "queue kernel launch");
}

}  // namespace nfft

// nfft_resident.cu -- dispatcher of the resident two-pass kernels
// (nfft_resident.cuh): registry, kernel attributes, persistent grid, lag.
#include <stdlib.h>

#include <algorithm>

#include <cuda.h>

#include "nfft_engine.h"
#include "nfft_resident.cuh"
#include "nfft_resident_tma.cuh"

namespace nfft {

void resident_register_a(std::vector<ResidentEntry>& v);
void resident_register_b(std::vector<ResidentEntry>& v);

const std::vector<ResidentEntry>& resident_registry() {
    static std::vector<ResidentEntry> r = [] {
        std::vector<ResidentEntry> v;
        resident_register_a(v);
        resident_register_b(v);
        return v;
    }();
    return r;
}

const ResidentEntry* resident_find(int r1, int r2) {
    for (auto& e : resident_registry())
        if (e.r1 == r1 && e.r2 == r2) return &e;
    return nullptr;
}

void resident_register_tma(std::vector<ResidentTmaEntry>& v);

static const std::vector<ResidentTmaEntry>& resident_tma_registry() {
    static std::vector<ResidentTmaEntry> r = [] {
        std::vector<ResidentTmaEntry> v;
        resident_register_tma(v);
        return v;
    }();
    return r;
}

const ResidentTmaEntry* resident_tma_find(int r1, int r2) {
    for (auto& e : resident_tma_registry())
        if (e.r1 == r1 && e.r2 == r2) return &e;
    return nullptr;
}

bool resident_set_attributes() {
    for (auto& e : resident_registry())
        if (!cuda_ok(cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem),
                     "cudaFuncSetAttribute(resident kernel)") ||
            !cuda_ok(cudaFuncSetAttribute(e.fn_pf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem_pf),
                     "cudaFuncSetAttribute(resident kernel)"))
            return false;
    for (auto& e : resident_tma_registry())
        if (!cuda_ok(cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem),
                     "cudaFuncSetAttribute(resident tensor-copy kernel)"))
            return false;
    return true;
}

// NOTORIOUS_FFT_RESIDENT_PREFETCH=1 selects the software-pipelined resident
// kernels (tile k+1 staged by cp.async while tile k computes).  Off by
// default: its staging buffer costs one CTA per SM, and on B200 that loses
// more than the hidden load latency gains.
static bool prefetch_enabled() {
    static const int v = [] {
        const char* e = getenv("NOTORIOUS_FFT_RESIDENT_PREFETCH");
        return (e && atoi(e) != 0) ? 1 : 0;
    }();
    return v == 1;
}

// Persistent CTAs of one kernel on this device.
static int resident_grid(const void* fn, int threads, size_t smem, const DeviceCtx* c) {
    int per_sm = 0;
    if (!cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem), "resident kernel occupancy"))
        return 0;
    return std::max(1, per_sm) * c->sm_count;
}

// cuTensorMapEncodeTiled from the driver (resolved once; no link-time
// dependency on the driver library).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (EncodeTiledFn) nullptr;
        }
        return (EncodeTiledFn)p;
    }();
    return fn;
}

// Tensor map of one pass input (tma_pass_geom); false when the buffer does
// not meet the copy engine's rules (16-byte base and strides).
static bool encode_pass_map(CUtensorMap* m, const PassArgs& a, int logR, int logJ, long long B) {
    EncodeTiledFn fn = encode_tiled();
    if (!fn || a.in_estride != 1) return false;
    const long long bstride = a.ndims > 1 ? a.istr[1] : (1ll << (a.logNj + logR));
    const TmaPassGeom g = tma_pass_geom(a.logNj, logR, logJ, B, bstride, sizeof(cplx_t));
    if (((uintptr_t)a.in & 15) || (g.stride_bytes[0] & 15) || (g.stride_bytes[1] & 15) ||
        g.stride_bytes[1] >= (1ull << 40) || g.dim[2] >= (1ull << 31))
        return false;
    const cuuint32_t es[3] = {1, 1, 1};
    const CUresult rc = fn(m, sizeof(real_t) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                           3, const_cast<void*>(a.in), (const cuuint64_t*)g.dim, (const cuuint64_t*)g.stride_bytes,
                           (const cuuint32_t*)g.box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return rc == CUDA_SUCCESS;
}

// NOTORIOUS_FFT_RESIDENT=2: the tensor-copy-fed kernel where one is listed.
static bool tma_variant_selected() {
    static const int v = [] {
        const char* e = getenv("NOTORIOUS_FFT_RESIDENT");
        return e ? atoi(e) : 0;
    }();
    return v == 2;
}

static bool launch_resident_tma(const DeviceCtx* c, const ResidentTmaEntry* e, const PassArgs& a1,
                                const PassArgs& a2, long long B, unsigned* ctr, long long spin, cudaStream_t s) {
    const int logt = e->logt;
    CUtensorMap m1, m2;
    if (!encode_pass_map(&m1, a1, e->r1, logt + 4 - e->r1, B) || !encode_pass_map(&m2, a2, e->r2, logt + 4 - e->r2, B))
        return false;
    ResidentArgs r;
    r.B = B;
    r.log_tiles = e->r1 + e->r2 - (logt + 4);
    const long long T = 1ll << r.log_tiles;
    const int grid = c->sm_count;   // one CTA per SM
    // lag: every group of a CTA holds up to two items; the pass-2 tiles of a
    // transform are claimed about 1.25 windows after its pass-1 tiles
    static const long long target_kb = [] {
        const char* v = getenv("NOTORIOUS_FFT_RESIDENT_KB");
        return v ? std::max(1ll, atoll(v)) : 32768ll;
    }();
    const long long per = (1ll << (e->r1 + e->r2)) * (long long)sizeof(cplx_t);
    const long long window = (long long)grid * (e->stages + 1);
    r.lag = std::max((5 * window + 4 * 2 * T - 1) / (4 * 2 * T), (target_kb << 10) / per);
    if (r.lag < 1) r.lag = 1;
    if (r.lag > B) r.lag = B;
    r.ctr = ctr;
    r.status = (int*)(ctr + 2 + B);
    r.spin_limit = spin;
    if (!cuda_ok(cudaMemsetAsync(ctr, 0, sizeof(unsigned) * (size_t)(B + 3), s), "resident counter reset")) return false;
    void* args[5] = {(void*)&m1, (void*)&m2, (void*)&a1, (void*)&a2, (void*)&r};
    note_launch();
    return cuda_ok(cudaLaunchKernel(e->fn, dim3(grid), dim3(e->ng << logt), args, e->smem, s),
                   "resident tensor-copy kernel launch");
}

bool launch_resident(const DeviceCtx* c, const PassArgs& a1, const PassArgs& a2, int r1, int r2, long long B,
                     unsigned* ctr, cudaStream_t s) {
    const ResidentEntry* e = resident_find(r1, r2);
    if (!e) {
        set_error(6, "no resident kernel for radices 2^%d x 2^%d", r1, r2);
        return false;
    }
    const bool pf = prefetch_enabled();
    const void* fn = pf ? e->fn_pf : e->fn;
    const size_t smem = pf ? e->smem_pf : e->smem;
    const int grid = resident_grid(fn, 1 << e->logt, smem, c);
    if (grid <= 0) return false;
    ResidentArgs r;
    r.B = B;
    r.log_tiles = r1 + r2 - (e->logt + 4);
    const long long T = 1ll << r.log_tiles;
    // lag: enough items between a transform's two passes that its pass-1 tiles
    // have finished when its pass-2 tiles are claimed (about two items per CTA
    // are in flight), and about NOTORIOUS_FFT_RESIDENT_KB of scratch in flight
    static const long long target_kb = [] {
        const char* v = getenv("NOTORIOUS_FFT_RESIDENT_KB");
        return v ? std::max(1ll, atoll(v)) : 32768ll;
    }();
    const long long per = (1ll << (r1 + r2)) * (long long)sizeof(cplx_t);
    const long long need = (5 * (2ll * grid + T) + 4 * 2 * T - 1) / (4 * 2 * T);   // 1.25 x window, in transforms
    r.lag = std::max(need, (target_kb << 10) / per);
    if (r.lag < 1) r.lag = 1;
    if (r.lag > B) r.lag = B;
    r.ctr = ctr;
    r.status = (int*)(ctr + 2 + B);
    static const long long spin = [] {
        const char* v = getenv("NOTORIOUS_FFT_QUEUE_SPIN");
        return v ? std::max(1ll, atoll(v)) : (1ll << 22);
    }();
    r.spin_limit = spin;
    if ((B << (r.log_tiles + 1)) >= (1ll << 32)) {
        set_error(6, "resident launch of %lld transforms exceeds its claim counter", B);
        return false;
    }
    if (tma_variant_selected()) {
        const ResidentTmaEntry* te = resident_tma_find(r1, r2);
        if (te && launch_resident_tma(c, te, a1, a2, B, ctr, spin, s)) return true;
        if (last_error()) return false;
    }
    if (!cuda_ok(cudaMemsetAsync(ctr, 0, sizeof(unsigned) * (size_t)(B + 3), s), "resident counter reset")) return false;
    void* args[3] = {(void*)&a1, (void*)&a2, (void*)&r};
    note_launch();
    return cuda_ok(cudaLaunchKernel(fn, dim3(grid), dim3(1 << e->logt), args, smem, s), "resident kernel launch");
}

}  // namespace nfft

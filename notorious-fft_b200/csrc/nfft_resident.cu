// nfft_resident.cu -- dispatcher of the resident two-pass kernels
// (nfft_resident.cuh): registry, kernel attributes, persistent grid, lag.
#include <stdlib.h>

#include <algorithm>

#include "nfft_engine.h"
#include "nfft_resident.cuh"

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

bool resident_set_attributes() {
    for (auto& e : resident_registry())
        if (!cuda_ok(cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem),
                     "cudaFuncSetAttribute(resident kernel)") ||
            !cuda_ok(cudaFuncSetAttribute(e.fn_pf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem_pf),
                     "cudaFuncSetAttribute(resident kernel)"))
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
    if (!cuda_ok(cudaMemsetAsync(ctr, 0, sizeof(unsigned) * (size_t)(B + 3), s), "resident counter reset")) return false;
    void* args[3] = {(void*)&a1, (void*)&a2, (void*)&r};
    note_launch();
    return cuda_ok(cudaLaunchKernel(fn, dim3(grid), dim3(1 << e->logt), args, smem, s), "resident kernel launch");
}

}  // namespace nfft

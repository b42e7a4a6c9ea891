// nfft_mid.cu -- the Bluestein middle kernels (lean_mid_kernel, nfft_lean.cuh):
// the last pass of the forward M-point FFT, the filter product and the first
// pass of the second FFT in one launch.  Registry, attributes, launch.
#include "nfft_engine.h"
#include "nfft_lean.cuh"

namespace nfft {

namespace {
struct MidEntry {
    int logr, logt;
    const void* fn;
    size_t smem;
};
// radix 2^5 .. 2^8 on 2048-point tiles, 2^9 / 2^10 on 4096-point tiles
#define NFFT_MID_LIST(X) X(5, 7) X(6, 7) X(7, 7) X(8, 7) X(9, 8) X(10, 8)
const MidEntry* mid_find(int logR) {
    static const MidEntry tab[] = {
#define X(R, T) {R, T, (const void*)lean_mid_kernel<real_t, R, T>, LeanMid<real_t, R, T>::SMEM_BYTES},
        NFFT_MID_LIST(X)
#undef X
    };
    for (const auto& e : tab)
        if (e.logr == logR) return &e;
    return nullptr;
}
}  // namespace

bool lean_mid_available(int logR) { return mid_find(logR) != nullptr; }

bool mid_set_attributes() {
    for (int r = 5; r <= 10; ++r)
        if (const MidEntry* e = mid_find(r))
            if (!cuda_ok(cudaFuncSetAttribute(e->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e->smem),
                         "cudaFuncSetAttribute(Bluestein middle)"))
                return false;
    return true;
}

bool launch_lean_mid(PassArgs a1, PassArgs a2, int logR, cudaStream_t s) {
    const MidEntry* e = mid_find(logR);
    if (!e) {
        set_error(6, "no Bluestein middle kernel for radix 2^%d", logR);
        return false;
    }
    a1.logJ = a2.logJ = e->logt + 4 - logR;
    const long long ntiles = (a1.nlines + (1ll << a1.logJ) - 1) >> a1.logJ;
    if (ntiles <= 0) return true;
    dim3 grid;
    if (ntiles <= 0x7fffffffll) grid = dim3((unsigned)ntiles, 1, 1);
    else grid = dim3(0x7fffffffu, (unsigned)((ntiles + 0x7fffffffll - 1) / 0x7fffffffll), 1);
    void* args[] = {(void*)&a1, (void*)&a2};
    note_launch();
    return cuda_ok(cudaLaunchKernel(e->fn, grid, dim3(1u << e->logt, 1, 1), args, e->smem, s),
                   "Bluestein middle kernel launch");
}

}  // namespace nfft

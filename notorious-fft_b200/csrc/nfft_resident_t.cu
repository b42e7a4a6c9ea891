// nfft_resident_t.cu -- instantiation of the resident two-pass kernels fed by
// tensor copies (NFFT_RESIDENT_TMA of nfft_resident_list.h), registered with
// the dispatcher in nfft_resident.cu.
#include "nfft_engine.h"
#include "nfft_resident_list.h"
#include "nfft_resident_tma.cuh"

namespace nfft {

void resident_register_tma(std::vector<ResidentTmaEntry>& v) {
#define X(R1, R2, LT, NG)                                                                                \
    v.push_back(ResidentTmaEntry{R1, R2, LT, NG, TmaRes<real_t, R1, R2, LT>::stages(NG),                \
                                 (const void*)tma_resident_kernel<real_t, R1, R2, LT, NG>,              \
                                 TmaRes<real_t, R1, R2, LT>::smem_bytes(NG)});
    NFFT_RESIDENT_TMA(X)
#undef X
}

}  // namespace nfft

// nfft_resident_b.cu -- instantiation of resident two-pass kernels (list B of
// nfft_resident_list.h), registered with the dispatcher in nfft_resident.cu.
#include "nfft_engine.h"
#include "nfft_resident.cuh"
#include "nfft_resident_list.h"

namespace nfft {

void resident_register_b(std::vector<ResidentEntry>& v) {
#define X(R1, R2, LT)                                                                                  \
    v.push_back(ResidentEntry{R1, R2, LT, (const void*)resident_kernel<real_t, R1, R2, LT>,            \
                              resident_smem_bytes<real_t, R1, R2, LT>(),                                \
                              (const void*)resident_pf_kernel<real_t, R1, R2, LT>,                      \
                              resident_pf_smem_bytes<real_t, R1, R2, LT>()});
    NFFT_RESIDENT_B(X)
#undef X
}

}  // namespace nfft

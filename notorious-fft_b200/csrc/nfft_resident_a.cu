// nfft_resident_a.cu -- instantiation of resident two-pass kernels (list A of
// nfft_resident_list.h), registered with the dispatcher in nfft_resident.cu.
#include "nfft_engine.h"
#include "nfft_resident.cuh"
#include "nfft_resident_list.h"

namespace nfft {

void resident_register_a(std::vector<ResidentEntry>& v) {
#define X(R1, R2, LT)                                                                                  \
    v.push_back(ResidentEntry{R1, R2, LT, (const void*)resident_kernel<real_t, R1, R2, LT>,            \
                              resident_smem_bytes<real_t, R1, R2, LT>(),                                \
                              (const void*)resident_pf_kernel<real_t, R1, R2, LT>,                      \
                              resident_pf_smem_bytes<real_t, R1, R2, LT>()});
    NFFT_RESIDENT_A(X)
#undef X
}

}  // namespace nfft

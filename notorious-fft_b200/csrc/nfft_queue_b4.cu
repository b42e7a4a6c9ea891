// nfft_queue_b4.cu -- queue kernel branches: multi-pass Bluestein passes.
#include "nfft_engine.h"
#include "nfft_queue_branches.cuh"

namespace nfft {

#define X(R, CI, CO, LD, ST) \
    template __device__ void qb_lean<real_t, R, CI, CO, LD, ST>(const QDesc*, long long, int, unsigned char*);
NFFT_QUEUE_LEAN_D(X)
#undef X

}  // namespace nfft

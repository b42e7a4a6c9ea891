// nfft_queue_b3.cu -- queue kernel branches: generic passes, unpack epilogues and size-1 transforms.
#include "nfft_engine.h"
#include "nfft_queue_branches.cuh"

namespace nfft {

#define X(LD, ST) template __device__ void qb_gen<real_t, LD, ST>(const QDesc*, long long, int, unsigned char*);
NFFT_QUEUE_GENERIC(X)
#undef X
template __device__ void qb_unpack<real_t, ST_R>(const QDesc*, long long, int);
template __device__ void qb_unpack<real_t, ST_T2>(const QDesc*, long long, int);
template __device__ void qb_scalar<real_t>(const QDesc*, long long, int);

}  // namespace nfft

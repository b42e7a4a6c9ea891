// One slice of the specialized pass kernels (see nfft_lean_slice.cuh).
#define NFFT_LEAN_SLICE 4
#include "nfft_lean_slice.cuh"

// One slice of the specialized pass kernels (see nfft_lean_slice.cuh).
#define NFFT_LEAN_SLICE 5
#include "nfft_lean_slice.cuh"

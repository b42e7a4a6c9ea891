// nfft_resident_list.h -- instantiated resident two-pass kernels:
// X(LOGR1, LOGR2, LOGT) for N = 2^(LOGR1 + LOGR2).  128-thread tiles (2048
// points, 4 CTAs per SM) while both passes keep the column-mode minimum of
// 64 contiguous bytes per tile row; 256 / 512 threads for the largest radices.
#pragma once

#if defined(NFFT_REAL_IS_FLOAT) && NFFT_REAL_IS_FLOAT
#define NFFT_RESIDENT_A(X) X(7, 6, 7) X(7, 7, 7) X(8, 7, 7) X(8, 8, 7)
#define NFFT_RESIDENT_B(X) X(9, 8, 8) X(9, 9, 8) X(10, 9, 9) X(10, 10, 9)
#else
#define NFFT_RESIDENT_A(X) X(7, 6, 7) X(7, 7, 7) X(8, 7, 7) X(8, 8, 7)
#define NFFT_RESIDENT_B(X) X(9, 8, 7) X(9, 9, 7) X(10, 9, 8) X(10, 10, 8)
#endif

// Resident kernels fed by tensor copies (nfft_resident_tma.cuh):
// X(LOGR1, LOGR2, LOGT, NG) with NG consumer groups of 2^LOGT threads per CTA.
#if defined(NFFT_REAL_IS_FLOAT) && NFFT_REAL_IS_FLOAT
#define NFFT_RESIDENT_TMA(X) X(7, 6, 7, 6) X(7, 7, 7, 6) X(8, 7, 7, 6) X(8, 8, 7, 6)
#else
#define NFFT_RESIDENT_TMA(X) X(7, 6, 7, 3) X(7, 7, 7, 3) X(8, 7, 7, 3) X(8, 8, 7, 3)
#endif

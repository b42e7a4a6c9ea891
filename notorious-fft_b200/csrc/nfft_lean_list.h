// nfft_lean_list.h -- the specialized pass kernels that are instantiated.
// X(LOGR, LOGT, COL_IN, COL_OUT, LOAD, STORE); one entry per kernel.
// LOGT: 256 threads (tile of 4096 points) unless the pass radix and the
// column-mode minimum of 4 lines per tile need 512 threads.
#pragma once

#define NFFT_LEAN_LT(R, ROW) (((R) <= 12 && ((ROW) || (R) <= 10)) ? 8 : 9)

// complex passes: row/row (single-pass), col/row (first of several), col/col
#define NFFT_LEAN_C2C(X)                                                                           \
    X(4, 8, 0, 0, LD_C, ST_C) X(5, 8, 0, 0, LD_C, ST_C) X(6, 8, 0, 0, LD_C, ST_C)                  \
    X(7, 8, 0, 0, LD_C, ST_C) X(8, 8, 0, 0, LD_C, ST_C) X(9, 8, 0, 0, LD_C, ST_C)                  \
    X(10, 8, 0, 0, LD_C, ST_C) X(11, 8, 0, 0, LD_C, ST_C) X(12, 8, 0, 0, LD_C, ST_C)               \
    X(13, 9, 0, 0, LD_C, ST_C)                                                                     \
    X(5, 8, 1, 0, LD_C, ST_C) X(6, 8, 1, 0, LD_C, ST_C) X(7, 8, 1, 0, LD_C, ST_C)                  \
    X(8, 8, 1, 0, LD_C, ST_C) X(9, 8, 1, 0, LD_C, ST_C) X(10, 8, 1, 0, LD_C, ST_C)                 \
    X(11, 9, 1, 0, LD_C, ST_C)                                                                     \
    X(4, 8, 1, 1, LD_C, ST_C) X(5, 8, 1, 1, LD_C, ST_C) X(6, 8, 1, 1, LD_C, ST_C)                  \
    X(7, 8, 1, 1, LD_C, ST_C) X(8, 8, 1, 1, LD_C, ST_C) X(9, 8, 1, 1, LD_C, ST_C)                  \
    X(10, 8, 1, 1, LD_C, ST_C) X(11, 9, 1, 1, LD_C, ST_C)

// single-pass real families (whole contiguous lines)
#define NFFT_LEAN_REAL_ONE(X, R, T)                                                                \
    X(R, T, 0, 0, LD_R2C, ST_R) X(R, T, 0, 0, LD_IR, ST_C2R) X(R, T, 0, 0, LD_T2, ST_T2)           \
    X(R, T, 0, 0, LD_T3, ST_T3) X(R, T, 0, 0, LD_T4, ST_T4)
#define NFFT_LEAN_REAL(X)                                                                          \
    NFFT_LEAN_REAL_ONE(X, 4, 8) NFFT_LEAN_REAL_ONE(X, 5, 8) NFFT_LEAN_REAL_ONE(X, 6, 8)            \
    NFFT_LEAN_REAL_ONE(X, 7, 8) NFFT_LEAN_REAL_ONE(X, 8, 8) NFFT_LEAN_REAL_ONE(X, 9, 8)            \
    NFFT_LEAN_REAL_ONE(X, 10, 8) NFFT_LEAN_REAL_ONE(X, 11, 8) NFFT_LEAN_REAL_ONE(X, 12, 8)         \
    NFFT_LEAN_REAL_ONE(X, 13, 9)

// first / last passes of multi-pass real transforms (the realdft / DCT-2 last
// passes unpack in mirror tiles)
#define NFFT_LEAN_MULTI_ONE(X, R, T)                                                               \
    X(R, T, 1, 0, LD_R2C, ST_C) X(R, T, 1, 0, LD_IR, ST_C) X(R, T, 1, 0, LD_T2, ST_C)             \
    X(R, T, 1, 0, LD_T3, ST_C) X(R, T, 1, 0, LD_T4, ST_C) X(R, T, 1, 1, LD_C, ST_C2R)             \
    X(R, T, 1, 1, LD_C, ST_T3) X(R, T, 1, 1, LD_C, ST_T4) X(R, T, 1, 1, LD_C, ST_R)              \
    X(R, T, 1, 1, LD_C, ST_T2)
#define NFFT_LEAN_MULTI(X)                                                                         \
    NFFT_LEAN_MULTI_ONE(X, 5, 8) NFFT_LEAN_MULTI_ONE(X, 6, 8) NFFT_LEAN_MULTI_ONE(X, 7, 8)         \
    NFFT_LEAN_MULTI_ONE(X, 8, 8) NFFT_LEAN_MULTI_ONE(X, 9, 8) NFFT_LEAN_MULTI_ONE(X, 10, 8)        \
    NFFT_LEAN_MULTI_ONE(X, 11, 9)

// complex passes on 2048-point tiles (128 threads: more CTAs per SM)
#define NFFT_LEAN_C2C_T7(X)                                                                        \
    X(4, 7, 0, 0, LD_C, ST_C) X(5, 7, 0, 0, LD_C, ST_C) X(6, 7, 0, 0, LD_C, ST_C)                  \
    X(7, 7, 0, 0, LD_C, ST_C) X(8, 7, 0, 0, LD_C, ST_C) X(9, 7, 0, 0, LD_C, ST_C)                  \
    X(10, 7, 0, 0, LD_C, ST_C) X(11, 7, 0, 0, LD_C, ST_C)                                          \
    X(5, 7, 1, 0, LD_C, ST_C) X(6, 7, 1, 0, LD_C, ST_C) X(7, 7, 1, 0, LD_C, ST_C)                  \
    X(8, 7, 1, 0, LD_C, ST_C) X(9, 7, 1, 0, LD_C, ST_C)                                            \
    X(4, 7, 1, 1, LD_C, ST_C) X(5, 7, 1, 1, LD_C, ST_C) X(6, 7, 1, 1, LD_C, ST_C)                  \
    X(7, 7, 1, 1, LD_C, ST_C) X(8, 7, 1, 1, LD_C, ST_C) X(9, 7, 1, 1, LD_C, ST_C)

// multi-pass Bluestein: chirp premultiply (first forward pass), filter product
// (first inverse pass), window + chirp postmultiply (last inverse pass)
#define NFFT_LEAN_BLUE(X)                                                                          \
    X(5, 8, 1, 0, LD_BLUE, ST_C) X(6, 8, 1, 0, LD_BLUE, ST_C) X(7, 8, 1, 0, LD_BLUE, ST_C)         \
    X(8, 8, 1, 0, LD_BLUE, ST_C) X(9, 8, 1, 0, LD_BLUE, ST_C) X(10, 8, 1, 0, LD_BLUE, ST_C)        \
    X(11, 9, 1, 0, LD_BLUE, ST_C)                                                                  \
    X(5, 8, 1, 0, LD_FILT, ST_C) X(6, 8, 1, 0, LD_FILT, ST_C) X(7, 8, 1, 0, LD_FILT, ST_C)         \
    X(8, 8, 1, 0, LD_FILT, ST_C) X(9, 8, 1, 0, LD_FILT, ST_C) X(10, 8, 1, 0, LD_FILT, ST_C)        \
    X(11, 9, 1, 0, LD_FILT, ST_C)                                                                  \
    X(4, 8, 1, 1, LD_C, ST_BLUE) X(5, 8, 1, 1, LD_C, ST_BLUE) X(6, 8, 1, 1, LD_C, ST_BLUE)         \
    X(7, 8, 1, 1, LD_C, ST_BLUE) X(8, 8, 1, 1, LD_C, ST_BLUE) X(9, 8, 1, 1, LD_C, ST_BLUE)         \
    X(10, 8, 1, 1, LD_C, ST_BLUE) X(11, 9, 1, 1, LD_C, ST_BLUE)

// the fused operators of multi-pass real and Bluestein transforms on 2048-point
// tiles for the radices whose column tiles keep >= 8 lines (the planner takes
// them where it prefers 128-thread tiles, as for the complex passes)
#define NFFT_LEAN_OPS_T7_ONE(X, R)                                                                 \
    NFFT_LEAN_MULTI_ONE(X, R, 7)                                                                   \
    X(R, 7, 1, 0, LD_BLUE, ST_C) X(R, 7, 1, 0, LD_FILT, ST_C) X(R, 7, 1, 1, LD_C, ST_BLUE)
#define NFFT_LEAN_OPS_T7(X) NFFT_LEAN_OPS_T7_ONE(X, 6) NFFT_LEAN_OPS_T7_ONE(X, 7) NFFT_LEAN_OPS_T7_ONE(X, 8)

#define NFFT_LEAN_ALL(X)                                                                           \
    NFFT_LEAN_C2C(X) NFFT_LEAN_REAL(X) NFFT_LEAN_MULTI(X) NFFT_LEAN_C2C_T7(X) NFFT_LEAN_BLUE(X)     \
    NFFT_LEAN_OPS_T7(X)

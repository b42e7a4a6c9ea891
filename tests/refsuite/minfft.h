/*
 * minfft.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A stand-in for minfft, the third-party library the reference project's own
 * test programs (tests/test_notoriousfft.c, tests/test_notoriousfft.cpp of
 * NotoriousLOB/Notorious-FFT) use as their oracle.  The reference fetches it
 * at configure time from github.com/aimukhin/minfft with an unpinned
 * `GIT_TAG master` (CMakeLists.txt:113-129); it is not available here.
 *
 * Only the part of minfft's interface those programs call is declared: the
 * types (minfft_real = double, minfft_cmpl = interleaved real[2], an opaque
 * minfft_aux), the 1-D/2-D/3-D plan constructors they use, the ten transforms
 * and minfft_free_aux.  minfft defines the same unnormalized transforms the
 * reference does (FFTW sign and layout conventions, N/2+1 real output), so
 * the definitions are answered by this repository's long-double oracle
 * (oracle/nfft_oracle.c) in minfft_oracle.c.
 */
#ifndef MINFFT_STANDIN_H
#define MINFFT_STANDIN_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double minfft_real;
typedef minfft_real minfft_cmpl[2];
typedef struct minfft_aux minfft_aux;

minfft_aux* minfft_mkaux_dft_1d(int N);
minfft_aux* minfft_mkaux_dft_2d(int N1, int N2);
minfft_aux* minfft_mkaux_dft_3d(int N1, int N2, int N3);
minfft_aux* minfft_mkaux_realdft_1d(int N);
minfft_aux* minfft_mkaux_t2t3_1d(int N);
minfft_aux* minfft_mkaux_t2t3_2d(int N1, int N2);
minfft_aux* minfft_mkaux_t2t3_3d(int N1, int N2, int N3);
minfft_aux* minfft_mkaux_t4_1d(int N);
minfft_aux* minfft_mkaux_t4_2d(int N1, int N2);
minfft_aux* minfft_mkaux_t4_3d(int N1, int N2, int N3);

void minfft_dft(minfft_cmpl* x, minfft_cmpl* y, const minfft_aux* a);
void minfft_invdft(minfft_cmpl* x, minfft_cmpl* y, const minfft_aux* a);
void minfft_realdft(minfft_real* x, minfft_cmpl* z, const minfft_aux* a);
void minfft_invrealdft(minfft_cmpl* z, minfft_real* y, const minfft_aux* a);
void minfft_dct2(minfft_real* x, minfft_real* y, const minfft_aux* a);
void minfft_dst2(minfft_real* x, minfft_real* y, const minfft_aux* a);
void minfft_dct3(minfft_real* x, minfft_real* y, const minfft_aux* a);
void minfft_dst3(minfft_real* x, minfft_real* y, const minfft_aux* a);
void minfft_dct4(minfft_real* x, minfft_real* y, const minfft_aux* a);
void minfft_dst4(minfft_real* x, minfft_real* y, const minfft_aux* a);

void minfft_free_aux(minfft_aux* a);

#ifdef __cplusplus
}
#endif

#endif /* MINFFT_STANDIN_H */

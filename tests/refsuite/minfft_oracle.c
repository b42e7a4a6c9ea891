/*
 * minfft_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * The minfft stand-in of minfft.h, answered by the oracle's long-double C
 * restatement (oracle/nfft_oracle.c, linked as oracle/_build/liboracle_d.so).
 * A plan only records the shape; every call evaluates the definition afresh.
 * Nothing here is product code: it exists so that the reference project's
 * own test programs can run unchanged against libnotorious_fft.so.
 */
#include <stdlib.h>

#include "minfft.h"

/* oracle/nfft_oracle.c, double build */
void oracle_d_dft(const double* x, double* y, long N, int inverse);
void oracle_d_realdft(const double* x, double* z, long N);
void oracle_d_invrealdft(const double* z, double* y, long N);
void oracle_d_r2r(int kind, const double* x, double* y, long N);
void oracle_d_dft_nd(int d, const int* Ns, const double* x, double* y, int inverse);
void oracle_d_r2r_nd(int kind, int d, const int* Ns, const double* x, double* y);
void oracle_d_realdft_nd(int d, const int* Ns, const double* x, double* z);
void oracle_d_invrealdft_nd(int d, const int* Ns, const double* z, double* y);

/* r2r kind codes of the oracle */
enum { R_DCT2 = 2, R_DST2 = 3, R_DCT3 = 4, R_DST3 = 5, R_DCT4 = 6, R_DST4 = 7 };

struct minfft_aux {
    int d;
    int Ns[3];
};

static minfft_aux* mk(int d, int n1, int n2, int n3) {
    if (n1 <= 0 || (d > 1 && n2 <= 0) || (d > 2 && n3 <= 0)) return NULL;
    minfft_aux* a = (minfft_aux*)malloc(sizeof *a);
    if (!a) return NULL;
    a->d = d;
    a->Ns[0] = n1;
    a->Ns[1] = n2;
    a->Ns[2] = n3;
    return a;
}

minfft_aux* minfft_mkaux_dft_1d(int N) { return mk(1, N, 0, 0); }
minfft_aux* minfft_mkaux_dft_2d(int N1, int N2) { return mk(2, N1, N2, 0); }
minfft_aux* minfft_mkaux_dft_3d(int N1, int N2, int N3) { return mk(3, N1, N2, N3); }
minfft_aux* minfft_mkaux_realdft_1d(int N) { return mk(1, N, 0, 0); }
minfft_aux* minfft_mkaux_t2t3_1d(int N) { return mk(1, N, 0, 0); }
minfft_aux* minfft_mkaux_t2t3_2d(int N1, int N2) { return mk(2, N1, N2, 0); }
minfft_aux* minfft_mkaux_t2t3_3d(int N1, int N2, int N3) { return mk(3, N1, N2, N3); }
minfft_aux* minfft_mkaux_t4_1d(int N) { return mk(1, N, 0, 0); }
minfft_aux* minfft_mkaux_t4_2d(int N1, int N2) { return mk(2, N1, N2, 0); }
minfft_aux* minfft_mkaux_t4_3d(int N1, int N2, int N3) { return mk(3, N1, N2, N3); }

void minfft_free_aux(minfft_aux* a) { free(a); }

static void cx(minfft_cmpl* x, minfft_cmpl* y, const minfft_aux* a, int inverse) {
    if (!a) return;
    if (a->d == 1)
        oracle_d_dft(&x[0][0], &y[0][0], a->Ns[0], inverse);
    else
        oracle_d_dft_nd(a->d, a->Ns, &x[0][0], &y[0][0], inverse);
}

static void rr(int kind, minfft_real* x, minfft_real* y, const minfft_aux* a) {
    if (!a) return;
    if (a->d == 1)
        oracle_d_r2r(kind, x, y, a->Ns[0]);
    else
        oracle_d_r2r_nd(kind, a->d, a->Ns, x, y);
}

void minfft_dft(minfft_cmpl* x, minfft_cmpl* y, const minfft_aux* a) { cx(x, y, a, 0); }
void minfft_invdft(minfft_cmpl* x, minfft_cmpl* y, const minfft_aux* a) { cx(x, y, a, 1); }

void minfft_realdft(minfft_real* x, minfft_cmpl* z, const minfft_aux* a) {
    if (!a) return;
    if (a->d == 1)
        oracle_d_realdft(x, &z[0][0], a->Ns[0]);
    else
        oracle_d_realdft_nd(a->d, a->Ns, x, &z[0][0]);
}

void minfft_invrealdft(minfft_cmpl* z, minfft_real* y, const minfft_aux* a) {
    if (!a) return;
    if (a->d == 1)
        oracle_d_invrealdft(&z[0][0], y, a->Ns[0]);
    else
        oracle_d_invrealdft_nd(a->d, a->Ns, &z[0][0], y);
}

void minfft_dct2(minfft_real* x, minfft_real* y, const minfft_aux* a) { rr(R_DCT2, x, y, a); }
void minfft_dst2(minfft_real* x, minfft_real* y, const minfft_aux* a) { rr(R_DST2, x, y, a); }
void minfft_dct3(minfft_real* x, minfft_real* y, const minfft_aux* a) { rr(R_DCT3, x, y, a); }
void minfft_dst3(minfft_real* x, minfft_real* y, const minfft_aux* a) { rr(R_DST3, x, y, a); }
void minfft_dct4(minfft_real* x, minfft_real* y, const minfft_aux* a) { rr(R_DCT4, x, y, a); }
void minfft_dst4(minfft_real* x, minfft_real* y, const minfft_aux* a) { rr(R_DST4, x, y, a); }

/*
 * nfft_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A plain-C, CPU restatement of the Notorious-FFT transforms, used by the
 * tests, by __graft_entry__.smoke() and by the CPU-baseline leg of bench.py
 * as the checker.  It is never linked into, called from, or shipped with the
 * CUDA library: the product path has no CPU fallback.
 *
 * Every transform follows the reference's own decomposition (file:line below,
 * paths relative to the NotoriousLOB/Notorious-FFT project) but evaluates it in
 * long double with exactly-reduced twiddle angles, so the oracle is a few
 * orders of magnitude more accurate than either reference build.  Results are
 * rounded to the caller's precision (double, or float when built with
 * -DORACLE_SINGLE) only at the very end.
 *
 * Parity pin: tests/test_oracle_pin.py checks this file against outputs of the
 * reference itself (tests/golden/*.npz, produced from the reference compiled
 * from its own sources by oracle/Makefile), against the reference test
 * suite's known-answer O(N^2) DFT for non-power-of-two sizes, and against
 * numpy/scipy definitions.
 *
 * Conventions restated here (all unnormalized, FFTW layout):
 *   dft      y_k = sum x_n e^{-2 pi i k n / N}                  src/07_legacy.h:146-148
 *   invdft   y_k = sum x_n e^{+2 pi i k n / N}  (power of two)  src/07_legacy.h:150-152
 *            y_k = (1/N) sum x_n e^{+2 pi i k n / N}  (other N; the Bluestein
 *            branch conjugates, runs forward, conjugates, scales 1/N)
 *                                                               src/05_algorithms.h:315-333
 *   realdft  N reals -> N/2+1 complex, Im of bins 0 and N/2 set to 0
 *                                                               src/07_legacy.h:162-237
 *   invrealdft  N/2+1 complex -> N reals, Im z_0 / Im z_{N/2} ignored
 *                                                               src/07_legacy.h:239-293
 *   dct2/dst2/dct3/dst3/dct4/dst4 = FFTW REDFT10/RODFT10/REDFT01/RODFT01/
 *            REDFT11/RODFT11                                    src/07_legacy.h:757-1387
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#ifdef ORACLE_SINGLE
typedef float R;
#define ORACLE_SYM(name) oracle_f_##name
#else
typedef double R;
#define ORACLE_SYM(name) oracle_d_##name
#endif

typedef long double L;
typedef struct { L re, im; } C;

static const L PI_L = 3.141592653589793238462643383279502884L;
static const L SQRT2_L = 1.414213562373095048801688724209698079L;

static int is_pow2(long n) { return n > 0 && (n & (n - 1)) == 0; }

/* e^{-2 pi i q / n} with q reduced exactly modulo n before the angle is formed */
static C cis_neg(long long q, long long n) {
    q %= n;
    if (q < 0) q += n;
    L a = -2.0L * PI_L * (L)q / (L)n;
    C w = { cosl(a), sinl(a) };
    return w;
}

static C cmul(C a, C b) { C r = { a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re }; return r; }
static C cconj(C a) { a.im = -a.im; return a; }

/* In-place iterative radix-2 DIT FFT, forward sign, power-of-two n.
 * Restates src/05_algorithms.h:28-117 (bit-reversal, then log2 n butterfly
 * stages with twiddles e^{-2 pi i j/len}), in long double. */
static void fft_pow2(C* a, long n) {
    if (n <= 1) return;
    for (long i = 1, j = 0; i < n; i++) {
        long bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { C t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    C* w = (C*)malloc(sizeof(C) * (size_t)(n / 2));
    for (long i = 0; i < n / 2; i++) w[i] = cis_neg(i, n);
    for (long len = 2; len <= n; len <<= 1) {
        long half = len >> 1, step = n / len;
        for (long i = 0; i < n; i += len)
            for (long j = 0; j < half; j++) {
                C u = a[i + j], v = cmul(a[i + j + half], w[j * step]);
                a[i + j].re = u.re + v.re; a[i + j].im = u.im + v.im;
                a[i + j + half].re = u.re - v.re; a[i + j + half].im = u.im - v.im;
            }
    }
    free(w);
}

/* Forward DFT of arbitrary length n (long double).  Power-of-two n uses
 * fft_pow2; other n use Bluestein's chirp-z identity as the reference does
 * (src/05_algorithms.h:742-896, plan src/06_plan.h:28-121): premultiply by
 * the chirp e^{-i pi k^2/n}, convolve with e^{+i pi m^2/n} through an M-point
 * FFT (M = next power of two >= 2n-1), postmultiply by the chirp.  The chirp
 * phase is formed from k^2 mod 2n in exact integer arithmetic. */
static void dft_fwd(C* a, long n) {
    if (n <= 1) return;
    if (is_pow2(n)) { fft_pow2(a, n); return; }
    long m = 1;
    while (m < 2 * n - 1) m <<= 1;
    C* chirp = (C*)malloc(sizeof(C) * (size_t)n);
    C* u = (C*)calloc((size_t)m, sizeof(C));
    C* v = (C*)calloc((size_t)m, sizeof(C));
    for (long k = 0; k < n; k++) {
        unsigned long long r = ((unsigned long long)k * (unsigned long long)k) % (unsigned long long)(2 * n);
        chirp[k] = cis_neg((long long)r, 2 * n);          /* e^{-i pi k^2 / n} */
    }
    for (long k = 0; k < n; k++) u[k] = cmul(a[k], chirp[k]);
    v[0] = cconj(chirp[0]);
    for (long k = 1; k < n; k++) { v[k] = cconj(chirp[k]); v[m - k] = cconj(chirp[k]); }
    fft_pow2(u, m);
    fft_pow2(v, m);
    for (long i = 0; i < m; i++) u[i] = cconj(cmul(u[i], v[i]));   /* inverse via conj */
    fft_pow2(u, m);
    for (long k = 0; k < n; k++) {
        C c = cconj(u[k]);
        c.re /= (L)m; c.im /= (L)m;
        a[k] = cmul(c, chirp[k]);
    }
    free(chirp); free(u); free(v);
}

/* Complex DFT with the reference's direction/normalization semantics
 * (src/07_legacy.h:146-152, src/05_algorithms.h:292-344). */
static void dft_ld(C* a, long n, int inverse) {
    if (!inverse) { dft_fwd(a, n); return; }
    for (long i = 0; i < n; i++) a[i].im = -a[i].im;
    dft_fwd(a, n);
    for (long i = 0; i < n; i++) a[i].im = -a[i].im;
    if (!is_pow2(n)) {                       /* Bluestein inverse scales by 1/N */
        for (long i = 0; i < n; i++) { a[i].re /= (L)n; a[i].im /= (L)n; }
    }
}

/* realdft: N reals -> N/2+1 complex (src/07_legacy.h:162-237).  N=1 and N=2
 * are the reference's special cases (:164-177); otherwise pack as N/2 complex,
 * FFT, and unpack with t_k = e^{-2 pi i k / N}. */
static void realdft_ld(const L* x, C* z, long N) {
    if (N == 1) { z[0].re = x[0]; z[0].im = 0; return; }
    if (N == 2) { z[0].re = x[0] + x[1]; z[0].im = 0; z[1].re = x[0] - x[1]; z[1].im = 0; return; }
    long M = N / 2;
    C* t = (C*)malloc(sizeof(C) * (size_t)M);
    for (long n = 0; n < M; n++) { t[n].re = x[2 * n]; t[n].im = x[2 * n + 1]; }
    fft_pow2(t, M);
    z[0].re = t[0].re + t[0].im; z[0].im = 0;
    z[M].re = t[0].re - t[0].im; z[M].im = 0;
    for (long k = 1; k < M; k++) {
        C a = t[k], b = cconj(t[M - k]);
        C s = { (a.re + b.re) * 0.5L, (a.im + b.im) * 0.5L };      /* even part */
        C d = { (a.re - b.re) * 0.5L, (a.im - b.im) * 0.5L };      /* odd part * e^{...} */
        C w = cis_neg(k, N);
        C od = cmul(d, w);                                       /* times -i below */
        z[k].re = s.re + od.im;
        z[k].im = s.im - od.re;
    }
    free(t);
}

/* invrealdft: N/2+1 complex -> N reals, unnormalized (src/07_legacy.h:239-293).
 * Only Re z_0 and Re z_{N/2} are read (:263-264). */
static void invrealdft_ld(const C* z, L* y, long N) {
    if (N == 1) { y[0] = z[0].re; return; }
    if (N == 2) { y[0] = z[0].re + z[1].re; y[1] = z[0].re - z[1].re; return; }
    long M = N / 2;
    C* t = (C*)malloc(sizeof(C) * (size_t)M);
    t[0].re = z[0].re + z[M].re;
    t[0].im = z[0].re - z[M].re;
    for (long k = 1; k < M; k++) {
        C a = z[k], b = cconj(z[M - k]);
        C s = { a.re + b.re, a.im + b.im };
        C d = { a.re - b.re, a.im - b.im };
        C w = cconj(cis_neg(k, N));                              /* e^{+2 pi i k / N} */
        C od = cmul(d, w);                                       /* times +i below */
        t[k].re = s.re - od.im;
        t[k].im = s.im + od.re;
    }
    for (long i = 0; i < M; i++) t[i].im = -t[i].im;              /* inverse via conj */
    fft_pow2(t, M);
    for (long n = 0; n < M; n++) { y[2 * n] = t[n].re; y[2 * n + 1] = -t[n].im; }
    free(t);
}

/* DCT-2 / DST-2 (REDFT10 / RODFT10): reorder even / reversed-odd (DST negates
 * the odd half), realdft, post-twiddle e^{-i pi k / 2N}, x2, sqrt2 at k = N/2.
 * src/07_legacy.h:757-797 (dct2), :870-898 (dst2); N=1,2 special cases :759-767. */
static void t2_ld(const L* x, L* y, long N, int dst) {
    if (N == 1) { y[0] = 2 * x[0]; return; }
    if (N == 2) {
        if (!dst) { y[0] = 2 * (x[0] + x[1]); y[1] = SQRT2_L * (x[0] - x[1]); }
        else      { y[0] = SQRT2_L * (x[0] + x[1]); y[1] = 2 * (x[0] - x[1]); }
        return;
    }
    L* v = (L*)malloc(sizeof(L) * (size_t)N);
    C* z = (C*)malloc(sizeof(C) * (size_t)(N / 2 + 1));
    for (long i = 0; i < N / 2; i++) {
        v[i] = x[2 * i];
        v[N / 2 + i] = dst ? -x[N - 1 - 2 * i] : x[N - 1 - 2 * i];
    }
    realdft_ld(v, z, N);
    if (!dst) {
        y[0] = 2 * z[0].re;
        for (long k = 1; k < N / 2; k++) {
            C w = cis_neg(k, 4 * N);                             /* e^{-i pi k / 2N} */
            y[k] = 2 * (z[k].re * w.re - z[k].im * w.im);
            y[N - k] = -2 * (z[k].re * w.im + z[k].im * w.re);
        }
        y[N / 2] = SQRT2_L * z[N / 2].re;
    } else {
        y[N - 1] = 2 * z[0].re;
        for (long k = 1; k < N / 2; k++) {
            C w = cis_neg(k, 4 * N);
            y[k - 1] = -2 * (z[k].re * w.im + z[k].im * w.re);
            y[N - k - 1] = 2 * (z[k].re * w.re - z[k].im * w.im);
        }
        y[N / 2 - 1] = SQRT2_L * z[N / 2].re;
    }
    free(v); free(z);
}

/* DCT-3 / DST-3 (REDFT01 / RODFT01): pre-twiddle, invrealdft, un-reorder
 * (DST-3 reads x reversed and negates the odd half).
 * src/07_legacy.h:956-982 (dct3), :1012-1038 (dst3); N=1,2 at :958-962,1014-1018. */
static void t3_ld(const L* x, L* y, long N, int dst) {
    if (N == 1) { y[0] = x[0]; return; }
    if (N == 2) {
        if (!dst) { L s = SQRT2_L * x[1]; y[0] = x[0] + s; y[1] = x[0] - s; }
        else      { L s = SQRT2_L * x[0]; y[0] = s + x[1]; y[1] = s - x[1]; }
        return;
    }
    C* z = (C*)malloc(sizeof(C) * (size_t)(N / 2 + 1));
    L* t = (L*)malloc(sizeof(L) * (size_t)N);
    z[0].re = dst ? x[N - 1] : x[0]; z[0].im = 0;
    for (long k = 1; k < N / 2; k++) {
        C w = cis_neg(k, 4 * N);
        L xr = dst ? x[N - k - 1] : x[k];
        L xi = dst ? x[k - 1] : x[N - k];
        z[k].re = xr * w.re - xi * w.im;
        z[k].im = -xr * w.im - xi * w.re;
    }
    z[N / 2].re = SQRT2_L * (dst ? x[N / 2 - 1] : x[N / 2]); z[N / 2].im = 0;
    invrealdft_ld(z, t, N);
    for (long i = 0; i < N / 2; i++) {
        y[2 * i] = t[i];
        y[N - 1 - 2 * i] = dst ? -t[N / 2 + i] : t[N / 2 + i];
    }
    free(z); free(t);
}

/* DCT-4 / DST-4 (REDFT11 / RODFT11): premultiply (x[2n] +/- i x[N-1-2n]) by
 * e^{-i pi n / N}, N/2-point forward DFT, postmultiply by e^{-i pi (2k+1)/4N}
 * and take 2 Re (DCT) or 2 Im (DST).  src/07_legacy.h:1091-1137 (body),
 * :536-549 (pre/post formulas), :1298-1303 (N=1 -> sqrt2 x). */
static void t4_ld(const L* x, L* y, long N, int dst) {
    if (N == 1) { y[0] = SQRT2_L * x[0]; return; }
    long M = N / 2;
    C* t = (C*)malloc(sizeof(C) * (size_t)M);
    for (long n = 0; n < M; n++) {
        C e = cis_neg(n, 2 * N);                                 /* e^{-i pi n / N} */
        L xe = x[2 * n], xo = x[N - 1 - 2 * n];
        if (!dst) { t[n].re = e.re * xe - e.im * xo; t[n].im = e.re * xo + e.im * xe; }
        else      { t[n].re = -e.re * xe - e.im * xo; t[n].im = e.re * xo - e.im * xe; }
    }
    fft_pow2(t, M);
    for (long k = 0; k < M; k++) {
        C f0 = cis_neg(2 * (2 * k) + 1, 8 * N);                  /* e^{-i pi (2(2k)+1) / 4N} */
        C f1 = cis_neg(2 * (2 * k + 1) + 1, 8 * N);
        C a = t[k];
        C b = { t[M - 1 - k].re, -t[M - 1 - k].im };
        if (!dst) {
            y[2 * k] = 2 * (f0.re * a.re - f0.im * a.im);
            y[2 * k + 1] = 2 * (f1.re * b.re - f1.im * b.im);
        } else {
            y[2 * k] = 2 * (f0.re * a.im + f0.im * a.re);
            y[2 * k + 1] = 2 * (f1.re * b.im + f1.im * b.re);
        }
    }
    free(t);
}

/* ------------------------------------------------------------------------- */
/* Exported 1-D entry points (double or float I/O, long double inside).      */
/* ------------------------------------------------------------------------- */

void ORACLE_SYM(dft)(const R* x, R* y, long N, int inverse) {
    C* a = (C*)malloc(sizeof(C) * (size_t)N);
    for (long i = 0; i < N; i++) { a[i].re = x[2 * i]; a[i].im = x[2 * i + 1]; }
    dft_ld(a, N, inverse);
    for (long i = 0; i < N; i++) { y[2 * i] = (R)a[i].re; y[2 * i + 1] = (R)a[i].im; }
    free(a);
}

void ORACLE_SYM(realdft)(const R* x, R* z, long N) {
    L* xl = (L*)malloc(sizeof(L) * (size_t)N);
    C* zl = (C*)malloc(sizeof(C) * (size_t)(N / 2 + 1));
    for (long i = 0; i < N; i++) xl[i] = x[i];
    realdft_ld(xl, zl, N);
    for (long k = 0; k <= N / 2; k++) { z[2 * k] = (R)zl[k].re; z[2 * k + 1] = (R)zl[k].im; }
    free(xl); free(zl);
}

void ORACLE_SYM(invrealdft)(const R* z, R* y, long N) {
    C* zl = (C*)malloc(sizeof(C) * (size_t)(N / 2 + 1));
    L* yl = (L*)malloc(sizeof(L) * (size_t)N);
    for (long k = 0; k <= N / 2; k++) { zl[k].re = z[2 * k]; zl[k].im = z[2 * k + 1]; }
    invrealdft_ld(zl, yl, N);
    for (long i = 0; i < N; i++) y[i] = (R)yl[i];
    free(zl); free(yl);
}

/* kind: 2 = dct2, 3 = dst2, 4 = dct3, 5 = dst3, 6 = dct4, 7 = dst4 */
static void r2r_ld(int kind, const L* x, L* y, long N) {
    switch (kind) {
    case 2: t2_ld(x, y, N, 0); break;
    case 3: t2_ld(x, y, N, 1); break;
    case 4: t3_ld(x, y, N, 0); break;
    case 5: t3_ld(x, y, N, 1); break;
    case 6: t4_ld(x, y, N, 0); break;
    case 7: t4_ld(x, y, N, 1); break;
    }
}

void ORACLE_SYM(r2r)(int kind, const R* x, R* y, long N) {
    L* xl = (L*)malloc(sizeof(L) * (size_t)N);
    L* yl = (L*)malloc(sizeof(L) * (size_t)N);
    for (long i = 0; i < N; i++) xl[i] = x[i];
    r2r_ld(kind, xl, yl, N);
    for (long i = 0; i < N; i++) y[i] = (R)yl[i];
    free(xl); free(yl);
}

/* ------------------------------------------------------------------------- */
/* N-D transforms, row-major, Ns[0] slowest (src/07_legacy.h:1654-1688).      */
/* ------------------------------------------------------------------------- */

/* Complex N-D DFT: the reference's mkcx recursion (src/07_legacy.h:109-140)
 * transforms every axis with the 1-D semantics above (including the 1/n
 * factor of a non-power-of-two inverse axis).  Restated as one pass per axis. */
void ORACLE_SYM(dft_nd)(int d, const int* Ns, const R* x, R* y, int inverse) {
    long total = 1;
    for (int i = 0; i < d; i++) total *= Ns[i];
    C* a = (C*)malloc(sizeof(C) * (size_t)total);
    for (long i = 0; i < total; i++) { a[i].re = x[2 * i]; a[i].im = x[2 * i + 1]; }
    long inner = total;
    for (int ax = 0; ax < d; ax++) {
        long n = Ns[ax];
        inner /= n;
        long outer = total / (n * inner);
        C* line = (C*)malloc(sizeof(C) * (size_t)n);
        for (long o = 0; o < outer; o++)
            for (long i = 0; i < inner; i++) {
                C* base = a + o * n * inner + i;
                for (long k = 0; k < n; k++) line[k] = base[k * inner];
                dft_ld(line, n, inverse);
                for (long k = 0; k < n; k++) base[k * inner] = line[k];
            }
        free(line);
    }
    for (long i = 0; i < total; i++) { y[2 * i] = (R)a[i].re; y[2 * i + 1] = (R)a[i].im; }
    free(a);
}

/* Real-to-real N-D (t2t3 / t4 auxes).  The reference's recursion
 * (src/07_legacy.h:822-861, :927-946, :987-1006, :1043-1062, :1339-1386)
 * transforms axis k only while the product of the axes after k exceeds 1
 * ("if (N1 == 1) { transform(x, y, a->sub2); return; }"), so trailing
 * length-1 axes behind the first axis are skipped (they would otherwise
 * scale by 2 or sqrt2).  The t4 branch also short-circuits a total size of 1
 * to the 1-D N=1 case (:1300-1303, :1337).  Both quirks are reproduced. */
void ORACLE_SYM(r2r_nd)(int kind, int d, const int* Ns, const R* x, R* y) {
    long total = 1;
    for (int i = 0; i < d; i++) total *= Ns[i];
    L* a = (L*)malloc(sizeof(L) * (size_t)total);
    for (long i = 0; i < total; i++) a[i] = x[i];
    int last = 0;                                   /* last axis that is transformed */
    for (int i = 0; i < d; i++) if (Ns[i] != 1) last = i;
    long inner = total;
    for (int ax = 0; ax < d; ax++) {
        long n = Ns[ax];
        inner /= n;
        if (ax > last) break;
        long outer = total / (n * inner);
        L* line = (L*)malloc(sizeof(L) * (size_t)n);
        L* out = (L*)malloc(sizeof(L) * (size_t)n);
        for (long o = 0; o < outer; o++)
            for (long i = 0; i < inner; i++) {
                L* base = a + o * n * inner + i;
                for (long k = 0; k < n; k++) line[k] = base[k * inner];
                r2r_ld(kind, line, out, n);
                for (long k = 0; k < n; k++) base[k * inner] = out[k];
            }
        free(line); free(out);
    }
    for (long i = 0; i < total; i++) y[i] = (R)a[i];
    free(a);
}

/* Multi-D realdft in FFTW layout (last axis -> Ns[d-1]/2+1 bins, then complex
 * DFTs along the other axes).  The reference declares mkaux_realdft_{2d,3d}
 * (src/07_legacy.h:1492-1524) but its execution path dereferences a NULL
 * scratch pointer, so this restates the documented layout (README.md:58-98)
 * and the FFTW convention it names. */
void ORACLE_SYM(realdft_nd)(int d, const int* Ns, const R* x, R* z) {
    long outer = 1;
    for (int i = 0; i < d - 1; i++) outer *= Ns[i];
    long n = Ns[d - 1], h = n / 2 + 1;
    C* a = (C*)malloc(sizeof(C) * (size_t)(outer * h));
    L* xl = (L*)malloc(sizeof(L) * (size_t)n);
    for (long o = 0; o < outer; o++) {
        for (long i = 0; i < n; i++) xl[i] = x[o * n + i];
        realdft_ld(xl, a + o * h, n);
    }
    long inner = outer * h;
    for (int ax = 0; ax < d - 1; ax++) {
        long m = Ns[ax];
        inner /= m;
        long oo = outer * h / (m * inner);
        C* line = (C*)malloc(sizeof(C) * (size_t)m);
        for (long o = 0; o < oo; o++)
            for (long i = 0; i < inner; i++) {
                C* base = a + o * m * inner + i;
                for (long k = 0; k < m; k++) line[k] = base[k * inner];
                dft_ld(line, m, 0);
                for (long k = 0; k < m; k++) base[k * inner] = line[k];
            }
        free(line);
    }
    for (long i = 0; i < outer * h; i++) { z[2 * i] = (R)a[i].re; z[2 * i + 1] = (R)a[i].im; }
    free(a); free(xl);
}

/* Inverse of realdft_nd (unnormalized): complex inverse DFTs along the leading
 * axes, then invrealdft along the last axis. */
void ORACLE_SYM(invrealdft_nd)(int d, const int* Ns, const R* z, R* y) {
    long outer = 1;
    for (int i = 0; i < d - 1; i++) outer *= Ns[i];
    long n = Ns[d - 1], h = n / 2 + 1;
    C* a = (C*)malloc(sizeof(C) * (size_t)(outer * h));
    for (long i = 0; i < outer * h; i++) { a[i].re = z[2 * i]; a[i].im = z[2 * i + 1]; }
    long inner = outer * h;
    for (int ax = 0; ax < d - 1; ax++) {
        long m = Ns[ax];
        inner /= m;
        long oo = outer * h / (m * inner);
        C* line = (C*)malloc(sizeof(C) * (size_t)m);
        for (long o = 0; o < oo; o++)
            for (long i = 0; i < inner; i++) {
                C* base = a + o * m * inner + i;
                for (long k = 0; k < m; k++) line[k] = base[k * inner];
                dft_ld(line, m, 1);
                for (long k = 0; k < m; k++) base[k * inner] = line[k];
            }
        free(line);
    }
    L* yl = (L*)malloc(sizeof(L) * (size_t)n);
    for (long o = 0; o < outer; o++) {
        invrealdft_ld(a + o * h, yl, n);
        for (long i = 0; i < n; i++) y[o * n + i] = (R)yl[i];
    }
    free(a); free(yl);
}

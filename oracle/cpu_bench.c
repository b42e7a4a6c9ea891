/*
 * cpu_bench.c -- TEST/BENCH INFRASTRUCTURE ONLY.
 *
 * Times a CPU implementation of the Notorious-FFT C API on the host cores:
 * the reference compiled from its own sources (oracle/_ref/libref_*.so).  The
 * library is dlopen()ed with RTLD_LOCAL so its symbols never meet the CUDA
 * library's identically named ones.
 *
 * Batched 1-D transforms run an OpenMP parallel-for over the batch with one
 * aux per thread, because an aux holds mutable scratch and is not
 * thread-safe (src/07_legacy.h:133 of the reference).  N-D transforms run as
 * one call, as the reference runs them (its N-D path has no parallelism).
 *
 *   cpu_bench <lib.so> <f64|f32> <kind> <N|N1xN2[xN3]> <batch> <threads> <reps>
 *   kind: dft invdft realdft invrealdft dct2 dst2 dct3 dst3 dct4 dst4
 *
 * Prints one JSON object: best-of-reps seconds for the whole batch.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef void* (*mk1_t)(int);
typedef void* (*mknd_t)(int, int*);
typedef void (*tr_t)(void*, void*, const void*);
typedef void (*free_t)(void*);

static uint64_t rng_state = 0x9E3779B97F4A7C15ull;
static double urand(void) {            /* splitmix64 -> uniform [-1, 1) */
    uint64_t z = (rng_state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

int main(int argc, char** argv) {
    if (argc < 8) {
        fprintf(stderr, "usage: %s lib.so f64|f32 kind dims batch threads reps\n", argv[0]);
        return 2;
    }
    const char* lib = argv[1];
    int f32 = strcmp(argv[2], "f32") == 0;
    const char* kind = argv[3];
    int dims[3] = {0, 0, 0}, d = 0;
    {
        char* s = strdup(argv[4]);
        for (char* tok = strtok(s, "x"); tok && d < 3; tok = strtok(NULL, "x")) dims[d++] = atoi(tok);
        free(s);
    }
    long batch = atol(argv[5]);
    int threads = atoi(argv[6]);
    int reps = atoi(argv[7]);
    void* h = dlopen(lib, RTLD_NOW | RTLD_LOCAL);
    if (!h) { fprintf(stderr, "dlopen: %s\n", dlerror()); return 1; }
    size_t rs = f32 ? sizeof(float) : sizeof(double);

    const char* mkname;
    int cin = 0, cout = 0, realout_half = 0, realin_half = 0;
    if (!strcmp(kind, "dft") || !strcmp(kind, "invdft")) { mkname = "notorious_fft_mkaux_dft"; cin = cout = 1; }
    else if (!strcmp(kind, "realdft")) { mkname = "notorious_fft_mkaux_realdft"; cout = 1; realout_half = 1; }
    else if (!strcmp(kind, "invrealdft")) { mkname = "notorious_fft_mkaux_realdft"; cin = 1; realin_half = 1; }
    else if (!strcmp(kind, "dct4") || !strcmp(kind, "dst4")) mkname = "notorious_fft_mkaux_t4";
    else mkname = "notorious_fft_mkaux_t2t3";
    char trname[64];
    snprintf(trname, sizeof trname, "notorious_fft_%s", kind);
    mknd_t mk = (mknd_t)dlsym(h, mkname);
    tr_t tr = (tr_t)dlsym(h, trname);
    free_t fr = (free_t)dlsym(h, "notorious_fft_free_aux");
    if (!mk || !tr || !fr) { fprintf(stderr, "dlsym failed\n"); return 1; }

    long total = 1;
    for (int i = 0; i < d; i++) total *= dims[i];
    long last = dims[d - 1];
    long half = total / last * (last / 2 + 1);
    long nin = cin ? 2 * (realin_half ? half : total) : total;
    long nout = cout ? 2 * (realout_half ? half : total) : total;
    char* x = (char*)malloc((size_t)(nin * batch) * rs);
    char* y = (char*)malloc((size_t)(nout * batch) * rs);
    for (long i = 0; i < nin * batch; i++) {
        double v = urand();
        if (f32) ((float*)x)[i] = (float)v; else ((double*)x)[i] = v;
    }
    if (threads < 1) threads = 1;
    double best = 1e30;
    int nd = d > 1;
    for (int rep = 0; rep < reps; rep++) {
        double t0 = 0, t1 = 0;
        if (nd) {
            void* a = mk(d, dims);
            if (!a) { fprintf(stderr, "mkaux failed\n"); return 1; }
            t0 = omp_get_wtime();
            for (long b = 0; b < batch; b++) tr(x + b * nin * rs, y + b * nout * rs, a);
            t1 = omp_get_wtime();
            fr(a);
        } else {
            #pragma omp parallel num_threads(threads)
            {
                void* a = mk(1, dims);
                #pragma omp barrier
                #pragma omp single
                t0 = omp_get_wtime();
                #pragma omp for schedule(static)
                for (long b = 0; b < batch; b++) tr(x + b * nin * rs, y + b * nout * rs, a);
                #pragma omp single
                t1 = omp_get_wtime();
                fr(a);
            }
        }
        if (t1 - t0 < best) best = t1 - t0;
    }
    double bytes = (double)batch * (double)(nin + nout) * (double)rs;
    printf("{\"kind\": \"%s\", \"dims\": \"%s\", \"batch\": %ld, \"threads\": %d, \"seconds\": %.6e, "
           "\"transforms_per_s\": %.6e, \"gbs\": %.6e}\n",
           kind, argv[4], batch, nd ? 1 : threads, best, (double)batch / best, bytes / best / 1e9);
    dlclose(h);
    return 0;
}

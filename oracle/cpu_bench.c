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
 * one call per array, as the reference runs them (its N-D path has no
 * parallelism).
 *
 *   cpu_bench <lib.so> <f64|f32> <kinds> <N|N1xN2[xN3]> <batch> <threads> <reps>
 *       kinds: one of dft invdft realdft invrealdft dct2 dst2 dct3 dst3 dct4
 *       dst4, or a comma-separated chain of length-preserving kinds (e.g.
 *       "dft,invdft"): the first runs x -> y, the others in place on y, one
 *       parallel loop per kind.  One rep = the whole chain over the batch.
 *
 *   cpu_bench <lib.so> <f64|f32> ragged <list file> - <threads> <reps>
 *       A ragged batch: the list file holds one "kind N" pair per line
 *       (dft, invdft, realdft or dct2; any N the reference accepts).
 *       Transforms of equal (kind, N) form a group; threads take groups in
 *       turn, build one aux per group (the reference's benchmarks keep one
 *       plan per size, benchmarks/bench_mixed_sizes.c), run the group's
 *       transforms and free it.  Reported: the wall time of the whole loop,
 *       and the execution time without plan building (per thread, summed over
 *       its groups; the maximum over threads).
 *
 * Prints one JSON object: best-of-reps seconds, and every rep's seconds.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

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

static void fill(char* x, long n, int f32) {
    for (long i = 0; i < n; i++) {
        double v = urand();
        if (f32) ((float*)x)[i] = (float)v; else ((double*)x)[i] = v;
    }
}

static const char* family_of(const char* kind) {
    if (!strcmp(kind, "dft") || !strcmp(kind, "invdft")) return "notorious_fft_mkaux_dft";
    if (!strcmp(kind, "realdft") || !strcmp(kind, "invrealdft")) return "notorious_fft_mkaux_realdft";
    if (!strcmp(kind, "dct4") || !strcmp(kind, "dst4")) return "notorious_fft_mkaux_t4";
    return "notorious_fft_mkaux_t2t3";
}

static void* sym(void* h, const char* name) {
    void* p = dlsym(h, name);
    if (!p) { fprintf(stderr, "dlsym %s failed\n", name); exit(1); }
    return p;
}

static void print_reps(const double* t, int reps) {
    printf("\"rep_seconds\": [");
    for (int r = 0; r < reps; r++) printf("%s%.6e", r ? ", " : "", t[r]);
    printf("]");
}

/* ---- ragged batch ------------------------------------------------------- */
typedef struct { int kind; int n; long in_off, out_off; } Item;
static const char* RAGGED_KINDS[4] = {"dft", "invdft", "realdft", "dct2"};

static int cmp_item(const void* a, const void* b) {
    const Item *x = (const Item*)a, *y = (const Item*)b;
    if (x->kind != y->kind) return x->kind - y->kind;
    return x->n - y->n;
}

static int run_ragged(void* h, int f32, const char* path, int threads, int reps) {
    FILE* f = fopen(path, "r");
    if (!f) { fprintf(stderr, "cannot open %s\n", path); return 1; }
    long cap = 1024, cnt = 0;
    Item* it = (Item*)malloc(sizeof(Item) * cap);
    char kname[32];
    int n;
    while (fscanf(f, "%31s %d", kname, &n) == 2) {
        int k = -1;
        for (int i = 0; i < 4; i++) if (!strcmp(kname, RAGGED_KINDS[i])) k = i;
        if (k < 0 || n < 1) { fprintf(stderr, "bad item %s %d\n", kname, n); return 1; }
        if (cnt == cap) { cap *= 2; it = (Item*)realloc(it, sizeof(Item) * cap); }
        it[cnt].kind = k;
        it[cnt].n = n;
        cnt++;
    }
    fclose(f);
    size_t rs = f32 ? sizeof(float) : sizeof(double);
    long in_tot = 0, out_tot = 0;
    for (long i = 0; i < cnt; i++) {           /* packed layout, even offsets */
        long ci = it[i].kind <= 1 ? 2L * it[i].n : it[i].n;
        long co = it[i].kind <= 1 ? 2L * it[i].n : (it[i].kind == 2 ? 2L * (it[i].n / 2 + 1) : it[i].n);
        it[i].in_off = in_tot;
        it[i].out_off = out_tot;
        in_tot += ci + (ci & 1);
        out_tot += co + (co & 1);
    }
    qsort(it, (size_t)cnt, sizeof(Item), cmp_item);
    long ng = 0;
    long* gstart = (long*)malloc(sizeof(long) * (cnt + 1));
    for (long i = 0; i < cnt; i++)
        if (i == 0 || cmp_item(&it[i], &it[i - 1])) gstart[ng++] = i;
    gstart[ng] = cnt;
    char* x = (char*)malloc((size_t)in_tot * rs);
    char* y = (char*)malloc((size_t)out_tot * rs);
    fill(x, in_tot, f32);
    mknd_t mk[4];
    tr_t tr[4];
    for (int k = 0; k < 4; k++) {
        char name[64];
        mk[k] = (mknd_t)sym(h, family_of(RAGGED_KINDS[k]));
        snprintf(name, sizeof name, "notorious_fft_%s", RAGGED_KINDS[k]);
        tr[k] = (tr_t)sym(h, name);
    }
    free_t fr = (free_t)sym(h, "notorious_fft_free_aux");
    double* wall = (double*)malloc(sizeof(double) * reps);
    double* exec = (double*)malloc(sizeof(double) * reps);
    double best_wall = 1e30, best_exec = 1e30;
    long skipped = 0, done = 0;
    double done_bytes = 0;
    for (int rep = 0; rep < reps; rep++) {
        double t_exec_max = 0;
        double t0 = omp_get_wtime();
        skipped = done = 0;
        done_bytes = 0;
        #pragma omp parallel num_threads(threads) reduction(max: t_exec_max) reduction(+: skipped, done, done_bytes)
        {
            double mine = 0;
            #pragma omp for schedule(dynamic, 1)
            for (long g = 0; g < ng; g++) {
                const Item* a0 = &it[gstart[g]];
                int nn = a0->n;
                void* aux = mk[a0->kind](1, &nn);
                if (!aux) { skipped += gstart[g + 1] - gstart[g]; continue; }
                double e0 = omp_get_wtime();
                for (long i = gstart[g]; i < gstart[g + 1]; i++)
                    tr[it[i].kind](x + (size_t)it[i].in_off * rs, y + (size_t)it[i].out_off * rs, aux);
                mine += omp_get_wtime() - e0;
                {
                    long ci = a0->kind <= 1 ? 2L * nn : nn;
                    long co = a0->kind <= 1 ? 2L * nn : (a0->kind == 2 ? 2L * (nn / 2 + 1) : nn);
                    done += gstart[g + 1] - gstart[g];
                    done_bytes += (double)(gstart[g + 1] - gstart[g]) * (double)(ci + co) * (double)rs;
                }
                fr(aux);
            }
            t_exec_max = mine;
        }
        wall[rep] = omp_get_wtime() - t0;
        exec[rep] = t_exec_max;
        if (wall[rep] < best_wall) best_wall = wall[rep];
        if (exec[rep] < best_exec) best_exec = exec[rep];
    }
    /* transforms the reference has no plan for (mkaux returned NULL) are not
       run and not counted */
    printf("{\"kind\": \"ragged\", \"transforms\": %ld, \"groups\": %ld, \"threads\": %d, "
           "\"executed\": %ld, \"skipped_no_plan\": %ld, \"seconds\": %.6e, \"seconds_with_plans\": %.6e, "
           "\"transforms_per_s\": %.6e, \"gbs\": %.6e, ",
           cnt, ng, threads, done, skipped, best_exec, best_wall, (double)done / best_exec,
           done_bytes / best_exec / 1e9);
    print_reps(exec, reps);
    printf("}\n");
    return 0;
}

/* ---- batched / N-D ------------------------------------------------------ */
int main(int argc, char** argv) {
    if (argc < 8) {
        fprintf(stderr, "usage: %s lib.so f64|f32 kinds dims batch threads reps\n"
                        "       %s lib.so f64|f32 ragged listfile - threads reps\n", argv[0], argv[0]);
        return 2;
    }
    const char* lib = argv[1];
    int f32 = strcmp(argv[2], "f32") == 0;
    int threads = atoi(argv[6]);
    int reps = atoi(argv[7]);
    if (threads < 1) threads = 1;
    if (reps < 1) reps = 1;
    void* h = dlopen(lib, RTLD_NOW | RTLD_LOCAL);
    if (!h) { fprintf(stderr, "dlopen: %s\n", dlerror()); return 1; }
    if (!strcmp(argv[3], "ragged")) return run_ragged(h, f32, argv[4], threads, reps);

    /* the chain of kinds */
    char* kinds_s = strdup(argv[3]);
    const char* kinds[8];
    int nk = 0;
    for (char* tok = strtok(kinds_s, ","); tok && nk < 8; tok = strtok(NULL, ",")) kinds[nk++] = tok;
    int dims[3] = {0, 0, 0}, d = 0;
    {
        char* s = strdup(argv[4]);
        for (char* tok = strtok(s, "x"); tok && d < 3; tok = strtok(NULL, "x")) dims[d++] = atoi(tok);
        free(s);
    }
    long batch = atol(argv[5]);
    size_t rs = f32 ? sizeof(float) : sizeof(double);

    const char* kind = kinds[0];
    const char* mkname = family_of(kind);
    int cin = 0, cout = 0, realout_half = 0, realin_half = 0;
    if (!strcmp(kind, "dft") || !strcmp(kind, "invdft")) cin = cout = 1;
    else if (!strcmp(kind, "realdft")) { cout = 1; realout_half = 1; }
    else if (!strcmp(kind, "invrealdft")) { cin = 1; realin_half = 1; }
    for (int i = 1; i < nk; i++)
        if (strcmp(family_of(kinds[i]), mkname) || realout_half || realin_half) {
            fprintf(stderr, "a chain needs length-preserving kinds of one family\n");
            return 2;
        }
    mknd_t mk = (mknd_t)sym(h, mkname);
    tr_t tr[8];
    for (int i = 0; i < nk; i++) {
        char trname[64];
        snprintf(trname, sizeof trname, "notorious_fft_%s", kinds[i]);
        tr[i] = (tr_t)sym(h, trname);
    }
    free_t fr = (free_t)sym(h, "notorious_fft_free_aux");

    long total = 1;
    for (int i = 0; i < d; i++) total *= dims[i];
    long last = dims[d - 1];
    long half = total / last * (last / 2 + 1);
    long nin = cin ? 2 * (realin_half ? half : total) : total;
    long nout = cout ? 2 * (realout_half ? half : total) : total;
    char* x = (char*)malloc((size_t)(nin * batch) * rs);
    char* y = (char*)malloc((size_t)(nout * batch) * rs);
    if (!x || !y) { fprintf(stderr, "host allocation failed\n"); return 1; }
    fill(x, nin * batch, f32);
    double best = 1e30;
    double* per = (double*)malloc(sizeof(double) * reps);
    int nd = d > 1;
    for (int rep = 0; rep < reps; rep++) {
        double t0 = 0, t1 = 0;
        if (nd) {
            void* a = mk(d, dims);
            if (!a) { fprintf(stderr, "mkaux failed\n"); return 1; }
            t0 = omp_get_wtime();
            for (int k = 0; k < nk; k++)
                for (long b = 0; b < batch; b++)
                    tr[k](k ? y + b * nout * rs : x + b * nin * rs, y + b * nout * rs, a);
            t1 = omp_get_wtime();
            fr(a);
        } else {
            #pragma omp parallel num_threads(threads)
            {
                void* a = mk(1, dims);
                #pragma omp barrier
                #pragma omp single
                t0 = omp_get_wtime();
                for (int k = 0; k < nk; k++) {
                    #pragma omp for schedule(static)
                    for (long b = 0; b < batch; b++)
                        tr[k](k ? y + b * nout * rs : x + b * nin * rs, y + b * nout * rs, a);
                }
                #pragma omp single
                t1 = omp_get_wtime();
                fr(a);
            }
        }
        per[rep] = t1 - t0;
        if (t1 - t0 < best) best = t1 - t0;
    }
    double bytes = (double)nk * (double)batch * (double)(nin + nout) * (double)rs;
    printf("{\"kind\": \"%s\", \"dims\": \"%s\", \"batch\": %ld, \"threads\": %d, \"seconds\": %.6e, "
           "\"transforms_per_s\": %.6e, \"gbs\": %.6e, ",
           argv[3], argv[4], batch, nd ? 1 : threads, best, (double)nk * (double)batch / best, bytes / best / 1e9);
    print_reps(per, reps);
    printf("}\n");
    dlclose(h);
    return 0;
}

/*
 * notorious_fft.h -- drop-in C API of the B200 (sm_100a) Notorious-FFT engine.
 *
 * Source-compatible with the reference's public header (include/notorious_fft.h
 * of NotoriousLOB/Notorious-FFT, generated from src/01..07_*.h).  Reference
 * line citations use the module files; H:<n> is the generated header's line.
 *
 * Two shared libraries export the same symbol names, one per precision, as the
 * reference does through its NOTORIOUS_FFT_SINGLE typedef switch:
 *   libnotorious_fft.so   notorious_fft_real = double
 *   libnotorious_fftf.so  notorious_fft_real = float  (define NOTORIOUS_FFT_SINGLE)
 *
 * Pointers passed to the transforms may be host memory (pageable or pinned;
 * the call copies in, runs on the GPU, copies out and returns when the result
 * is in place, like the reference's synchronous CPU call) or device memory
 * (the call is enqueued on the library stream, see notorious_fft_set_stream,
 * and returns without waiting).  There is no CPU fallback: without a usable
 * GPU every mkaux_* returns NULL and notorious_fft_last_error() says why.
 */
#ifndef NOTORIOUS_FFT_B200_H
#define NOTORIOUS_FFT_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Scalar type: src/01_core.h:36-40 (H:135). */
#ifdef NOTORIOUS_FFT_SINGLE
typedef float notorious_fft_real;
#else
typedef double notorious_fft_real;
#endif

/* Interleaved complex (FFTW layout): src/07_legacy.h:19-23.  A plain struct in
 * C++ (no _Complex dependency), real[2] in C, exactly as the reference. */
#ifdef __cplusplus
typedef struct { notorious_fft_real re, im; } notorious_fft_cmpl;
#else
typedef notorious_fft_real notorious_fft_cmpl[2];
#endif

/* Plan handle.  Same field names and layout as the reference struct
 * (src/01_core.h:96-105); only N is meaningful to callers (the product of the
 * dimensions, as in the reference).  The remaining fields are owned by the
 * library: plan points to the device plan, sub1/sub2 are unused. */
struct notorious_fft_plan;
typedef struct notorious_fft_aux {
    int N;
    void* t;
    void* e;
    struct notorious_fft_aux *sub1, *sub2;
    struct notorious_fft_plan* plan;
    notorious_fft_real* scratch_re;
    notorious_fft_real* scratch_im;
} notorious_fft_aux;

/* ------------------------------------------------------------------------ */
/* The 27 reference entry points (src/07_legacy.h:29-57 = H:2226-2254).      */
/* ------------------------------------------------------------------------ */

/* Complex DFT, unnormalized, forward sign -1: src/07_legacy.h:146-148. */
void notorious_fft_dft(notorious_fft_cmpl* x, notorious_fft_cmpl* y, const notorious_fft_aux* a);
/* Inverse complex DFT, sign +1, unnormalized for power-of-two lengths and
 * scaled by 1/N for other lengths (the reference's Bluestein branch,
 * src/05_algorithms.h:315-333): src/07_legacy.h:150-152. */
void notorious_fft_invdft(notorious_fft_cmpl* x, notorious_fft_cmpl* y, const notorious_fft_aux* a);
/* Real DFT, N reals -> N/2+1 complex (Im of bins 0 and N/2 are 0):
 * src/07_legacy.h:162-237. */
void notorious_fft_realdft(notorious_fft_real* x, notorious_fft_cmpl* z, const notorious_fft_aux* a);
/* Inverse real DFT, unnormalized, reads only Re z_0 and Re z_{N/2}:
 * src/07_legacy.h:239-293. */
void notorious_fft_invrealdft(notorious_fft_cmpl* z, notorious_fft_real* y, const notorious_fft_aux* a);
/* DCT-2 / DST-2 (FFTW REDFT10 / RODFT10): src/07_legacy.h:798-865, :897-950. */
void notorious_fft_dct2(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a);
void notorious_fft_dst2(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a);
/* DCT-3 / DST-3 (REDFT01 / RODFT01): src/07_legacy.h:984-1010, :1040-1066. */
void notorious_fft_dct3(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a);
void notorious_fft_dst3(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a);
/* DCT-4 / DST-4 (REDFT11 / RODFT11): src/07_legacy.h:1336-1387. */
void notorious_fft_dct4(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a);
void notorious_fft_dst4(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a);

/* Plans.  NULL on N <= 0, on a non-power-of-two length for realdft / t2t3 / t4
 * (src/07_legacy.h:1406,1442,1579), or when device memory or the GPU is not
 * available.  Ns[0] is the slowest (outermost) dimension, C row-major:
 * src/07_legacy.h:1405-1688. */
notorious_fft_aux* notorious_fft_mkaux_dft_1d(int N);                          /* :1405-1420 */
notorious_fft_aux* notorious_fft_mkaux_dft_2d(int N1, int N2);                 /* :1430-1433 */
notorious_fft_aux* notorious_fft_mkaux_dft_3d(int N1, int N2, int N3);         /* :1435-1438 */
notorious_fft_aux* notorious_fft_mkaux_dft(int d, int* Ns);                    /* :1426-1428 */
notorious_fft_aux* notorious_fft_mkaux_realdft_1d(int N);                      /* :1441-1486 */
notorious_fft_aux* notorious_fft_mkaux_realdft_2d(int N1, int N2);             /* :1516-1519 */
notorious_fft_aux* notorious_fft_mkaux_realdft_3d(int N1, int N2, int N3);     /* :1521-1524 */
notorious_fft_aux* notorious_fft_mkaux_realdft(int d, int* Ns);                /* :1492-1514 */
notorious_fft_aux* notorious_fft_mkaux_t2t3_1d(int N);                         /* :1527-1558 */
notorious_fft_aux* notorious_fft_mkaux_t2t3_2d(int N1, int N2);                /* :1568-1571 */
notorious_fft_aux* notorious_fft_mkaux_t2t3_3d(int N1, int N2, int N3);        /* :1573-1576 */
notorious_fft_aux* notorious_fft_mkaux_t2t3(int d, int* Ns);                   /* :1564-1566 */
notorious_fft_aux* notorious_fft_mkaux_t4_1d(int N);                           /* :1578-1634 */
notorious_fft_aux* notorious_fft_mkaux_t4_2d(int N1, int N2);                  /* :1644-1647 */
notorious_fft_aux* notorious_fft_mkaux_t4_3d(int N1, int N2, int N3);          /* :1649-1652 */
notorious_fft_aux* notorious_fft_mkaux_t4(int d, int* Ns);                     /* :1640-1642 */

/* Recursive free, NULL-safe: src/07_legacy.h:1690-1700. */
void notorious_fft_free_aux(notorious_fft_aux* a);

/* ------------------------------------------------------------------------ */
/* Extensions (no counterpart in the reference, which is CPU-only).          */
/* ------------------------------------------------------------------------ */

/* Error reporting.  The reference transforms return void and silently do
 * nothing on a NULL plan (src/07_legacy.h:85); these calls keep that ABI and
 * record the last failure of the calling thread instead.  0 = success. */
enum {
    NOTORIOUS_FFT_OK = 0,
    NOTORIOUS_FFT_ERR_INVALID = 1,      /* bad size, NULL aux, wrong aux kind */
    NOTORIOUS_FFT_ERR_NO_DEVICE = 2,    /* no usable CUDA device */
    NOTORIOUS_FFT_ERR_ALLOC = 3,        /* device / pinned allocation failed */
    NOTORIOUS_FFT_ERR_CUDA = 4,         /* a CUDA runtime call failed */
    NOTORIOUS_FFT_ERR_TIMEOUT = 5,      /* a bounded device wait gave up */
    NOTORIOUS_FFT_ERR_UNSUPPORTED = 6   /* valid request this build cannot run */
};
int notorious_fft_last_error(void);
const char* notorious_fft_last_error_string(void);
void notorious_fft_clear_error(void);

/* Stream used for device-pointer calls (a cudaStream_t passed as void*).
 * NULL selects the legacy default stream.  Per calling thread. */
void notorious_fft_set_stream(void* stream);
void* notorious_fft_get_stream(void);
/* Block until all work the library enqueued on the current stream is done. */
int notorious_fft_synchronize(void);

/* Batched forms: `howmany` independent transforms of the aux's shape, the
 * b-th reading x + b*idist and writing y + b*odist.  Distances count elements
 * of the pointed-to type (notorious_fft_cmpl or notorious_fft_real), like
 * FFTW's advanced interface. */
void notorious_fft_dft_batched(notorious_fft_cmpl* x, notorious_fft_cmpl* y, const notorious_fft_aux* a,
                               int howmany, ptrdiff_t idist, ptrdiff_t odist);
void notorious_fft_invdft_batched(notorious_fft_cmpl* x, notorious_fft_cmpl* y, const notorious_fft_aux* a,
                                  int howmany, ptrdiff_t idist, ptrdiff_t odist);
void notorious_fft_realdft_batched(notorious_fft_real* x, notorious_fft_cmpl* z, const notorious_fft_aux* a,
                                   int howmany, ptrdiff_t idist, ptrdiff_t odist);
void notorious_fft_invrealdft_batched(notorious_fft_cmpl* z, notorious_fft_real* y, const notorious_fft_aux* a,
                                      int howmany, ptrdiff_t idist, ptrdiff_t odist);
void notorious_fft_dct2_batched(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a,
                                int howmany, ptrdiff_t idist, ptrdiff_t odist);
void notorious_fft_dst2_batched(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a,
                                int howmany, ptrdiff_t idist, ptrdiff_t odist);
void notorious_fft_dct3_batched(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a,
                                int howmany, ptrdiff_t idist, ptrdiff_t odist);
void notorious_fft_dst3_batched(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a,
                                int howmany, ptrdiff_t idist, ptrdiff_t odist);
void notorious_fft_dct4_batched(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a,
                                int howmany, ptrdiff_t idist, ptrdiff_t odist);
void notorious_fft_dst4_batched(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a,
                                int howmany, ptrdiff_t idist, ptrdiff_t odist);

/* Adjoints (vector-Jacobian products).  Given the cotangent g of a
 * transform's output, write the cotangent of its input, treating complex
 * data as pairs of reals.  Same argument order and shapes as the forward
 * call with input and output roles swapped:
 *   dft_vjp        g (N cmpl) -> invdft(g) for power-of-two axes
 *   invdft_vjp     g (N cmpl) -> dft(g)
 *   realdft_vjp    g (N/2+1 cmpl) -> N reals
 *   invrealdft_vjp g (N reals) -> N/2+1 cmpl
 *   dct2_vjp ... dst4_vjp  g (N reals) -> N reals                         */
void notorious_fft_dft_vjp(notorious_fft_cmpl* g, notorious_fft_cmpl* gx, const notorious_fft_aux* a);
void notorious_fft_invdft_vjp(notorious_fft_cmpl* g, notorious_fft_cmpl* gx, const notorious_fft_aux* a);
void notorious_fft_realdft_vjp(notorious_fft_cmpl* g, notorious_fft_real* gx, const notorious_fft_aux* a);
void notorious_fft_invrealdft_vjp(notorious_fft_real* g, notorious_fft_cmpl* gz, const notorious_fft_aux* a);
void notorious_fft_dct2_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a);
void notorious_fft_dst2_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a);
void notorious_fft_dct3_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a);
void notorious_fft_dst3_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a);
void notorious_fft_dct4_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a);
void notorious_fft_dst4_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a);
/* Batched adjoints: same batching convention as the *_batched calls, with
 * idist/odist measured on g and gx respectively. */
void notorious_fft_vjp_batched(int kind, void* g, void* gx, const notorious_fft_aux* a,
                               int howmany, ptrdiff_t idist, ptrdiff_t odist);

/* Transform kinds, for the generic entry points below. */
enum {
    NOTORIOUS_FFT_KIND_DFT = 0, NOTORIOUS_FFT_KIND_INVDFT = 1,
    NOTORIOUS_FFT_KIND_REALDFT = 2, NOTORIOUS_FFT_KIND_INVREALDFT = 3,
    NOTORIOUS_FFT_KIND_DCT2 = 4, NOTORIOUS_FFT_KIND_DST2 = 5,
    NOTORIOUS_FFT_KIND_DCT3 = 6, NOTORIOUS_FFT_KIND_DST3 = 7,
    NOTORIOUS_FFT_KIND_DCT4 = 8, NOTORIOUS_FFT_KIND_DST4 = 9
};

/* Generic batched transform: kind selects the transform (the aux must be of
 * the matching family). */
void notorious_fft_execute_batched(int kind, void* x, void* y, const notorious_fft_aux* a,
                                   int howmany, ptrdiff_t idist, ptrdiff_t odist);

/* Precision forms (float library only).  FORM_PLAIN runs every stage on the
 * FP32 CUDA-core path.  FORM_SPLIT_TC runs the radix-16 inner DFTs of a
 * power-of-two complex DFT as FP16 hi+lo split products on the tensor cores
 * with FP32 accumulation and per-tile power-of-two scaling; twiddles and
 * Bluestein chirps are still generated in FP64 at plan time.  Returns 0, or
 * an error code (the double library returns UNSUPPORTED for SPLIT_TC). */
enum { NOTORIOUS_FFT_FORM_PLAIN = 0, NOTORIOUS_FFT_FORM_SPLIT_TC = 1 };
int notorious_fft_set_form(notorious_fft_aux* a, int form);
int notorious_fft_get_form(const notorious_fft_aux* a);

/* Allocation-free batched complex DFT (no counterpart in the reference).
 * For callers that cannot call cudaMalloc -- code running inside another
 * framework's memory manager, which owns the device heap, and latency-critical
 * code that cannot take cudaMalloc's implicit device synchronization.  It
 * runs `howmany` contiguous power-of-two transforms of length N
 * (1 <= N <= 2^20; other lengths return NOTORIOUS_FFT_ERR_INVALID) from
 * device memory x to device memory y (x == y allowed) on `stream`
 * (a cudaStream_t, NULL for the legacy stream), forward (inverse = 0) or
 * unnormalized inverse (inverse = 1), and allocates nothing: its scratch is a
 * fixed 16 MiB __device__ array (plus the twiddle tables) that every GPU
 * loading the library holds until exit.  The first call on a device resolves
 * those arrays' addresses and fills the tables, waiting for that kernel, so it
 * should come before any stream capture.  All calls share the scratch array:
 * calls that overlap on the GPU race.  Returns 0 or an error code. */
int notorious_fft_dft_noalloc(const notorious_fft_cmpl* x, notorious_fft_cmpl* y, int N, int howmany, int inverse,
                              void* stream);

/* Ragged batches (no counterpart in the reference, whose callers loop over
 * transforms one aux at a time, e.g. benchmarks/bench_mixed_sizes.c).  A
 * batch is `count` independent 1-D transforms of mixed kinds
 * (NOTORIOUS_FFT_KIND_*) and lengths, executed by ONE persistent GPU launch
 * (captured in a CUDA graph) that works through a device queue of tiles.
 * Transform i reads in + in_offsets[i] and writes out + out_offsets[i];
 * offsets count notorious_fft_real elements (complex data: even offsets).
 * NULL offsets select the packed layout: transforms back to back in index
 * order, each starting at an even offset.  Every kind accepts power-of-two
 * lengths; dft, invdft, realdft and dct2 accept any length >= 1 (Bluestein;
 * realdft then returns floor(N/2)+1 bins, invdft scales by 1/N as the
 * reference does).  Returns NULL on error (see notorious_fft_last_error). */
typedef struct notorious_fft_batch notorious_fft_batch;
notorious_fft_batch* notorious_fft_mkbatch(int count, const int* kinds, const int* Ns, const long long* in_offsets,
                                           const long long* out_offsets);
/* Input / output buffer sizes the batch needs, in notorious_fft_real. */
long long notorious_fft_batch_in_size(const notorious_fft_batch* b);
long long notorious_fft_batch_out_size(const notorious_fft_batch* b);
/* Run the batch.  Device pointers: asynchronous on the current stream (check
 * notorious_fft_batch_status afterwards).  Host pointers: staged, synchronous,
 * returns the status.  Device buffers may be the same (in == out) only when
 * every transform maps onto itself (equal offsets, length-preserving kinds);
 * host buffers are staged and may always coincide.  Returns 0 or an error. */
int notorious_fft_batch_execute(notorious_fft_batch* b, const notorious_fft_real* in, notorious_fft_real* out);
/* Wait for the batch's last launch; NOTORIOUS_FFT_ERR_TIMEOUT if a bounded
 * device wait gave up (the launch was abandoned and the output is invalid). */
int notorious_fft_batch_status(notorious_fft_batch* b);
/* Launch through a CUDA graph (default 1) or directly (0). */
int notorious_fft_batch_set_graph(notorious_fft_batch* b, int enable);
/* Queue statistics: items, tiles, device scratch bytes, persistent CTAs. */
int notorious_fft_batch_info(const notorious_fft_batch* b, long long* items, long long* tiles,
                             long long* scratch_bytes, int* ctas);
void notorious_fft_free_batch(notorious_fft_batch* b);
/* Test hook for the bounded waits: the next execution withholds one
 * dependency (its counter is never published) and waits at most spin_limit
 * polls, so the launch must end with NOTORIOUS_FFT_ERR_TIMEOUT. */
int notorious_fft_batch_debug_withhold(notorious_fft_batch* b, long long spin_limit);

/* Autotuner.  Times the executable pass splits of a power-of-two transform
 * (kind, N) in the queue on this GPU, keeps the fastest, and stores it in the
 * tune cache (a JSON file: $NOTORIOUS_FFT_TUNE_CACHE, default
 * ~/.cache/notorious_fft/tune.json, keyed by GPU name + driver, precision,
 * kind and N).  Later batches use the cached split.  It then tunes standalone
 * plans of the same length (see notorious_fft_tune_lookup_plan).  Returns 0
 * or an error. */
int notorious_fft_autotune(int kind, int N);
/* The cached split for (kind, N): writes up to max_passes log2 radices and
 * returns their count (0: none cached). */
int notorious_fft_tune_lookup(int kind, int N, int* log2_radices, int max_passes);
/* notorious_fft_autotune also times standalone plans of the family of `kind`
 * (the default schedule and the executable pass splits, each with the
 * default thread rule and with 128- and 256-thread pass kernels) and caches
 * the fastest; every later mkaux_* of that family uses the cached schedule
 * for power-of-two axes of length N.  This returns the cached split (up to
 * max_passes log2 radices; 0 = the default schedule) and writes the thread
 * count (log2, 0 = the default rule) to *log2_threads; -1: nothing cached. */
int notorious_fft_tune_lookup_plan(int kind, int N, int* log2_radices, int max_passes, int* log2_threads);
/* The schedule an aux runs on one axis (0 = slowest, -1 = last): the pass
 * radices (log2) of the axis's power-of-two inner FFT and the thread count
 * (log2, 0 = the default rule) of its pass kernels.  Returns the pass count,
 * 0 for a Bluestein axis, -1 on error. */
int notorious_fft_aux_schedule(const notorious_fft_aux* a, int axis, int* log2_radices, int max_passes,
                               int* log2_threads);

/* Library identification: precision of this build's notorious_fft_real
 * (8 or 4) and a short version string. */
int notorious_fft_real_size(void);
const char* notorious_fft_version(void);
/* Number of GPU kernels this library has launched in the calling process. */
long long notorious_fft_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* NOTORIOUS_FFT_B200_H */

// nfft_engine.h -- host-side engine of the B200 FFT library (internal).
//
// A plan (struct notorious_fft_plan) is a list of axis steps.  Each step runs
// one 1-D transform along one axis of a strided view, as one or more Stockham
// passes (nfft_pass.cuh), with the transform family's pre/post operators fused
// into the first and last pass.  Power-of-two axes use the passes directly;
// other complex axes use Bluestein (chirp premultiply fused into the first
// forward pass, the filter product into the first inverse pass -- or, when the
// padded length fits one tile, the whole convolution in one pass -- and window
// + chirp postmultiply into the last inverse pass).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "nfft_pass.cuh"

#ifndef NFFT_REAL
#define NFFT_REAL double
#endif

namespace nfft {

using real_t = NFFT_REAL;
using cplx_t = C2<real_t>;

// ---- errors ---------------------------------------------------------------
void set_error(int code, const char* fmt, ...);
int last_error();
const char* last_error_string();
void clear_error();
bool cuda_ok(cudaError_t e, const char* what);

// ---- per-device context ---------------------------------------------------
struct DeviceCtx {
    int device = -1;
    int sm_count = 0;
    size_t l2_bytes = 0;
    TwTables<real_t>* tw = nullptr;   // device twiddle tables
    bool ready = false;
};
DeviceCtx* device_ctx(int device);   // initializes on first use (tables, kernel attributes)
DeviceCtx* current_ctx();            // context of the calling thread's current device, or null

// ---- transform families / kinds ---------------------------------------------
enum Family { FAM_DFT = 0, FAM_REAL = 1, FAM_T2T3 = 2, FAM_T4 = 3 };
enum Kind {
    K_DFT = 0, K_INVDFT = 1, K_REALDFT = 2, K_INVREALDFT = 3,
    K_DCT2 = 4, K_DST2 = 5, K_DCT3 = 6, K_DST3 = 7, K_DCT4 = 8, K_DST4 = 9
};
Family family_of(int kind);

// ---- strided views ----------------------------------------------------------
// Lines of one axis: element e of line (b0, b1, ...) lives at
//   ptr + sum_d b_d * str[d] + e * estride        (units: elements of the view type)
constexpr int MAX_BATCH_DIMS = 3;
struct View {
    void* ptr = nullptr;
    long long estride = 1;
    int nb = 0;                          // batch dims, innermost first
    long long cnt[MAX_BATCH_DIMS] = {1, 1, 1};
    long long str[MAX_BATCH_DIMS] = {0, 0, 0};
    long long lines() const {
        long long n = 1;
        for (int i = 0; i < nb; ++i) n *= cnt[i];
        return n;
    }
};

// ---- power-of-two complex FFT schedule ------------------------------------
struct FftSchedule {
    int logL = 0;
    int npass = 0;
    int logt = 0;                    // threads (log2) of the specialized pass kernels; 0: the default rule
    int plog[4] = {0, 0, 0, 0};      // pass radices (log2), in execution order
    int tile[4] = {12, 12, 12, 12};  // log2 tile size of each pass
    int nsub[4] = {0, 0, 0, 0};
    int sub[4][MAX_SUB] = {};
};
// strided: the axis is not contiguous (every pass runs in column mode).
// max_tile: log2 of the largest tile (13: 512-thread kernels; 12: the queue).
// max_pass_log: largest pass radix (log2); -1 = the default rule, 0 = no cap.
FftSchedule make_schedule(int logL, bool strided, int max_tile = 13, int max_pass_log = -1);
// Explicit pass radices (log2, execution order; 4096-point tiles).  False when
// the split is not executable (radix too large for its tile, wrong sum).
bool make_split_schedule(int logL, const int* plog, int npass, FftSchedule* out);
FftSchedule reversed(const FftSchedule& s);

// ---- one axis of a plan -------------------------------------------------------
struct AxisPlan {
    int n = 1;                 // axis length (real length for the real families)
    bool pow2 = true;
    int logn = 0;
    // power-of-two inner complex FFT (length n for dft, n/2 for the real families)
    FftSchedule fft_contig, fft_strided;
    // Bluestein (complex family, n not a power of two)
    int logM = 0;
    cplx_t* chirp = nullptr;   // e^{-i pi k^2/n}, k < n
    cplx_t* filt = nullptr;    // FFT_M(conj chirp, wrapped) / M
    cplx_t* post = nullptr;    // DCT-2 of any length: e^{-i pi q / 2n}, q < n (queue plans only)
    FftSchedule mfwd, minv;    // M-point forward schedule and its reverse
};

}  // namespace nfft

struct notorious_fft_batch;   // a ragged batch (nfft_queue_build.cu)

// The plan behind notorious_fft_aux::plan.
struct notorious_fft_plan {
    int family = 0;
    int device = -1;
    std::vector<int> dims;            // Ns[0] slowest
    std::vector<nfft::AxisPlan> axes;
    int form = 0;                     // precision form (NOTORIOUS_FFT_FORM_*)
    // scratch (device), grown on demand; [0],[1] ping-pong of multi-pass axes
    void* scratch[2] = {nullptr, nullptr};
    size_t scratch_bytes[2] = {0, 0};
    // device staging for host-pointer calls
    void* stage_in = nullptr;
    void* stage_out = nullptr;
    size_t stage_in_bytes = 0, stage_out_bytes = 0;
    // pipelined host-pointer calls: copy streams, events, double-buffered staging
    cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
    cudaEvent_t ev_h[2] = {nullptr, nullptr}, ev_c[2] = {nullptr, nullptr}, ev_d[2] = {nullptr, nullptr};
    // pageable host calls: pinned host bounce buffers of the chunks in flight
    void* host_in = nullptr;
    void* host_out = nullptr;
    size_t host_in_bytes = 0, host_out_bytes = 0;
    // temporary of the multi-dimensional inverse real transform
    void* nd_tmp = nullptr;
    size_t nd_tmp_bytes = 0;
    // ordering across streams: the scratch above is shared by every call on
    // this plan, so a call on another stream than the previous call's first
    // waits for the event recorded at the end of that call
    cudaStream_t last_stream = nullptr;
    cudaEvent_t ev_last = nullptr;
    bool ev_pending = false;
    std::mutex mu;
};

namespace nfft {

notorious_fft_plan* plan_create(int family, int d, const int* Ns);
void plan_destroy(notorious_fft_plan* p);
// Elements (of the family's input / output type) of one transform.
long long plan_in_elems(const notorious_fft_plan* p, int kind);
long long plan_out_elems(const notorious_fft_plan* p, int kind);
// Element sizes (bytes) of the input / output type of `kind`.
size_t in_elem_bytes(int kind);
size_t out_elem_bytes(int kind);
// Run `kind` on device pointers (asynchronous on `stream`).  Returns 0 on success.
// vjp != 0 runs the adjoint of `kind` (input: the cotangent of its output).
int plan_execute(notorious_fft_plan* p, int kind, const void* in, void* out, long long howmany,
                 long long idist, long long odist, cudaStream_t stream, int vjp = 0);

// Fused operators of one transform (first-pass load / last-pass store).
struct OpSpec {
    int ld = LD_C, st = ST_C;
    int conj_in = 0, conj_out = 0;
    double scale = 1.0;
    long long N = 0;
    int logN = 0;
    int dst = 0;
    bool paired = false;   // st is ST_R / ST_T2 (needs whole lines or the unpack epilogue)
    int vjp = 0;           // adjoint weights of the real operators
    int tc = 0;            // split tensor-core radix-16 sub-stages (float library)
    int logt = 0;          // threads (log2) of the specialized pass kernels; 0: the default rule
    const void* post = nullptr;   // ST_BLUE_T2 post-twiddle table
};

// ---- launch recording (ragged-batch queue, nfft_queue.h) ---------------------
// While recorder() is non-null on the calling thread, the planner records the
// passes it would launch (queue branch key, arguments, tile count) instead of
// launching them, and plans for the queue's 4096-point tiles.
struct RecLaunch {
    int op;                   // QOP_* key
    PassArgs a;
    long long ntiles;
    const void* z = nullptr;  // unpack: packed spectrum and its line distance
    long long zdist = 0;
};
struct Recorder {
    std::vector<RecLaunch> launches;
};
Recorder*& recorder();
bool queue_has_lean(int logR, int ci, int co, int ld, int st);
// A 1-D plan of `kind` for the queue: 4096-point tiles, optional explicit pass
// split of the inner power-of-two FFT (npass = 0: default schedule).  Any
// length n >= 2 for dft / invdft, and for realdft / DCT-2 (Bluestein with
// real-input operators when n is not a power of two); powers of two otherwise.
notorious_fft_plan* plan_create_queue(int kind, int n, const int* plog, int npass);
// Record the passes of `count` transforms of `kind` from in to out (recorder()
// must be set).  Returns 0 on success.
int plan_record(notorious_fft_plan* p, int kind, const void* in, void* out, long long count, long long idist,
                long long odist);

// One Stockham pass of an axis of length 2^logL (nfft_plan.cu).
bool run_pass(const DeviceCtx* c, const View& src, const View& dst, int logL, int logNs, int logR, int tile,
              int nsub, const int* sub, const OpSpec& op, bool first, bool last, int mid, int logNs_out,
              const cplx_t* chirp, const cplx_t* filt, cudaStream_t s, bool in_scratch = false,
              bool out_scratch = false);
// Inter-pass scratch layout with the lines of `like` and axis length L.
View scratch_view(void* ptr, const View& like, long long L, bool strided);

// Kernel launchers (nfft_kernels.cu)
bool launch_pass(const PassArgs& a, int load_op, int store_op, int log_tile, long long ntiles, cudaStream_t s);
bool launch_unpack(const PassArgs& a, int store_op, const cplx_t* Z, long long zdist, long long nlines, cudaStream_t s);
bool launch_tiny(const real_t* x, real_t* y, long long howmany, long long inner, long long idist, long long odist,
                 int in_cplx, int out_cplx, double factor, cudaStream_t s);
bool launch_init_tables(TwTables<real_t>* tw, cudaStream_t s);
bool launch_chirp(cplx_t* chirp, cplx_t* bwrap, long long n, long long M, cudaStream_t s);
// post[q] = e^{-i pi q / 2n}, q < n (FP64 sincospi)
bool launch_post(cplx_t* post, long long n, cudaStream_t s);
bool set_kernel_attributes();

// Persistent queue kernel (nfft_queue_kernel.cu)
struct QueueArgs;
int queue_grid(const DeviceCtx* c);   // resident CTAs (0 on error)
bool launch_queue(const QueueArgs& q, int grid, cudaStream_t s);

// Ragged batches (nfft_queue_build.cu).  Offsets in reals, NULL: packed.
notorious_fft_batch* batch_create_default(int count, const int* kinds, const int* Ns, const long long* in_off,
                                          const long long* out_off);
void batch_destroy(notorious_fft_batch* b);
int batch_run(notorious_fft_batch* b, const void* din, void* dout, cudaStream_t s);        // device pointers, async
int batch_run_host(notorious_fft_batch* b, const void* hin, void* hout, cudaStream_t s);   // host pointers, sync
int batch_status(notorious_fft_batch* b);
long long batch_in_reals(const notorious_fft_batch* b);
long long batch_out_reals(const notorious_fft_batch* b);
void batch_info(const notorious_fft_batch* b, long long* items, long long* tiles, long long* scratch, int* ctas);
void batch_set_graph(notorious_fft_batch* b, int enable);
void batch_withhold(notorious_fft_batch* b, long long spin_limit);
int autotune(int kind, int n, cudaStream_t s);
int tune_lookup(int kind, int n, int* plog, int max_passes);
// Standalone plans: the cached pass split and thread count of a power-of-two
// axis of transform family `family` and length n (false: none cached), and
// the same for the C API.
bool tune_get_plan(int family, int n, std::vector<int>& split, int& logt);
int tune_lookup_plan(int kind, int n, int* plog, int max_passes, int* logt);
// While set on the calling thread, build_axis uses this split / thread count
// for every power-of-two axis instead of the cache (the autotuner's trials).
struct PlanOverride {
    std::vector<int> split;
    int logt = 0;
};
PlanOverride*& plan_override();
long long launch_count();
void note_launch();

// Split-tensor-core pass (nfft_tc.cu, float library): LD_C / ST_C passes.
bool launch_tc_pass(const PassArgs& a, int log_tile, long long ntiles, cudaStream_t s);
// Radix-256 passes of the split tensor-core form (16-line tiles, persistent
// CTAs, nfft_tc_lean.cuh); NOTORIOUS_FFT_TC_LEAN=0 selects tc_pass_kernel.
bool tc_lean_enabled();
bool launch_tc_lean(const PassArgs& a, int sm_count, cudaStream_t s);
// The same passes on the sm_100 tensor cores (tcgen05, nfft_umma.cuh) for
// unit-stride lines with 16-byte aligned buffers and strides; returns false
// without launching (and without an error) when the pass is not of that
// shape.  NOTORIOUS_FFT_TC_UMMA=0 keeps every pass on launch_tc_lean.
bool tc_umma_enabled();
bool try_launch_tc_umma(const PassArgs& a, int sm_count, cudaStream_t s, bool& launched);
// First wait of a tcgen05 pass that gave up since the last call (0: none), cleared.
unsigned tc_umma_take_status();

// Specialized pass kernels (nfft_lean.cuh), registered by the slice files.
constexpr int NFFT_LEAN_SLICES = 8;
inline unsigned lean_key(int logR, int logT, int ci, int co, int ld, int st) {
    return (unsigned)logR | ((unsigned)logT << 5) | ((unsigned)ci << 10) | ((unsigned)co << 11) | ((unsigned)ld << 12) |
           ((unsigned)st << 16);
}
struct LeanEntry {
    const void* fn = nullptr;
    size_t smem = 0;
    int threads = 0;
};
struct LeanRegistry {
    std::vector<std::pair<unsigned, LeanEntry>> entries;
    void add(unsigned key, const void* fn, size_t smem, int threads) { entries.push_back({key, LeanEntry{fn, smem, threads}}); }
    const LeanEntry* find(unsigned key) const {
        for (auto& e : entries)
            if (e.first == key) return &e.second;
        return nullptr;
    }
};
const LeanRegistry& lean_registry();
// Launch the specialized kernel for this pass shape, or return false with no
// error set when none is instantiated (the caller then uses pass_kernel).
bool lean_available(int logR, int logT, int ci, int co, int ld, int st);
bool launch_lean(const PassArgs& a, int logT, int ci, int co, int ld, int st, long long ntiles, cudaStream_t s);

}  // namespace nfft

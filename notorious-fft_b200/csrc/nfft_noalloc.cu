// nfft_noalloc.cu -- an allocation-free batched complex DFT.
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory manager, which owns the device heap and does not allow
// direct driver allocations, and latency-critical code for which the
// implicit device synchronization of cudaMalloc / cudaFree is not
// acceptable.  notorious_fft_dft_noalloc serves them: it runs the same
// Stockham passes as the regular multi-pass complex DFT, but its inter-pass
// scratch and its twiddle tables live in file-scope __device__ arrays of a
// fixed size instead of memory the library allocates.  Every GPU that loads
// this library holds those arrays (16 MiB of scratch plus the tables) until
// the process exits.
//
// The arrays are shared by every call: a call leaves its intermediate data
// in the scratch array, and two calls whose kernels overlap on the GPU (for
// example on two streams, or from two host threads) race on it.  The scratch
// is always written before it is read, so nothing needs clearing.
//
// In host code the arrays' names are host-side stand-ins, not device
// addresses, so the first call on each device looks up their device
// addresses with cudaGetSymbolAddress (with that device current), fills the
// twiddle tables with a kernel and waits for it.  That first call per device
// should therefore come before any stream capture.
#include <algorithm>
#include <mutex>

#include "../../include/notorious_fft.h"
#include "nfft_engine.h"

namespace {

using namespace nfft;

constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)16 << 20;
constexpr long long NOALLOC_SCRATCH_ELEMS = (long long)(NOALLOC_SCRATCH_BYTES / sizeof(cplx_t));
constexpr int NOALLOC_MAX_LOGN = 20;

__device__ __align__(256) cplx_t g_noalloc_scratch[NOALLOC_SCRATCH_ELEMS];
__device__ __align__(256) TwTables<real_t> g_noalloc_tw;

struct NoallocDevice {
    bool ready = false;
    cplx_t* scratch = nullptr;
    TwTables<real_t>* tw = nullptr;
    int sm_count = 0;       // read once per device; the pass launcher sizes grids
    size_t l2_bytes = 0;    // and picks its L2 policy from these, as for plans
};
std::mutex g_noalloc_mu;
NoallocDevice g_noalloc_dev[64];

// One-time set-up of the calling thread's current device (see the file header).
// The set-up waits for a kernel, so it cannot run while `stream` is being
// captured into a CUDA graph: such a first call is refused with a message.
NoallocDevice* noalloc_device(cudaStream_t stream) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        set_error(NOTORIOUS_FFT_ERR_NO_DEVICE, "no CUDA device available");
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoallocDevice& d = g_noalloc_dev[dev];
    if (d.ready) return &d;
    int major = 0, sms = 0, l2 = 0;
    if (!cuda_ok(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev), "cudaDeviceGetAttribute") ||
        !cuda_ok(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute") ||
        !cuda_ok(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev), "cudaDeviceGetAttribute"))
        return nullptr;
    if (major < 10) {
        set_error(NOTORIOUS_FFT_ERR_NO_DEVICE, "device %d (sm_%d) is not an sm_100 GPU", dev, major);
        return nullptr;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (!cuda_ok(cudaStreamIsCapturing(stream, &cap), "cudaStreamIsCapturing")) return nullptr;
    if (cap != cudaStreamCaptureStatusNone) {
        set_error(NOTORIOUS_FFT_ERR_UNSUPPORTED,
                  "notorious_fft_dft_noalloc: the first call on a device sets up its tables and waits for them; "
                  "make one call on this device before capturing a stream");
        return nullptr;
    }
    void* scratch = nullptr;
    void* tw = nullptr;
    if (!cuda_ok(cudaGetSymbolAddress(&scratch, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)")) return nullptr;
    if (!cuda_ok(cudaGetSymbolAddress(&tw, g_noalloc_tw), "cudaGetSymbolAddress(twiddle tables)")) return nullptr;
    if (!set_kernel_attributes()) return nullptr;
    if (!launch_init_tables((TwTables<real_t>*)tw, 0)) return nullptr;
    if (!cuda_ok(cudaStreamSynchronize(0), "twiddle table set-up")) return nullptr;
    d.scratch = (cplx_t*)scratch;
    d.tw = (TwTables<real_t>*)tw;
    d.sm_count = sms;
    d.l2_bytes = (size_t)l2;
    d.ready = true;
    return &d;
}

}  // namespace

extern "C" int notorious_fft_dft_noalloc(const notorious_fft_cmpl* x, notorious_fft_cmpl* y, int N, int howmany,
                                         int inverse, void* stream) {
    clear_error();
    if (!x || !y) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "NULL data pointer");
        return NOTORIOUS_FFT_ERR_INVALID;
    }
    if (N < 1 || (N & (N - 1)) != 0 || N > (1 << NOALLOC_MAX_LOGN)) {
        set_error(NOTORIOUS_FFT_ERR_INVALID,
                  "notorious_fft_dft_noalloc: N=%d must be a power of two <= %d (scratch limit %zu bytes per GPU); "
                  "use notorious_fft_dft_batched for other lengths",
                  N, 1 << NOALLOC_MAX_LOGN, NOALLOC_SCRATCH_BYTES);
        return NOTORIOUS_FFT_ERR_INVALID;
    }
    if (howmany < 0) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "negative batch count");
        return NOTORIOUS_FFT_ERR_INVALID;
    }
    if (((uintptr_t)x | (uintptr_t)y) % sizeof(cplx_t)) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "device pointers must be aligned to notorious_fft_cmpl");
        return NOTORIOUS_FFT_ERR_INVALID;
    }
    if (howmany == 0) return 0;
    cudaStream_t s = (cudaStream_t)stream;
    NoallocDevice* d = noalloc_device(s);
    if (!d) return last_error();
    DeviceCtx ctx;
    ctx.tw = d->tw;
    ctx.sm_count = d->sm_count;
    ctx.l2_bytes = d->l2_bytes;
    int logN = 0;
    while ((1 << logN) < N) ++logN;
    const long long L = N;
    const long long half = NOALLOC_SCRATCH_ELEMS / 2;
    // The default schedule, unless it runs more than two passes (the passes
    // then alternate between the two halves of the scratch array) and a
    // transform does not fit in half: then the uncapped two-pass schedule,
    // which for N <= 2^20 always has at most two passes and so needs only one
    // buffer of at most the whole array (FP64 2^20 fills it exactly).
    FftSchedule sch = make_schedule(logN, false);
    if (sch.npass > 2 && L > half) sch = make_schedule(logN, false, 13, 0);
    OpSpec op;
    op.conj_in = op.conj_out = inverse ? 1 : 0;
    // whole transforms per scratch fill
    const long long per_buf = sch.npass > 2 ? half : NOALLOC_SCRATCH_ELEMS;
    const long long chunk = sch.npass == 1 ? howmany : std::max<long long>(1, per_buf / L);
    cplx_t* const bufs[2] = {d->scratch, d->scratch + half};
    for (long long b0 = 0; b0 < howmany; b0 += chunk) {
        const long long cn = std::min(chunk, (long long)howmany - b0);
        View vs, vd;
        vs.ptr = (void*)((const cplx_t*)x + b0 * L);
        vd.ptr = (void*)((cplx_t*)y + b0 * L);
        vs.estride = vd.estride = 1;
        if (cn > 1) {
            vs.nb = vd.nb = 1;
            vs.cnt[0] = vd.cnt[0] = cn;
            vs.str[0] = vd.str[0] = L;
        }
        View cur = vs;
        int logNs = 0;
        for (int i = 0; i < sch.npass; ++i) {
            const bool first = i == 0, last = i == sch.npass - 1;
            const View out = last ? vd : scratch_view(sch.npass > 2 ? bufs[i & 1] : d->scratch, vs, L, false);
            if (!run_pass(&ctx, cur, out, logN, logNs, sch.plog[i], sch.tile[i], sch.nsub[i], sch.sub[i], op, first,
                          last, 0, logNs, nullptr, nullptr, s, !first, !last))
                return last_error() ? last_error() : NOTORIOUS_FFT_ERR_CUDA;
            logNs += sch.plog[i];
            cur = out;
        }
    }
    return 0;
}

// nfft_api.cu -- the C ABI: the reference's 27 entry points
// (src/07_legacy.h:29-57 of Notorious-FFT) plus the extensions declared in
// include/notorious_fft.h.  Everything here is host code; all arithmetic runs
// in the pass kernels.  Host pointers are staged through device buffers owned
// by the plan; device pointers are used in place.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "../../include/notorious_fft.h"
#include "nfft_engine.h"

using namespace nfft;

static_assert(sizeof(notorious_fft_real) == sizeof(real_t), "header precision must match the build precision");

namespace {

thread_local cudaStream_t t_stream = 0;

notorious_fft_aux* make_aux(int family, int d, const int* Ns) {
    clear_error();
    notorious_fft_plan* p = plan_create(family, d, Ns);
    if (!p) return nullptr;
    notorious_fft_aux* a = (notorious_fft_aux*)calloc(1, sizeof(notorious_fft_aux));
    if (!a) {
        plan_destroy(p);
        set_error(NOTORIOUS_FFT_ERR_ALLOC, "host allocation of the aux failed");
        return nullptr;
    }
    long long total = 1;
    for (int i = 0; i < d; ++i) total *= Ns[i];
    a->N = (int)total;
    a->plan = p;
    return a;
}

bool grow(void** buf, size_t* have, size_t need);

bool is_pinned_host_ptr(const void* ptr) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeHost;
}

// Batched call with both buffers in pinned host memory: the batch goes through
// the GPU in chunks, with the copy-in of chunk k+1 and the copy-out of chunk
// k-1 overlapping the transform of chunk k (copy engines in both directions
// plus the compute stream).  Transforms stay ordered on the caller's stream, so
// the plan's scratch is never used by two chunks at once.
// Host-side copy of n bytes between pageable and pinned memory, split over
// worker threads (NOTORIOUS_FFT_HOST_COPY_THREADS, default every hardware
// thread up to 32): the pageable pipeline is bound by these copies (B200 host,
// 16 threads: 4 / 8 / 12 / 16 threads gave 19 / 26 / 31 / 35 GB/s end to end on
// 4096 x 2^16 FP64 dft + invdft, against 9.7 GB/s through the driver's own
// staging of pageable memory).
// Input bytes per chunk of the host-pointer pipelines (NOTORIOUS_FFT_PIPE_CHUNK_MB).
size_t pipe_chunk_bytes() {
    static size_t v = 0;
    if (!v) {
        const char* e = getenv("NOTORIOUS_FFT_PIPE_CHUNK_MB");
        const long long mb = e ? atoll(e) : 64;
        v = (size_t)std::max(1ll, std::min(mb, 4096ll)) << 20;
    }
    return v;
}

int host_copy_threads() {
    static int v = 0;
    if (!v) {
        const char* e = getenv("NOTORIOUS_FFT_HOST_COPY_THREADS");
        int n = e ? atoi(e) : (int)std::min(32u, std::max(1u, std::thread::hardware_concurrency()));
        v = std::max(1, std::min(n, 64));
    }
    return v;
}
void host_copy(void* dst, const void* src, size_t n) {
    const int T = host_copy_threads();
    const size_t min_piece = (size_t)4 << 20;
    const int parts = (int)std::max<size_t>(1, std::min<size_t>((size_t)T, n / min_piece));
    if (parts <= 1) {
        memcpy(dst, src, n);
        return;
    }
    const size_t piece = (n / parts + 63) & ~(size_t)63;
    std::vector<std::thread> th;
    th.reserve(parts - 1);
    for (int k = 1; k < parts; ++k) {
        const size_t off = (size_t)k * piece;
        if (off >= n) break;
        const size_t len = std::min(piece, n - off);
        th.emplace_back([=]() { memcpy((char*)dst + off, (const char*)src + off, len); });
    }
    memcpy(dst, src, std::min(piece, n));
    for (auto& t : th) t.join();
}

bool grow_pinned(void** buf, size_t* have, size_t need) {
    if (*have >= need && *buf) return true;
    if (*buf) cudaFreeHost(*buf);
    *buf = nullptr;
    *have = 0;
    if (!cuda_ok(cudaMallocHost(buf, need), "cudaMallocHost(bounce buffers)")) return false;
    *have = need;
    return true;
}

bool ensure_copy_streams(notorious_fft_plan* p) {
    if (p->s_h2d) return true;
    if (!cuda_ok(cudaStreamCreateWithFlags(&p->s_h2d, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
    if (!cuda_ok(cudaStreamCreateWithFlags(&p->s_d2h, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
    for (int i = 0; i < 2; ++i) {
        if (!cuda_ok(cudaEventCreateWithFlags(&p->ev_h[i], cudaEventDisableTiming), "cudaEventCreate") ||
            !cuda_ok(cudaEventCreateWithFlags(&p->ev_c[i], cudaEventDisableTiming), "cudaEventCreate") ||
            !cuda_ok(cudaEventCreateWithFlags(&p->ev_d[i], cudaEventDisableTiming), "cudaEventCreate"))
            return false;
    }
    return true;
}

// Batched call with both buffers in pageable host memory: the pinned path's
// chunks (copy-in of chunk k+1 and copy-out of chunk k-1 around the transform
// of chunk k), with two pinned bounce buffers per direction that host threads
// fill from x and drain into y.  The host copies chunk k in, queues its device
// work, then drains chunk k-1 once its device-to-host copy is done; a bounce
// buffer is refilled only after the copy that read it (an event) completed.
bool run_pageable_pipelined(notorious_fft_plan* p, int kind, const void* x, void* y, long long howmany,
                            long long idist, long long odist, long long in_elems, long long out_elems, size_t in_eb,
                            size_t out_eb, int vjp, cudaStream_t s) {
    const size_t target = pipe_chunk_bytes();
    long long chunk = (long long)(target / std::max<size_t>((size_t)idist * in_eb, 1));
    if (chunk < 1) chunk = 1;
    if (chunk > howmany) chunk = howmany;
    const size_t cin = (size_t)((chunk - 1) * idist + in_elems) * in_eb;
    const size_t cout = (size_t)((chunk - 1) * odist + out_elems) * out_eb;
    if (!ensure_copy_streams(p)) return false;
    if (!grow(&p->stage_in, &p->stage_in_bytes, 2 * cin)) return false;
    if (!grow(&p->stage_out, &p->stage_out_bytes, 2 * cout)) return false;
    if (!grow_pinned(&p->host_in, &p->host_in_bytes, 2 * cin)) return false;
    if (!grow_pinned(&p->host_out, &p->host_out_bytes, 2 * cout)) return false;
    char* in_st[2] = {(char*)p->stage_in, (char*)p->stage_in + cin};
    char* out_st[2] = {(char*)p->stage_out, (char*)p->stage_out + cout};
    char* hin[2] = {(char*)p->host_in, (char*)p->host_in + cin};
    char* hout[2] = {(char*)p->host_out, (char*)p->host_out + cout};
    cudaEvent_t start;
    if (!cuda_ok(cudaEventCreateWithFlags(&start, cudaEventDisableTiming), "cudaEventCreate")) return false;
    cudaEventRecord(start, s);
    cudaStreamWaitEvent(p->s_h2d, start, 0);
    cudaStreamWaitEvent(p->s_d2h, start, 0);
    bool ok = true;
    long long k = 0, prev_b0 = -1, prev_cn = 0;
    auto drain = [&](long long b0, long long cn, int buf) {
        // chunk at b0 (bounce buffer buf): wait for its device-to-host copy, copy out
        if (!cuda_ok(cudaEventSynchronize(p->ev_d[buf]), "cudaEventSynchronize(copy-out)")) return false;
        const size_t nout = (size_t)((cn - 1) * odist + out_elems) * out_eb;
        host_copy((char*)y + (size_t)b0 * odist * out_eb, hout[buf], nout);
        return true;
    };
    for (long long b0 = 0; b0 < howmany && ok; b0 += chunk, ++k) {
        const long long cn = std::min(chunk, howmany - b0);
        const int buf = (int)(k & 1);
        const size_t nin = (size_t)((cn - 1) * idist + in_elems) * in_eb;
        const size_t nout = (size_t)((cn - 1) * odist + out_elems) * out_eb;
        // the bounce buffer's previous host-to-device copy (chunk k-2) has read it
        if (k >= 2) ok = cuda_ok(cudaEventSynchronize(p->ev_h[buf]), "cudaEventSynchronize(copy-in)");
        if (!ok) break;
        host_copy(hin[buf], (const char*)x + (size_t)b0 * idist * in_eb, nin);
        if (k >= 2) cudaStreamWaitEvent(p->s_h2d, p->ev_c[buf], 0);
        ok = cuda_ok(cudaMemcpyAsync(in_st[buf], hin[buf], nin, cudaMemcpyHostToDevice, p->s_h2d), "H2D copy");
        ok = ok && cuda_ok(cudaEventRecord(p->ev_h[buf], p->s_h2d), "cudaEventRecord");
        ok = ok && cuda_ok(cudaStreamWaitEvent(s, p->ev_h[buf], 0), "cudaStreamWaitEvent");
        if (ok && k >= 2) ok = cuda_ok(cudaStreamWaitEvent(s, p->ev_d[buf], 0), "cudaStreamWaitEvent");
        ok = ok && plan_execute(p, kind, in_st[buf], out_st[buf], cn, idist, odist, s, vjp) == 0;
        ok = ok && cuda_ok(cudaEventRecord(p->ev_c[buf], s), "cudaEventRecord");
        ok = ok && cuda_ok(cudaStreamWaitEvent(p->s_d2h, p->ev_c[buf], 0), "cudaStreamWaitEvent");
        // hout[buf] was drained (chunk k-2) before this iteration's copy-out is queued
        ok = ok && cuda_ok(cudaMemcpyAsync(hout[buf], out_st[buf], nout, cudaMemcpyDeviceToHost, p->s_d2h),
                           "D2H copy");
        ok = ok && cuda_ok(cudaEventRecord(p->ev_d[buf], p->s_d2h), "cudaEventRecord");
        // drain the previous chunk while this one is on the GPU
        if (ok && prev_b0 >= 0) ok = drain(prev_b0, prev_cn, buf ^ 1);
        prev_b0 = b0;
        prev_cn = cn;
    }
    if (ok && prev_b0 >= 0) ok = drain(prev_b0, prev_cn, (int)((k - 1) & 1));
    ok = cuda_ok(cudaStreamSynchronize(p->s_d2h), "stream synchronize") && ok;
    ok = cuda_ok(cudaStreamSynchronize(s), "stream synchronize") && ok;
    ok = cuda_ok(cudaStreamSynchronize(p->s_h2d), "stream synchronize") && ok;
    cudaEventDestroy(start);
    return ok;
}

bool run_pipelined(notorious_fft_plan* p, int kind, const void* x, void* y, long long howmany, long long idist,
                   long long odist, long long in_elems, long long out_elems, size_t in_eb, size_t out_eb, int vjp,
                   cudaStream_t s) {
    const size_t target = pipe_chunk_bytes();
    long long chunk = (long long)(target / std::max<size_t>((size_t)idist * in_eb, 1));
    if (chunk < 1) chunk = 1;
    if (chunk > howmany) chunk = howmany;
    const size_t cin = (size_t)((chunk - 1) * idist + in_elems) * in_eb;
    const size_t cout = (size_t)((chunk - 1) * odist + out_elems) * out_eb;
    if (!p->s_h2d) {
        if (!cuda_ok(cudaStreamCreateWithFlags(&p->s_h2d, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
        if (!cuda_ok(cudaStreamCreateWithFlags(&p->s_d2h, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
        for (int i = 0; i < 2; ++i) {
            if (!cuda_ok(cudaEventCreateWithFlags(&p->ev_h[i], cudaEventDisableTiming), "cudaEventCreate") ||
                !cuda_ok(cudaEventCreateWithFlags(&p->ev_c[i], cudaEventDisableTiming), "cudaEventCreate") ||
                !cuda_ok(cudaEventCreateWithFlags(&p->ev_d[i], cudaEventDisableTiming), "cudaEventCreate"))
                return false;
        }
    }
    if (!grow(&p->stage_in, &p->stage_in_bytes, 2 * cin)) return false;
    if (!grow(&p->stage_out, &p->stage_out_bytes, 2 * cout)) return false;
    char* in_st[2] = {(char*)p->stage_in, (char*)p->stage_in + cin};
    char* out_st[2] = {(char*)p->stage_out, (char*)p->stage_out + cout};
    // the staging buffers must not be rewritten while earlier work still reads them
    cudaEvent_t start;
    if (!cuda_ok(cudaEventCreateWithFlags(&start, cudaEventDisableTiming), "cudaEventCreate")) return false;
    cudaEventRecord(start, s);
    cudaStreamWaitEvent(p->s_h2d, start, 0);
    cudaStreamWaitEvent(p->s_d2h, start, 0);
    bool ok = true;
    long long k = 0;
    for (long long b0 = 0; b0 < howmany && ok; b0 += chunk, ++k) {
        const long long cn = std::min(chunk, howmany - b0);
        const int buf = (int)(k & 1);
        const size_t nin = (size_t)((cn - 1) * idist + in_elems) * in_eb;
        const size_t nout = (size_t)((cn - 1) * odist + out_elems) * out_eb;
        if (k >= 2) cudaStreamWaitEvent(p->s_h2d, p->ev_c[buf], 0);
        ok = cuda_ok(cudaMemcpyAsync(in_st[buf], (const char*)x + (size_t)b0 * idist * in_eb, nin,
                                     cudaMemcpyHostToDevice, p->s_h2d), "H2D copy");
        ok = ok && cuda_ok(cudaEventRecord(p->ev_h[buf], p->s_h2d), "cudaEventRecord");
        ok = ok && cuda_ok(cudaStreamWaitEvent(s, p->ev_h[buf], 0), "cudaStreamWaitEvent");
        if (ok && k >= 2) ok = cuda_ok(cudaStreamWaitEvent(s, p->ev_d[buf], 0), "cudaStreamWaitEvent");
        ok = ok && plan_execute(p, kind, in_st[buf], out_st[buf], cn, idist, odist, s, vjp) == 0;
        ok = ok && cuda_ok(cudaEventRecord(p->ev_c[buf], s), "cudaEventRecord");
        ok = ok && cuda_ok(cudaStreamWaitEvent(p->s_d2h, p->ev_c[buf], 0), "cudaStreamWaitEvent");
        ok = ok && cuda_ok(cudaMemcpyAsync((char*)y + (size_t)b0 * odist * out_eb, out_st[buf], nout,
                                           cudaMemcpyDeviceToHost, p->s_d2h), "D2H copy");
        ok = ok && cuda_ok(cudaEventRecord(p->ev_d[buf], p->s_d2h), "cudaEventRecord");
    }
    ok = cuda_ok(cudaStreamSynchronize(p->s_d2h), "stream synchronize") && ok;
    ok = cuda_ok(cudaStreamSynchronize(s), "stream synchronize") && ok;
    ok = cuda_ok(cudaStreamSynchronize(p->s_h2d), "stream synchronize") && ok;
    cudaEventDestroy(start);
    return ok;
}

// Calls on one plan share its device scratch.  Calls on one stream are
// ordered by that stream; a call on a different stream than the previous
// call first waits for the previous call's work (an event recorded at the end
// of every call).  Streams being captured into a CUDA graph are neither made
// to wait nor recorded: ordering a capture against earlier calls on other
// streams is the caller's (synchronize before capturing).
bool is_capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return st != cudaStreamCaptureStatusNone;
}

bool order_after_previous_call(notorious_fft_plan* p, cudaStream_t s, bool capturing) {
    if (capturing || !p->ev_pending || p->last_stream == s) return true;
    return cuda_ok(cudaStreamWaitEvent(s, p->ev_last, 0), "cudaStreamWaitEvent(previous call)");
}

void note_call(notorious_fft_plan* p, cudaStream_t s, bool capturing) {
    if (capturing) return;
    if (!p->ev_last && !cuda_ok(cudaEventCreateWithFlags(&p->ev_last, cudaEventDisableTiming), "cudaEventCreate"))
        return;
    if (cuda_ok(cudaEventRecord(p->ev_last, s), "cudaEventRecord(call end)")) {
        p->last_stream = s;
        p->ev_pending = true;
    }
}

bool is_device_ptr(const void* ptr) {
    cudaPointerAttributes attr;
    cudaError_t e = cudaPointerGetAttributes(&attr, ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

bool grow(void** buf, size_t* have, size_t need) {
    if (*have >= need && *buf) return true;
    if (*buf) cudaFree(*buf);
    *buf = nullptr;
    *have = 0;
    if (!cuda_ok(cudaMalloc(buf, need), "cudaMalloc(staging)")) return false;
    *have = need;
    return true;
}

// One public call: validate, stage host data if needed, execute, unstage.
void run(int kind, const void* x, void* y, const notorious_fft_aux* a, long long howmany, long long idist,
         long long odist, int vjp) {
    clear_error();
    if (!a || !a->plan) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "NULL aux");
        return;
    }
    if (!x || !y) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "NULL data pointer");
        return;
    }
    if (howmany <= 0) return;
    notorious_fft_plan* p = a->plan;
    std::lock_guard<std::mutex> lk(p->mu);
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != p->device && !cuda_ok(cudaSetDevice(p->device), "cudaSetDevice")) return;
    // element counts of one transform, as the vjp swaps the roles of in and out
    int kin = kind, kout = kind;
    if (vjp) {
        // the cotangent has the output's shape and the result the input's
        static const int swap_kind[10] = {K_DFT, K_INVDFT, K_INVREALDFT, K_REALDFT, K_DCT2,
                                          K_DST2, K_DCT3, K_DST3, K_DCT4, K_DST4};
        (void)swap_kind;
    }
    long long in_elems = vjp ? plan_out_elems(p, kind) : plan_in_elems(p, kin);
    long long out_elems = vjp ? plan_in_elems(p, kind) : plan_out_elems(p, kout);
    size_t in_eb = vjp ? out_elem_bytes(kind) : in_elem_bytes(kind);
    size_t out_eb = vjp ? in_elem_bytes(kind) : out_elem_bytes(kind);
    if (howmany == 1) {
        idist = in_elems;
        odist = out_elems;
    }
    if (idist < 0 || odist < 0) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "negative distance");
        return;
    }
    size_t in_bytes = (size_t)((howmany - 1) * idist + in_elems) * in_eb;
    size_t out_bytes = (size_t)((howmany - 1) * odist + out_elems) * out_eb;
    bool xd = is_device_ptr(x), yd = is_device_ptr(y);
    cudaStream_t s = t_stream;
    const void* din = x;
    void* dout = y;
    const bool capturing = is_capturing(s);
    // In place (x == y), chunk k's copy-out may land while chunk k+1 is copied
    // in, so the pipeline is only taken when every transform's output stays
    // inside its own input slot: equal byte distances and an output no longer
    // than that distance.  Other in-place layouts take the staged path below.
    const bool inplace_ok = x != y || ((size_t)idist * in_eb == (size_t)odist * out_eb &&
                                       (size_t)out_elems * out_eb <= (size_t)idist * in_eb &&
                                       (size_t)in_elems * in_eb <= (size_t)idist * in_eb);
    if (!order_after_previous_call(p, s, capturing)) goto done;
    if (!xd && !yd && howmany >= 4 && inplace_ok && is_pinned_host_ptr(x) && is_pinned_host_ptr(y)) {
        run_pipelined(p, kind, x, y, howmany, idist, odist, in_elems, out_elems, in_eb, out_eb, vjp, s);
        goto done;
    }
    if (!xd && !yd && howmany >= 4 && inplace_ok && !capturing && !is_pinned_host_ptr(x) && !is_pinned_host_ptr(y)) {
        run_pageable_pipelined(p, kind, x, y, howmany, idist, odist, in_elems, out_elems, in_eb, out_eb, vjp, s);
        goto done;
    }
    if (!xd) {
        if (!grow(&p->stage_in, &p->stage_in_bytes, in_bytes)) goto done;
        if (!cuda_ok(cudaMemcpyAsync(p->stage_in, x, in_bytes, cudaMemcpyHostToDevice, s), "H2D copy")) goto done;
        din = p->stage_in;
    } else {
        size_t al = in_eb == sizeof(cplx_t) ? sizeof(cplx_t) : sizeof(real_t);
        if (((uintptr_t)x) % al) {
            set_error(NOTORIOUS_FFT_ERR_INVALID, "device input pointer is not aligned to its element type");
            goto done;
        }
    }
    if (!yd) {
        if (!grow(&p->stage_out, &p->stage_out_bytes, out_bytes)) goto done;
        dout = p->stage_out;
        if (xd && x == y) {
            set_error(NOTORIOUS_FFT_ERR_INVALID, "in-place call mixing device and host memory");
            goto done;
        }
    } else {
        size_t al = out_eb == sizeof(cplx_t) ? sizeof(cplx_t) : sizeof(real_t);
        if (((uintptr_t)y) % al) {
            set_error(NOTORIOUS_FFT_ERR_INVALID, "device output pointer is not aligned to its element type");
            goto done;
        }
    }
    if (plan_execute(p, kind, din, dout, howmany, idist, odist, s, vjp) != 0) goto done;
    if (!yd) {
        if (!cuda_ok(cudaMemcpyAsync(y, dout, out_bytes, cudaMemcpyDeviceToHost, s), "D2H copy")) goto done;
    }
    if (!xd || !yd) cuda_ok(cudaStreamSynchronize(s), "stream synchronize");
done:
    note_call(p, s, capturing);
    if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
}

}  // namespace

extern "C" {

// ---- plans ------------------------------------------------------------------
notorious_fft_aux* notorious_fft_mkaux_dft(int d, int* Ns) { return make_aux(FAM_DFT, d, Ns); }
notorious_fft_aux* notorious_fft_mkaux_dft_1d(int N) { return make_aux(FAM_DFT, 1, &N); }
notorious_fft_aux* notorious_fft_mkaux_dft_2d(int N1, int N2) {
    int Ns[2] = {N1, N2};
    return make_aux(FAM_DFT, 2, Ns);
}
notorious_fft_aux* notorious_fft_mkaux_dft_3d(int N1, int N2, int N3) {
    int Ns[3] = {N1, N2, N3};
    return make_aux(FAM_DFT, 3, Ns);
}
notorious_fft_aux* notorious_fft_mkaux_realdft(int d, int* Ns) { return make_aux(FAM_REAL, d, Ns); }
notorious_fft_aux* notorious_fft_mkaux_realdft_1d(int N) { return make_aux(FAM_REAL, 1, &N); }
notorious_fft_aux* notorious_fft_mkaux_realdft_2d(int N1, int N2) {
    int Ns[2] = {N1, N2};
    return make_aux(FAM_REAL, 2, Ns);
}
notorious_fft_aux* notorious_fft_mkaux_realdft_3d(int N1, int N2, int N3) {
    int Ns[3] = {N1, N2, N3};
    return make_aux(FAM_REAL, 3, Ns);
}
notorious_fft_aux* notorious_fft_mkaux_t2t3(int d, int* Ns) { return make_aux(FAM_T2T3, d, Ns); }
notorious_fft_aux* notorious_fft_mkaux_t2t3_1d(int N) { return make_aux(FAM_T2T3, 1, &N); }
notorious_fft_aux* notorious_fft_mkaux_t2t3_2d(int N1, int N2) {
    int Ns[2] = {N1, N2};
    return make_aux(FAM_T2T3, 2, Ns);
}
notorious_fft_aux* notorious_fft_mkaux_t2t3_3d(int N1, int N2, int N3) {
    int Ns[3] = {N1, N2, N3};
    return make_aux(FAM_T2T3, 3, Ns);
}
notorious_fft_aux* notorious_fft_mkaux_t4(int d, int* Ns) { return make_aux(FAM_T4, d, Ns); }
notorious_fft_aux* notorious_fft_mkaux_t4_1d(int N) { return make_aux(FAM_T4, 1, &N); }
notorious_fft_aux* notorious_fft_mkaux_t4_2d(int N1, int N2) {
    int Ns[2] = {N1, N2};
    return make_aux(FAM_T4, 2, Ns);
}
notorious_fft_aux* notorious_fft_mkaux_t4_3d(int N1, int N2, int N3) {
    int Ns[3] = {N1, N2, N3};
    return make_aux(FAM_T4, 3, Ns);
}

void notorious_fft_free_aux(notorious_fft_aux* a) {
    if (!a) return;
    if (a->plan) plan_destroy(a->plan);
    free(a);
}

// ---- transforms -------------------------------------------------------------
void notorious_fft_dft(notorious_fft_cmpl* x, notorious_fft_cmpl* y, const notorious_fft_aux* a) { run(K_DFT, x, y, a, 1, 0, 0, 0); }
void notorious_fft_invdft(notorious_fft_cmpl* x, notorious_fft_cmpl* y, const notorious_fft_aux* a) { run(K_INVDFT, x, y, a, 1, 0, 0, 0); }
void notorious_fft_realdft(notorious_fft_real* x, notorious_fft_cmpl* z, const notorious_fft_aux* a) { run(K_REALDFT, x, z, a, 1, 0, 0, 0); }
void notorious_fft_invrealdft(notorious_fft_cmpl* z, notorious_fft_real* y, const notorious_fft_aux* a) { run(K_INVREALDFT, z, y, a, 1, 0, 0, 0); }
void notorious_fft_dct2(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a) { run(K_DCT2, x, y, a, 1, 0, 0, 0); }
void notorious_fft_dst2(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a) { run(K_DST2, x, y, a, 1, 0, 0, 0); }
void notorious_fft_dct3(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a) { run(K_DCT3, x, y, a, 1, 0, 0, 0); }
void notorious_fft_dst3(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a) { run(K_DST3, x, y, a, 1, 0, 0, 0); }
void notorious_fft_dct4(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a) { run(K_DCT4, x, y, a, 1, 0, 0, 0); }
void notorious_fft_dst4(notorious_fft_real* x, notorious_fft_real* y, const notorious_fft_aux* a) { run(K_DST4, x, y, a, 1, 0, 0, 0); }

void notorious_fft_execute_batched(int kind, void* x, void* y, const notorious_fft_aux* a, int howmany, ptrdiff_t idist,
                                   ptrdiff_t odist) {
    if (kind < 0 || kind > 9) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "unknown transform kind %d", kind);
        return;
    }
    run(kind, x, y, a, howmany, idist, odist, 0);
}

#define NFFT_BATCHED(name, K, TI, TO)                                                                               \
    void notorious_fft_##name##_batched(TI* x, TO* y, const notorious_fft_aux* a, int howmany, ptrdiff_t idist,    \
                                        ptrdiff_t odist) {                                                          \
        run(K, x, y, a, howmany, idist, odist, 0);                                                                  \
    }
NFFT_BATCHED(dft, K_DFT, notorious_fft_cmpl, notorious_fft_cmpl)
NFFT_BATCHED(invdft, K_INVDFT, notorious_fft_cmpl, notorious_fft_cmpl)
NFFT_BATCHED(realdft, K_REALDFT, notorious_fft_real, notorious_fft_cmpl)
NFFT_BATCHED(invrealdft, K_INVREALDFT, notorious_fft_cmpl, notorious_fft_real)
NFFT_BATCHED(dct2, K_DCT2, notorious_fft_real, notorious_fft_real)
NFFT_BATCHED(dst2, K_DST2, notorious_fft_real, notorious_fft_real)
NFFT_BATCHED(dct3, K_DCT3, notorious_fft_real, notorious_fft_real)
NFFT_BATCHED(dst3, K_DST3, notorious_fft_real, notorious_fft_real)
NFFT_BATCHED(dct4, K_DCT4, notorious_fft_real, notorious_fft_real)
NFFT_BATCHED(dst4, K_DST4, notorious_fft_real, notorious_fft_real)
#undef NFFT_BATCHED

// ---- adjoints ---------------------------------------------------------------
void notorious_fft_dft_vjp(notorious_fft_cmpl* g, notorious_fft_cmpl* gx, const notorious_fft_aux* a) { run(K_DFT, g, gx, a, 1, 0, 0, 1); }
void notorious_fft_invdft_vjp(notorious_fft_cmpl* g, notorious_fft_cmpl* gx, const notorious_fft_aux* a) { run(K_INVDFT, g, gx, a, 1, 0, 0, 1); }
void notorious_fft_realdft_vjp(notorious_fft_cmpl* g, notorious_fft_real* gx, const notorious_fft_aux* a) { run(K_REALDFT, g, gx, a, 1, 0, 0, 1); }
void notorious_fft_invrealdft_vjp(notorious_fft_real* g, notorious_fft_cmpl* gz, const notorious_fft_aux* a) { run(K_INVREALDFT, g, gz, a, 1, 0, 0, 1); }
void notorious_fft_dct2_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a) { run(K_DCT2, g, gx, a, 1, 0, 0, 1); }
void notorious_fft_dst2_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a) { run(K_DST2, g, gx, a, 1, 0, 0, 1); }
void notorious_fft_dct3_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a) { run(K_DCT3, g, gx, a, 1, 0, 0, 1); }
void notorious_fft_dst3_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a) { run(K_DST3, g, gx, a, 1, 0, 0, 1); }
void notorious_fft_dct4_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a) { run(K_DCT4, g, gx, a, 1, 0, 0, 1); }
void notorious_fft_dst4_vjp(notorious_fft_real* g, notorious_fft_real* gx, const notorious_fft_aux* a) { run(K_DST4, g, gx, a, 1, 0, 0, 1); }

void notorious_fft_vjp_batched(int kind, void* g, void* gx, const notorious_fft_aux* a, int howmany, ptrdiff_t idist,
                               ptrdiff_t odist) {
    if (kind < 0 || kind > 9) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "unknown transform kind %d", kind);
        return;
    }
    run(kind, g, gx, a, howmany, idist, odist, 1);
}

// ---- errors / streams / info -------------------------------------------------
int notorious_fft_last_error(void) { return last_error(); }
const char* notorious_fft_last_error_string(void) { return last_error_string(); }
void notorious_fft_clear_error(void) { clear_error(); }

void notorious_fft_set_stream(void* stream) { t_stream = (cudaStream_t)stream; }
void* notorious_fft_get_stream(void) { return (void*)t_stream; }
int notorious_fft_synchronize(void) {
    clear_error();
    if (!cuda_ok(cudaStreamSynchronize(t_stream), "cudaStreamSynchronize")) return last_error();
    if (const unsigned st = tc_umma_take_status()) {
        set_error(NOTORIOUS_FFT_ERR_CUDA, "tensor-core pass: wait %u gave up (results incomplete)", st);
        return last_error();
    }
    return 0;
}

int notorious_fft_set_form(notorious_fft_aux* a, int form) {
    clear_error();
    if (!a || !a->plan) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "NULL aux");
        return NOTORIOUS_FFT_ERR_INVALID;
    }
    if (form == NOTORIOUS_FFT_FORM_PLAIN) {
        a->plan->form = form;
        return 0;
    }
    if (form == NOTORIOUS_FFT_FORM_SPLIT_TC) {
        if (sizeof(real_t) != 4) {
            set_error(NOTORIOUS_FFT_ERR_UNSUPPORTED, "the split tensor-core form is a float-library form");
            return NOTORIOUS_FFT_ERR_UNSUPPORTED;
        }
        a->plan->form = form;
        return 0;
    }
    set_error(NOTORIOUS_FFT_ERR_INVALID, "unknown form %d", form);
    return NOTORIOUS_FFT_ERR_INVALID;
}
int notorious_fft_get_form(const notorious_fft_aux* a) { return (a && a->plan) ? a->plan->form : -1; }

// ---- ragged batches (persistent queue) -----------------------------------------
notorious_fft_batch* notorious_fft_mkbatch(int count, const int* kinds, const int* Ns, const long long* in_offsets,
                                           const long long* out_offsets) {
    clear_error();
    return batch_create_default(count, kinds, Ns, in_offsets, out_offsets);
}
long long notorious_fft_batch_in_size(const notorious_fft_batch* b) { return b ? batch_in_reals(b) : 0; }
long long notorious_fft_batch_out_size(const notorious_fft_batch* b) { return b ? batch_out_reals(b) : 0; }

int notorious_fft_batch_execute(notorious_fft_batch* b, const notorious_fft_real* in, notorious_fft_real* out) {
    clear_error();
    if (!b || ((!in || !out) && batch_in_reals(b) > 0)) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "NULL batch or buffer");
        return NOTORIOUS_FFT_ERR_INVALID;
    }
    if (batch_in_reals(b) == 0) return 0;
    const bool din = is_device_ptr(in), dout = is_device_ptr(out);
    if (din != dout) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "batch input and output must both be device or both be host memory");
        return NOTORIOUS_FFT_ERR_INVALID;
    }
    return din ? batch_run(b, in, out, t_stream) : batch_run_host(b, in, out, t_stream);
}
int notorious_fft_batch_status(notorious_fft_batch* b) {
    clear_error();
    if (!b) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "NULL batch");
        return NOTORIOUS_FFT_ERR_INVALID;
    }
    return batch_status(b);
}
int notorious_fft_batch_set_graph(notorious_fft_batch* b, int enable) {
    if (!b) return NOTORIOUS_FFT_ERR_INVALID;
    batch_set_graph(b, enable);
    return 0;
}
int notorious_fft_batch_info(const notorious_fft_batch* b, long long* items, long long* tiles, long long* scratch_bytes,
                             int* ctas) {
    if (!b) return NOTORIOUS_FFT_ERR_INVALID;
    batch_info(b, items, tiles, scratch_bytes, ctas);
    return 0;
}
void notorious_fft_free_batch(notorious_fft_batch* b) { batch_destroy(b); }
int notorious_fft_batch_debug_withhold(notorious_fft_batch* b, long long spin_limit) {
    if (!b) return NOTORIOUS_FFT_ERR_INVALID;
    batch_withhold(b, spin_limit);
    return 0;
}

int notorious_fft_autotune(int kind, int N) {
    clear_error();
    if (!current_ctx()) return last_error();
    return autotune(kind, N, t_stream);
}
int notorious_fft_tune_lookup(int kind, int N, int* log2_radices, int max_passes) {
    clear_error();
    if (!log2_radices || max_passes < 1) return 0;
    return tune_lookup(kind, N, log2_radices, max_passes);
}

int notorious_fft_tune_lookup_plan(int kind, int N, int* log2_radices, int max_passes, int* log2_threads) {
    clear_error();
    int scratch[4];
    if (!log2_radices || max_passes < 1) {
        log2_radices = scratch;
        max_passes = 4;
    }
    return tune_lookup_plan(kind, N, log2_radices, max_passes, log2_threads);
}

int notorious_fft_aux_schedule(const notorious_fft_aux* a, int axis, int* log2_radices, int max_passes,
                               int* log2_threads) {
    clear_error();
    if (!a || !a->plan) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "NULL aux");
        return -1;
    }
    const notorious_fft_plan* p = a->plan;
    const int d = (int)p->axes.size();
    if (axis < 0) axis += d;
    if (axis < 0 || axis >= d) {
        set_error(NOTORIOUS_FFT_ERR_INVALID, "axis %d out of range for a %d-dimensional aux", axis, d);
        return -1;
    }
    const AxisPlan& ax = p->axes[axis];
    if (!ax.pow2) return 0;
    const FftSchedule& sch = ax.fft_contig;
    for (int i = 0; i < sch.npass && log2_radices && i < max_passes; ++i) log2_radices[i] = sch.plog[i];
    if (log2_threads) *log2_threads = sch.logt;
    return sch.npass;
}

int notorious_fft_real_size(void) { return (int)sizeof(real_t); }
long long notorious_fft_launch_count(void) { return launch_count(); }
const char* notorious_fft_version(void) { return "notorious-fft-b200 0.1 (sm_100a)"; }

}  // extern "C"

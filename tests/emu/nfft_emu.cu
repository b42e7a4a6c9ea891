// nfft_emu.cu -- TEST INFRASTRUCTURE ONLY: a CPU emulation build of the
// library's host logic, used by the CPU test suite (tests/test_emulator.py).
//
// It compiles the library's planner and C ABI (notorious-fft_b200/csrc/
// nfft_plan.cu, nfft_api.cu) against an emulated CUDA runtime (host memory,
// synchronous copies) and replaces every kernel launch with a host loop that
// runs the kernel's own per-thread phase functions (nfft_pass.cuh: line_setup,
// load_slot, substage_read/write, mid_slot, store_slot, paired_slot,
// unpack_item) for every thread of every tile.  Every global and shared
// memory access is bounds-checked against live allocations; a violation
// aborts the process with the offending address.  Fresh allocations are
// filled with NaN so reads of unwritten scratch show up in the results.
//
// This build is never shipped: the product libraries have no CPU path.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <type_traits>
#include <mutex>
#include <vector>

// ---------------------------------------------------------------------------
// emulated runtime
// ---------------------------------------------------------------------------
namespace emu {
static std::mutex mu;
static std::map<uintptr_t, size_t> allocs;   // base -> bytes
static std::map<uintptr_t, size_t> host_ok;  // user host buffers registered by the tests
static long long n_checks = 0;

static bool inside(const std::map<uintptr_t, size_t>& m, uintptr_t p, size_t b) {
    auto it = m.upper_bound(p);
    if (it == m.begin()) return false;
    --it;
    return p >= it->first && p + b <= it->first + it->second;
}

cudaError_t Malloc(void** p, size_t bytes) {
    // 256-byte aligned, like cudaMalloc (tensor copies and L2 discards rely on it)
    void* q = aligned_alloc(256, (bytes + 255) / 256 * 256 + (bytes ? 0 : 256));
    if (!q) return cudaErrorMemoryAllocation;
    // NaN fill: scratch read before it is written poisons the result
    double nan = NAN;
    for (size_t i = 0; i + sizeof(double) <= bytes; i += sizeof(double)) memcpy((char*)q + i, &nan, sizeof(double));
    std::lock_guard<std::mutex> lk(mu);
    allocs[(uintptr_t)q] = bytes;
    *p = q;
    return cudaSuccess;
}
cudaError_t Free(void* p) {
    if (!p) return cudaSuccess;
    std::lock_guard<std::mutex> lk(mu);
    auto it = allocs.find((uintptr_t)p);
    if (it == allocs.end()) {
        fprintf(stderr, "nfft_emu: cudaFree of unknown pointer %p\n", p);
        abort();
    }
    allocs.erase(it);
    free(p);
    return cudaSuccess;
}
static bool is_dev(const void* p, size_t b) {
    std::lock_guard<std::mutex> lk(mu);
    return inside(allocs, (uintptr_t)p, b);
}
static void check_range(const void* p, size_t b, const char* what) {
    std::lock_guard<std::mutex> lk(mu);
    if (!inside(allocs, (uintptr_t)p, b) && !inside(host_ok, (uintptr_t)p, b)) {
        fprintf(stderr, "nfft_emu: %s out of bounds: %p + %zu\n", what, p, b);
        abort();
    }
}
cudaError_t MemcpyAsync(void* d, const void* s, size_t b, cudaMemcpyKind, cudaStream_t = 0) {
    check_range(d, b, "memcpy dst");
    check_range(s, b, "memcpy src");
    memmove(d, s, b);
    return cudaSuccess;
}
// Synchronous copy between library-internal host memory and device memory:
// only the device side is checked.
cudaError_t Memcpy(void* d, const void* s, size_t b, cudaMemcpyKind k) {
    if (k != cudaMemcpyHostToDevice) check_range(s, b, "memcpy src");
    if (k != cudaMemcpyDeviceToHost) check_range(d, b, "memcpy dst");
    memmove(d, s, b);
    return cudaSuccess;
}
cudaError_t MemsetAsync(void* d, int v, size_t b, cudaStream_t = 0) {
    check_range(d, b, "memset");
    memset(d, v, b);
    return cudaSuccess;
}
cudaError_t DriverGetVersion(int* v) {
    *v = 0;
    return cudaSuccess;
}
cudaError_t Memcpy2DAsync(void* d, size_t dp, const void* s, size_t sp, size_t w, size_t h, cudaMemcpyKind k,
                          cudaStream_t st = 0) {
    for (size_t r = 0; r < h; ++r) MemcpyAsync((char*)d + r * dp, (const char*)s + r * sp, w, k, st);
    return cudaSuccess;
}
cudaError_t Ok(...) { return cudaSuccess; }
cudaError_t GetDevice(int* d) {
    *d = 0;
    return cudaSuccess;
}
cudaError_t GetDeviceProperties(cudaDeviceProp* p, int) {
    memset(p, 0, sizeof *p);
    strcpy(p->name, "emulated sm_100");
    p->major = 10;
    p->minor = 0;
    p->multiProcessorCount = 148;
    p->l2CacheSize = 126 << 20;
    return cudaSuccess;
}
cudaError_t PointerGetAttributes(cudaPointerAttributes* a, const void* p) {
    memset(a, 0, sizeof *a);
    bool pinned;
    {
        std::lock_guard<std::mutex> lk(mu);
        pinned = inside(host_ok, (uintptr_t)p, 1);
    }
    // buffers registered by the tests stand for pinned host memory
    a->type = is_dev(p, 1) ? cudaMemoryTypeDevice : (pinned ? cudaMemoryTypeHost : cudaMemoryTypeUnregistered);
    return cudaSuccess;
}
// streams and events: the emulator runs everything synchronously
cudaError_t StreamCreateWithFlags(cudaStream_t* s, unsigned) {
    static int dummy[64];
    static int n = 0;
    *s = (cudaStream_t)&dummy[(n++) & 63];
    return cudaSuccess;
}
cudaError_t EventCreateWithFlags(cudaEvent_t* e, unsigned) {
    static int dummy[256];
    static int n = 0;
    *e = (cudaEvent_t)&dummy[(n++) & 255];
    return cudaSuccess;
}
cudaError_t EventCreate(cudaEvent_t* e) { return EventCreateWithFlags(e, 0); }
cudaError_t EventElapsedTime(float* ms, cudaEvent_t, cudaEvent_t) {
    *ms = 1.0f;
    return cudaSuccess;
}
const char* ErrorString(cudaError_t) { return "emulated CUDA error"; }
}  // namespace emu

static int g_smem_elems = 0;
__host__ __device__ void nfft_emu_check(const void* p, size_t bytes, int write) {
#ifndef __CUDA_ARCH__
    emu::n_checks++;
    emu::check_range(p, bytes, write ? "global store" : "global load");
#endif
}
namespace nfft {
__host__ __device__ void nfft_emu_smem_check(int idx) {
#ifndef __CUDA_ARCH__
    if (idx < 0 || idx >= g_smem_elems) {
        fprintf(stderr, "nfft_emu: shared memory index %d outside [0, %d)\n", idx, g_smem_elems);
        abort();
    }
#endif
}
}  // namespace nfft

#define cudaMalloc(p, b) emu::Malloc((void**)(p), (b))
#define cudaFree emu::Free
#define cudaMemcpyAsync emu::MemcpyAsync
#define cudaMemcpy2DAsync emu::Memcpy2DAsync
#define cudaMemcpy emu::Memcpy
#define cudaMemsetAsync emu::MemsetAsync
#define cudaDriverGetVersion emu::DriverGetVersion
#define cudaEventCreate emu::EventCreate
#define cudaEventElapsedTime emu::EventElapsedTime
#define cudaStreamSynchronize(s) emu::Ok()
#define cudaDeviceSynchronize() emu::Ok()
#define cudaSetDevice(d) emu::Ok()
#define cudaGetDevice emu::GetDevice
#undef cudaGetDeviceProperties
#define cudaGetDeviceProperties emu::GetDeviceProperties
#define cudaPointerGetAttributes emu::PointerGetAttributes
#define cudaGetLastError() emu::Ok()
#define cudaGetErrorString emu::ErrorString
#define cudaStreamCreateWithFlags emu::StreamCreateWithFlags
#define cudaEventCreateWithFlags emu::EventCreateWithFlags
#define cudaEventRecord(e, s) emu::Ok()
#define cudaStreamWaitEvent(s, e, f) emu::Ok()
#define cudaEventDestroy(e) emu::Ok()
#define cudaStreamDestroy(s) emu::Ok()
#define cudaStreamIsCapturing(s, st) (*(st) = cudaStreamCaptureStatusNone, emu::Ok())

#include "../../notorious-fft_b200/csrc/nfft_plan.cu"
#include "../../notorious-fft_b200/csrc/nfft_api.cu"
#include "../../notorious-fft_b200/csrc/nfft_queue_build.cu"
#include "../../notorious-fft_b200/csrc/nfft_lean.cuh"
#include "../../notorious-fft_b200/csrc/nfft_lean_list.h"
#include "../../notorious-fft_b200/csrc/nfft_tc.cuh"
#include "../../notorious-fft_b200/csrc/nfft_tc_lean.cuh"
#include "../../notorious-fft_b200/csrc/nfft_umma.cuh"
#include "../../notorious-fft_b200/csrc/nfft_queue.h"

// ---------------------------------------------------------------------------
// emulated launches: the kernels' phase functions for every thread
// ---------------------------------------------------------------------------
namespace nfft {

template <int LOG_TILE, int LOAD, int STORE>
static void emu_pass(const PassArgs& a, long long t0, long long t1) {
    using T = real_t;
    using V = C2<T>;
    constexpr int THREADS = (1 << LOG_TILE) / 16;
    const TwTables<T>* tw = (const TwTables<T>*)a.tw;
    const int logE = a.logR + a.logJ, J = 1 << a.logJ, E = 1 << logE;
    g_smem_elems = (int)pass_smem_elems<T>(LOG_TILE);
    std::vector<V> sm(g_smem_elems);
    std::vector<long long> lin(MAX_J), lout(MAX_J), lj(MAX_J);
    std::vector<V> regs((size_t)THREADS * 16);
    TileLines tl{lin.data(), lout.data(), lj.data()};
    if (J > MAX_J || E > (1 << LOG_TILE)) {
        fprintf(stderr, "nfft_emu: tile of %d lines x 2^%d exceeds the kernel limits\n", J, a.logR);
        abort();
    }
    auto fft = [&]() {
        int lns = 0;
        for (int s = 0; s < a.nsub; ++s) {
            int lr = a.sublog[s];
            for (int t = 0; t < THREADS; ++t) {
                V* v = &regs[(size_t)t * 16];
                switch (lr) {
                case 4: substage_read<T, THREADS, 16, 4>(sm.data(), v, a.logR, logE, t); break;
                case 3: substage_read<T, THREADS, 8, 3>(sm.data(), v, a.logR, logE, t); break;
                case 2: substage_read<T, THREADS, 4, 2>(sm.data(), v, a.logR, logE, t); break;
                default: substage_read<T, THREADS, 2, 1>(sm.data(), v, a.logR, logE, t); break;
                }
            }
            for (int t = 0; t < THREADS; ++t) {
                V* v = &regs[(size_t)t * 16];
                switch (lr) {
                case 4: substage_write<T, THREADS, 16, 4>(sm.data(), v, tw, a.logR, logE, lns, t); break;
                case 3: substage_write<T, THREADS, 8, 3>(sm.data(), v, tw, a.logR, logE, lns, t); break;
                case 2: substage_write<T, THREADS, 4, 2>(sm.data(), v, tw, a.logR, logE, lns, t); break;
                default: substage_write<T, THREADS, 2, 1>(sm.data(), v, tw, a.logR, logE, lns, t); break;
                }
            }
            lns += lr;
        }
    };
    for (long long tile = t0; tile < t1; ++tile) {
        const long long line0 = tile << a.logJ;
        if (line0 >= a.nlines) continue;
        for (auto& x : sm) x = mkc((T)NAN, (T)NAN);
        for (int l = 0; l < J; ++l) line_setup(a, line0 + l, l, tl);
        for (int t = 0; t < THREADS; ++t)
            for (int it = 0; it < 16; ++it) {
                int e = t + it * THREADS;
                if (e >= E) break;
                load_slot_commit<T>(a, tw, sm.data(), tl, e, load_slot_value<T, LOAD>(a, tw, tl, e));
            }
        fft();
        if (a.mid) {
            for (int e = 0; e < E; ++e) mid_slot<T>(a, sm.data(), tl, e);
            fft();
        }
        if constexpr (STORE == ST_R || STORE == ST_T2) {
            const int items = paired_items(a);
            for (int w = 0; w < items; ++w) paired_slot<T, STORE>(a, tw, sm.data(), tl, w);
        } else {
            for (int e = 0; e < E; ++e) store_slot<T, STORE>(a, tw, sm.data(), tl, e);
        }
    }
}

using EmuFn = void (*)(const PassArgs&, long long, long long);

#define NFFT_PAIRS(X) \
    X(LD_C, ST_C) X(LD_C, ST_R) X(LD_C, ST_T2) X(LD_C, ST_T3) X(LD_C, ST_T4) X(LD_C, ST_BLUE) X(LD_T2, ST_C) \
    X(LD_T2, ST_T2) X(LD_T3, ST_C) X(LD_T3, ST_T3) X(LD_IR, ST_C) X(LD_T4, ST_C) X(LD_T4, ST_T4)          \
    X(LD_BLUE, ST_C) X(LD_BLUE, ST_BLUE) X(LD_R2C, ST_C) X(LD_R2C, ST_R) X(LD_C, ST_C2R) X(LD_IR, ST_C2R)   \
    X(LD_FILT, ST_C)

static long long g_launches = 0;

bool launch_pass(const PassArgs& a, int ld, int st, int log_tile, long long ntiles, cudaStream_t) {
    static EmuFn t12[NUM_LOAD_OPS][NUM_STORE_OPS] = {}, t13[NUM_LOAD_OPS][NUM_STORE_OPS] = {};
    static bool filled = false;
    if (!filled) {
#define X(L, S) t12[L][S] = emu_pass<12, L, S>; t13[L][S] = emu_pass<13, L, S>;
        NFFT_PAIRS(X)
#undef X
        filled = true;
    }
    EmuFn f = (log_tile == 13 ? t13 : t12)[ld][st];
    if (!f || (log_tile != 12 && log_tile != 13)) {
        set_error(6, "no pass kernel for load op %d / store op %d / tile %d", ld, st, log_tile);
        return false;
    }
    g_launches++;
    f(a, 0, ntiles);
    return true;
}

bool launch_unpack(const PassArgs& a, int st, const cplx_t* Z, long long zdist, long long nlines, cudaStream_t) {
    const TwTables<real_t>* tw = (const TwTables<real_t>*)a.tw;
    long long M = a.N / 2, per = M >= 2 ? M / 2 : 1;
    g_launches++;
    for (long long w = 0; w < per * nlines; ++w) {
        if (st == ST_R) unpack_item<real_t, ST_R>(a, tw, Z, zdist, w);
        else unpack_item<real_t, ST_T2>(a, tw, Z, zdist, w);
    }
    return true;
}

bool launch_tiny(const real_t* x, real_t* y, long long howmany, long long inner, long long idist, long long odist,
                 int in_cplx, int out_cplx, double factor, cudaStream_t) {
    g_launches++;
    for (long long b = 0; b < howmany; ++b)
        for (long long i = 0; i < inner; ++i) {
            real_t v = NFFT_GLD(&x[(b * idist + i) * (in_cplx ? 2 : 1)]);
            real_t r = (real_t)(factor * (double)v);
            if (out_cplx) {
                NFFT_GST(&y[(b * odist + i) * 2], r);
                NFFT_GST(&y[(b * odist + i) * 2 + 1], (real_t)0);
            } else {
                NFFT_GST(&y[b * odist + i], r);
            }
        }
    return true;
}

bool launch_init_tables(TwTables<real_t>* tw, cudaStream_t) {
    for (int level = 0; level < 3; ++level)
        for (int m = 0; m < TW_SIZE; ++m) {
            long double frac = ldexpl((long double)m, 1 - TW_BITS * (level + 1));
            long double ang = 3.141592653589793238462643383279502884L * frac;
            tw->t[level][m] = mkc((real_t)cosl(ang), (real_t)-sinl(ang));
        }
    return true;
}

bool launch_chirp(cplx_t* chirp, cplx_t* bwrap, long long n, long long M, cudaStream_t) {
    for (long long k = 0; k < M; ++k) {
        if (k < n) {
            unsigned long long r = ((unsigned long long)k * (unsigned long long)k) % (unsigned long long)(2 * n);
            long double ang = 3.141592653589793238462643383279502884L * (long double)r / (long double)n;
            real_t c = (real_t)cosl(ang), s = (real_t)sinl(ang);
            chirp[k] = mkc(c, (real_t)-s);
            bwrap[k] = mkc(c, s);
            if (k > 0) bwrap[M - k] = mkc(c, s);
        } else if (k <= M - n) {
            bwrap[k] = mkc((real_t)0, (real_t)0);
        }
    }
    return true;
}

bool set_kernel_attributes() { return true; }

// ---- specialized (lean) pass kernels: the kernel body of nfft_lean.cuh, with
// every phase run for all threads before the next (its __syncthreads points)
template <int LOGR, int LOGT, bool CI, bool CO, int LD, int ST>
static void emu_lean(const PassArgs& a, long long t0, long long t1) {
    using T = real_t;
    using V = C2<T>;
    using Lt = Lean<T, LOGR, LOGT, CI, CO, LD, ST>;
    const TwTables<T>* tw = (const TwTables<T>*)a.tw;
    constexpr int TH = Lt::THREADS;
    g_smem_elems = Lt::SMEM_ELEMS;
    std::vector<V> sm(Lt::SMEM_ELEMS);
    std::vector<LeanLine> lines(Lt::J);
    std::vector<V> regs((size_t)TH * 16);
    std::vector<int> ls((size_t)TH * 16), is((size_t)TH * 16);
    auto middle = [&](auto Sc) {
        constexpr int S = decltype(Sc)::value;
        constexpr int RHO = 1 << LeanSched<LOGR>::lr[S];
        for (int t = 0; t < TH; ++t)
            for (int q = 0; q < 16 / RHO; ++q)
                Lt::template read<S, Lt::COLL>(sm.data(), t, q, &regs[t * 16 + q * RHO], ls[t * 16 + q], is[t * 16 + q]);
        for (int t = 0; t < TH; ++t)
            for (int q = 0; q < 16 / RHO; ++q) {
                Lt::template twiddle_dft<S>(tw, is[t * 16 + q], &regs[t * 16 + q * RHO]);
                Lt::template write_smem<S>(sm.data(), ls[t * 16 + q], is[t * 16 + q], &regs[t * 16 + q * RHO]);
            }
    };
    for (long long tile = t0; tile < t1; ++tile) {
        const long long line0 = tile << Lt::LOGJ;
        if (line0 >= a.nlines) continue;
        for (auto& x : sm) x = mkc((T)NAN, (T)NAN);
        const long long ns = 1ll << a.logNj, tpt = Lt::MIRROR ? (ns >> Lt::LOGJ) : 1;
        const long long tt = Lt::MIRROR ? tile - (tile / tpt) * tpt : 0;
        for (int t = 0; t < Lt::J; ++t) {
            long long tmp[3];
            TileLines tl{&tmp[0], &tmp[1], &tmp[2]};
            if constexpr (Lt::MIRROR) {
                if (tpt < 1) {
                    fprintf(stderr, "nfft_emu: mirror tile larger than the transform's lines\n");
                    abort();
                }
                const long long jj = mirror_line(tt, t, Lt::J, ns);
                if (jj < 0 || jj >= ns || mirror_local(tt, jj, Lt::J, ns) != t) {
                    fprintf(stderr, "nfft_emu: mirror line map of tile %lld line %d is not invertible\n", tt, t);
                    abort();
                }
                line_setup(a, (tile / tpt) * ns + jj, 0, tl);
            } else {
                line_setup(a, line0 + t, 0, tl);
            }
            lines[t] = LeanLine{tmp[0], tmp[1], tmp[2]};
        }
        if constexpr (Lt::PREPACK) {
            // the paired repack phase, then every thread's first-sub-stage reads
            // (a barrier in the kernel) before any sub-stage write
            for (int t = 0; t < TH; ++t) pair_prepack_thread<Lt, T, LD>(a, tw, sm.data(), lines.data(), t);
            std::vector<int> fl(TH), fi(TH);
            for (int t = 0; t < TH; ++t) Lt::first_smem(a, tw, sm.data(), lines.data(), t, &regs[t * 16], fl[t], fi[t]);
            for (int t = 0; t < TH; ++t) {
                if constexpr (Lt::NS == 1) Lt::template write_global<0>(a, tw, lines.data(), fl[t], fi[t], &regs[t * 16]);
                else Lt::template write_smem<0>(sm.data(), fl[t], fi[t], &regs[t * 16]);
            }
        } else
        for (int t = 0; t < TH; ++t) {
            int l, i;
            Lt::first(a, tw, lines.data(), t, &regs[t * 16], l, i);
            if constexpr (Lt::NS == 1) {
                if constexpr (Lt::PAIRED) Lt::template write_smem<0>(sm.data(), l, i, &regs[t * 16]);
                else Lt::template write_global<0>(a, tw, lines.data(), l, i, &regs[t * 16]);
            } else {
                Lt::template write_smem<0>(sm.data(), l, i, &regs[t * 16]);
            }
        }
        if constexpr (Lt::NS >= 2) {
            if constexpr (Lt::NS >= 3) middle(std::integral_constant<int, 1>{});
            if constexpr (Lt::NS >= 4) middle(std::integral_constant<int, 2>{});
            constexpr int S = Lt::NS - 1;
            constexpr int RHO = 1 << LeanSched<LOGR>::lr[S];
            for (int t = 0; t < TH; ++t)
                for (int q = 0; q < 16 / RHO; ++q)
                    Lt::template read<S, CO>(sm.data(), t, q, &regs[t * 16 + q * RHO], ls[t * 16 + q], is[t * 16 + q]);
            for (int t = 0; t < TH; ++t)
                for (int q = 0; q < 16 / RHO; ++q) {
                    Lt::template twiddle_dft<S>(tw, is[t * 16 + q], &regs[t * 16 + q * RHO]);
                    if constexpr (Lt::PAIRED)
                        Lt::template write_smem<S>(sm.data(), ls[t * 16 + q], is[t * 16 + q], &regs[t * 16 + q * RHO]);
                    else
                        Lt::template write_global<S>(a, tw, lines.data(), ls[t * 16 + q], is[t * 16 + q],
                                                     &regs[t * 16 + q * RHO]);
                }
        }
        if constexpr (Lt::MIRROR) {
            for (int t = 0; t < TH; ++t) mirror_unpack_thread<Lt, T, ST>(a, tw, sm.data(), lines.data(), tile, t);
        } else if constexpr (Lt::PAIRED) {
            for (int t = 0; t < TH; ++t) paired_unpack_thread<Lt, T, ST>(a, tw, sm.data(), lines.data(), t);
        }
    }
}

void note_launch() { g_launches++; }

// ---- split tensor-core pass: a host model of mma.sync.m16n8k16 (f16 x f16
// -> f32) from the fragment layout documented in nfft_tc.cuh, and the
// tc_substage phases for every lane of every warp.
static void emu_mma(const uint32_t (*a)[4], const uint32_t (*b)[2], float (*d)[4]) {
    float A[16][16], B[16][8];
    auto lo = [](uint32_t v) { return __half2float(__ushort_as_half((unsigned short)(v & 0xffff))); };
    auto hi = [](uint32_t v) { return __half2float(__ushort_as_half((unsigned short)(v >> 16))); };
    for (int lane = 0; lane < 32; ++lane) {
        int g = lane >> 2, t4 = lane & 3;
        for (int r = 0; r < 4; ++r) {
            int row = g + 8 * (r & 1), col = 2 * t4 + 8 * (r >> 1);
            A[row][col] = lo(a[lane][r]);
            A[row][col + 1] = hi(a[lane][r]);
        }
        for (int r = 0; r < 2; ++r) {
            int k = 2 * t4 + 8 * r;
            B[k][g] = lo(b[lane][r]);
            B[k + 1][g] = hi(b[lane][r]);
        }
    }
    for (int lane = 0; lane < 32; ++lane) {
        int g = lane >> 2, t4 = lane & 3;
        for (int r = 0; r < 4; ++r) {
            int row = g + 8 * (r >> 1), col = 2 * t4 + (r & 1);
            float acc = d[lane][r];
            for (int k = 0; k < 16; ++k) acc += A[row][k] * B[k][col];
            d[lane][r] = acc;
        }
    }
}

template <int THREADS>
static void emu_tc_substage(std::vector<C2<real_t>>& smv, const TwTables<real_t>* tw, int logR, int logE, int lns) {
    if constexpr (sizeof(real_t) == 4) {
        float2* sm = (float2*)smv.data();
        const TwTables<float>* twf = (const TwTables<float>*)tw;
        const int nbf = 1 << (logE - 4);
        const int W = THREADS / 32;
        std::vector<float2> x((size_t)W * 32 * 16);
        std::vector<int> ls((size_t)W * 32 * 4), is((size_t)W * 32 * 4);
        for (int w = 0; w < W; ++w)
            for (int lane = 0; lane < 32; ++lane)
                for (int q = 0; q < 4; ++q) {
                    float2* xp = &x[(((size_t)w * 32 + lane) * 4 + q) * 4];
                    int& l = ls[((size_t)w * 32 + lane) * 4 + q];
                    int& i = is[((size_t)w * 32 + lane) * 4 + q];
                    if (w * 32 + q * 8 + (lane >> 2) < nbf) tc_read(sm, logR, lns, w, q, lane, xp, l, i);
                    else { for (int p = 0; p < 4; ++p) xp[p] = make_float2(0.f, 0.f); i = 0; }
                }
        TcA A[32];
        for (int lane = 0; lane < 32; ++lane) tc_make_A(lane, A[lane]);
        for (int w = 0; w < W; ++w)
            for (int q = 0; q < 4; ++q) {
                if (w * 32 + q * 8 >= nbf) continue;
                float sc[32], amax[32];
                for (int lane = 0; lane < 32; ++lane) {
                    float2* xp = &x[(((size_t)w * 32 + lane) * 4 + q) * 4];
                    tc_twiddle(twf, lns, is[((size_t)w * 32 + lane) * 4 + q], lane, xp);
                    float m = 0.f;
                    for (int p = 0; p < 4; ++p) m = fmaxf(m, fmaxf(fabsf(xp[p].x), fabsf(xp[p].y)));
                    amax[lane] = m;
                }
                for (int lane = 0; lane < 32; ++lane) {
                    int b0 = lane & ~3;
                    float m = fmaxf(fmaxf(amax[b0], amax[b0 + 1]), fmaxf(amax[b0 + 2], amax[b0 + 3]));
                    sc[lane] = tc_scale(m);
                }
                uint32_t a_rl[32][4], a_rh[32][4], a_il[32][4], a_ih[32][4], a_nil[32][4], a_nih[32][4];
                uint32_t b_rh[32][2], b_rl[32][2], b_ih[32][2], b_il[32][2];
                for (int lane = 0; lane < 32; ++lane) {
                    float2* xp = &x[(((size_t)w * 32 + lane) * 4 + q) * 4];
                    for (int p = 0; p < 4; ++p) xp[p] = make_float2(xp[p].x * sc[lane], xp[p].y * sc[lane]);
                    TcB B;
                    tc_make_B(xp, B);
                    for (int r = 0; r < 4; ++r) {
                        a_rl[lane][r] = A[lane].rl[r]; a_rh[lane][r] = A[lane].rh[r];
                        a_il[lane][r] = A[lane].il[r]; a_ih[lane][r] = A[lane].ih[r];
                        a_nil[lane][r] = A[lane].nil[r]; a_nih[lane][r] = A[lane].nih[r];
                    }
                    for (int r = 0; r < 2; ++r) {
                        b_rh[lane][r] = B.rh[r]; b_rl[lane][r] = B.rl[r];
                        b_ih[lane][r] = B.ih[r]; b_il[lane][r] = B.il[r];
                    }
                }
                float yr[32][4] = {}, yi[32][4] = {}, cr[32][4] = {}, ci[32][4] = {};
                emu_mma(a_rl, b_rh, cr); emu_mma(a_il, b_rh, ci);
                emu_mma(a_rh, b_rh, yr); emu_mma(a_ih, b_rh, yi);
                emu_mma(a_rh, b_rl, cr); emu_mma(a_ih, b_rl, ci);
                emu_mma(a_nih, b_ih, yr); emu_mma(a_rh, b_ih, yi);
                emu_mma(a_nil, b_ih, cr); emu_mma(a_rl, b_ih, ci);
                emu_mma(a_nih, b_il, cr); emu_mma(a_rh, b_il, ci);
                for (int lane = 0; lane < 32; ++lane)
                    for (int r = 0; r < 4; ++r) { yr[lane][r] += cr[lane][r]; yi[lane][r] += ci[lane][r]; }
                for (int lane = 0; lane < 32; ++lane) {
                    int t4 = lane & 3;
                    float u0 = 1.0f / sc[8 * t4], u1 = 1.0f / sc[8 * t4 + 4];
                    float r_[4] = {yr[lane][0] * u0, yr[lane][1] * u1, yr[lane][2] * u0, yr[lane][3] * u1};
                    float i_[4] = {yi[lane][0] * u0, yi[lane][1] * u1, yi[lane][2] * u0, yi[lane][3] * u1};
                    if (w * 32 + q * 8 + 2 * t4 + 1 < nbf) tc_write(sm, logR, lns, w, q, lane, r_, i_);
                }
            }
    }
}

bool launch_tc_pass(const PassArgs& a, int log_tile, long long ntiles, cudaStream_t) {
    if (sizeof(real_t) != 4 || log_tile != 12) {
        set_error(6, "the split tensor-core form exists in the float library only");
        return false;
    }
    using T = real_t;
    using V = C2<T>;
    constexpr int LT = 12, THREADS = (1 << LT) / 16;
    g_launches++;
    const TwTables<T>* tw = (const TwTables<T>*)a.tw;
    const int logE = a.logR + a.logJ, J = 1 << a.logJ, E = 1 << logE;
    g_smem_elems = (int)pass_smem_elems<T>(LT);
    std::vector<V> sm(g_smem_elems);
    std::vector<long long> lin(MAX_J), lout(MAX_J), lj(MAX_J);
    std::vector<V> regs((size_t)THREADS * 16);
    TileLines tl{lin.data(), lout.data(), lj.data()};
    for (long long tile = 0; tile < ntiles; ++tile) {
        const long long line0 = tile << a.logJ;
        if (line0 >= a.nlines) continue;
        for (auto& x : sm) x = mkc((T)NAN, (T)NAN);
        for (int l = 0; l < J; ++l) line_setup(a, line0 + l, l, tl);
        for (int e = 0; e < E; ++e) load_slot_commit<T>(a, tw, sm.data(), tl, e, load_slot_value<T, LD_C>(a, tw, tl, e));
        int lns = 0;
        for (int s = 0; s < a.nsub; ++s) {
            int lr = a.sublog[s];
            if (lr == 4) {
                emu_tc_substage<THREADS>(sm, tw, a.logR, logE, lns);
            } else {
                for (int t = 0; t < THREADS; ++t) {
                    V* v = &regs[(size_t)t * 16];
                    if (lr == 3) substage_read<T, THREADS, 8, 3>(sm.data(), v, a.logR, logE, t);
                    else if (lr == 2) substage_read<T, THREADS, 4, 2>(sm.data(), v, a.logR, logE, t);
                    else substage_read<T, THREADS, 2, 1>(sm.data(), v, a.logR, logE, t);
                }
                for (int t = 0; t < THREADS; ++t) {
                    V* v = &regs[(size_t)t * 16];
                    if (lr == 3) substage_write<T, THREADS, 8, 3>(sm.data(), v, tw, a.logR, logE, lns, t);
                    else if (lr == 2) substage_write<T, THREADS, 4, 2>(sm.data(), v, tw, a.logR, logE, lns, t);
                    else substage_write<T, THREADS, 2, 1>(sm.data(), v, tw, a.logR, logE, lns, t);
                }
            }
            lns += lr;
        }
        for (int e = 0; e < E; ++e) store_slot<T, ST_C>(a, tw, sm.data(), tl, e);
    }
    return true;
}

// ---- radix-256 split tensor-core pass (nfft_tc_lean.cuh): the kernel's lane
// phases for the 32 lanes of a warp around host models of its collectives (the
// max reduction, and emu_mma for the FP16 hi / lo products).
static void emu_tcl_stage(const TcA* A, uint32_t (*xb)[2][2][2][2], float (*acc)[2][2][4]) {
    uint32_t a_h[32][4], a_l[32][4], b[32][2];
    float d[32][4];
    for (int nt = 0; nt < 2; ++nt)
        for (int mt = 0; mt < 2; ++mt) {
            for (int lane = 0; lane < 32; ++lane)
                for (int i = 0; i < 4; ++i) d[lane][i] = 0.0f;
            for (int kt = 0; kt < 2; ++kt) {
                for (int lane = 0; lane < 32; ++lane) {
                    const uint32_t* ah = mt == kt ? A[lane].rh : (mt == 0 ? A[lane].nih : A[lane].ih);
                    const uint32_t* al = mt == kt ? A[lane].rl : (mt == 0 ? A[lane].nil : A[lane].il);
                    for (int i = 0; i < 4; ++i) { a_h[lane][i] = ah[i]; a_l[lane][i] = al[i]; }
                }
                // Flo Xhi, Fhi Xlo, Fhi Xhi
                for (int term = 0; term < 3; ++term) {
                    const int hl = term == 1 ? 1 : 0;
                    for (int lane = 0; lane < 32; ++lane)
                        for (int r = 0; r < 2; ++r) b[lane][r] = xb[lane][kt][nt][hl][r];
                    emu_mma(term == 0 ? a_l : a_h, b, d);
                }
            }
            for (int lane = 0; lane < 32; ++lane)
                for (int i = 0; i < 4; ++i) acc[lane][mt][nt][i] = d[lane][i];
        }
}

// ---- radix-256 split tensor-core pass on tcgen05 (nfft_tc.cu, layout and
// index maps in nfft_umma.cuh): the kernel's phases for the 128 threads of a
// tile, in order, around host models of what the hardware does between them:
//  * the tensor copy in: box (8 lines x 256 rows) written row-major and
//    64-byte swizzled by address bits (bits 4-5 ^= bits 7-8);
//  * the products: D = Ah Bh + Al Bh + Ah Bl with every operand element read
//    through the descriptors' strides (stage 1 A and B K-major, stage 2 A
//    M-major), FP16 values, sums in double, rounded to float;
//  * tensor memory: D row t is thread t's;
//  * the tensor store out: the same box layouts read back.
static long long g_umma_launches = 0, g_umma_kind[3] = {0, 0, 0};
bool tc_umma_enabled() {
    const char* e = getenv("NOTORIOUS_FFT_TC_UMMA");
    return !e || atoi(e) != 0;
}
unsigned tc_umma_take_status() { return 0; }

static int emu_swz64(int o) { return o ^ (((o >> 7) & 3) << 4); }
static float emu_f16(const unsigned char* base, int off) {
    __half h;
    memcpy(&h, base + off, 2);
    return __half2float(h);
}
// D[m][n] = sum over the three hi / lo products, K = 32 (element offsets per the descriptors)
static void emu_umma(const unsigned char* ah, const unsigned char* al, const unsigned char* bh,
                     const unsigned char* bl, bool a_mmajor, float (*d)[32]) {
    auto aoff = [&](int m, int k) {
        return a_mmajor ? (m >> 3) * TCU_SBO + (k >> 3) * TCU_LBO + (k & 7) * 16 + (m & 7) * 2
                        : (m >> 3) * TCU_SBO + (k >> 3) * TCU_LBO + (m & 7) * 16 + (k & 7) * 2;
    };
    auto boff = [](int n, int k) { return (n >> 3) * TCU_BSBO + (k >> 3) * TCU_BLBO + (n & 7) * 16 + (k & 7) * 2; };
    for (int m = 0; m < 128; ++m)
        for (int n = 0; n < 32; ++n) {
            double acc = 0;
            for (int k = 0; k < 32; ++k) {
                const double xh = emu_f16(ah, aoff(m, k)), xl = emu_f16(al, aoff(m, k));
                const double fh = emu_f16(bh, boff(n, k)), fl = emu_f16(bl, boff(n, k));
                acc += xh * fh + xl * fh + xh * fl;
            }
            d[m][n] = (float)acc;
        }
}

bool try_launch_tc_umma(const PassArgs& a, int, cudaStream_t, bool& launched) {
    launched = false;
    if (sizeof(real_t) != 4 || !tc_umma_enabled()) return true;
    TcuArgs u;
    if (!tcu_shape(a, u)) return true;
    launched = true;
    g_launches++;
    g_umma_launches++;
    g_umma_kind[u.out_kind]++;
    const TwTables<float>* tw = (const TwTables<float>*)a.tw;
    // constants: the DFT matrix operands, the internal twiddles [k1][i]
    std::vector<unsigned char> Bh(TCU_BOP), Bl(TCU_BOP);
    for (int n = 0; n < 32; ++n)
        for (int c = 0; c < 32; ++c) {
            const float v = tcu_b_entry(tw, n, c);
            const __half h = __float2half_rn(v), lo = __float2half_rn(v - __half2float(h));
            const int off = tcu_b_off(n, c >> 1) + (c & 1) * 2;
            memcpy(&Bh[off], &h, 2);
            memcpy(&Bl[off], &lo, 2);
        }
    float2 twt[256];
    for (int q = 0; q < 256; ++q) {
        const int ii = q >> 4, k1 = q & 15;
        const C2<float> c = NFFT_GLD(&tw->t[0][(ii * k1 * 16) & (TW_SIZE - 1)]);
        twt[k1 * 16 + ii] = make_float2(c.x, c.y);
    }
    std::vector<unsigned char> stage(TCU_STAGE), A(2 * TCU_AOP);
    unsigned char* Ah = A.data();
    unsigned char* Al = A.data() + TCU_AOP;
    static float D1[128][32], D2[128][32];
    const float2* in = (const float2*)u.a.in;
    float2* out = (float2*)u.a.out;
    const float fscale = (float)a.scale;
    for (long long tile = 0; tile < u.ntiles; ++tile) {
        long long b;
        int j0;
        tcu_tile(u, tile, b, j0);
        for (auto& x : stage) x = 0xff;   // NaN bytes: a read of an unwritten slot shows
        for (auto& x : A) x = 0xff;
        for (int l = 0; l < TCU_J; ++l)
            for (int r = 0; r < 256; ++r) {
                const float2 v = NFFT_GLD(in + tcu_in_index(u, b, j0 + l, r));
                memcpy(&stage[emu_swz64((r * TCU_J + l) * 8)], &v, 8);
            }
        // stage 1: rows, pre-twiddles, per-line exponent, split
        static float2 X[128][16];
        float mx[TCU_J] = {0};
        int e1[TCU_J];
        for (int t = 0; t < 128; ++t) {
            int l, i;
            tcu_role_a(t, l, i);
            const int j = j0 + l;
            float2* x = X[t];
            for (int m = 0; m < 16; ++m) memcpy(&x[m], &stage[tcu_st_off(i + 16 * m, l)], 8);
            if (a.conj_in)
                for (int m = 0; m < 16; ++m) x[m].y = -x[m].y;
            const long long k = a.logNs > 0 ? (j & ((1ll << a.logNs) - 1)) : 0;
            if (k) {
                const C2<float> wb = twiddle<float>(tw, (uint64_t)i * (uint64_t)k, a.logNs + 8);
                const C2<float> s1 = twiddle<float>(tw, (uint64_t)k, a.logNs + 4);
                C2<float> pw[16];
                pw[0] = wb;
                pw[1] = tcu_cmul(wb, s1);
                const C2<float> s2 = tcu_cmul(s1, s1), s4 = tcu_cmul(s2, s2), s8 = tcu_cmul(s4, s4);
                pw[2] = tcu_cmul(wb, s2);
                pw[3] = tcu_cmul(pw[1], s2);
                for (int m = 4; m < 8; ++m) pw[m] = tcu_cmul(pw[m - 4], s4);
                for (int m = 8; m < 16; ++m) pw[m] = tcu_cmul(pw[m - 8], s8);
                for (int m = 0; m < 16; ++m) x[m] = tcu_cmul(x[m], pw[m]);
            }
            for (int m = 0; m < 16; ++m) mx[l] = fmaxf(mx[l], fmaxf(fabsf(x[m].x), fabsf(x[m].y)));
        }
        for (int l = 0; l < TCU_J; ++l) e1[l] = (mx[l] >= TCU_LO && mx[l] < TCU_HI) ? 0 : tcu_exp(mx[l]);
        for (int t = 0; t < 128; ++t) {
            int l, i;
            tcu_role_a(t, l, i);
            const float s_in = tcu_pow2(-e1[l]);
            for (int m = 0; m < 16; ++m) {
                const float re = X[t][m].x * s_in, im = X[t][m].y * s_in;
                const __half hr = __float2half_rn(re), hi = __float2half_rn(im);
                const __half lr = __float2half_rn(re - __half2float(hr)), li = __float2half_rn(im - __half2float(hi));
                const int off = tcu_a_off(t, m);
                memcpy(Ah + off, &hr, 2);
                memcpy(Ah + off + 2, &hi, 2);
                memcpy(Al + off, &lr, 2);
                memcpy(Al + off + 2, &li, 2);
            }
        }
        emu_umma(Ah, Al, Bh.data(), Bl.data(), false, D1);
        // stage-1 outputs: twiddle, M-major stage-2 operand
        for (auto& x : A) x = 0xff;
        for (int t = 0; t < 128; ++t) {
            int l, i;
            tcu_role_a(t, l, i);
            for (int q = 0; q < 16; ++q) {
                const float2 c = twt[q * 16 + i];
                const float re = D1[t][2 * q] * c.x - D1[t][2 * q + 1] * c.y;
                const float im = D1[t][2 * q] * c.y + D1[t][2 * q + 1] * c.x;
                const int off = tcu_at_off(tcu_row_b(u.out_kind, l, q & ~7), 2 * i) + (q & 7) * 2;
                const float pr[2] = {re, im};
                for (int c2 = 0; c2 < 2; ++c2) {
                    const __half h = __float2half_rn(pr[c2]);
                    const __half lo = __float2half_rn(pr[c2] - __half2float(h));
                    memcpy(Ah + off + 16 * c2, &h, 2);
                    memcpy(Al + off + 16 * c2, &lo, 2);
                }
            }
        }
        emu_umma(Ah, Al, Bh.data(), Bl.data(), true, D2);
        // stage 2: scale, stage in the A region, tensor store
        for (auto& x : A) x = 0xff;
        for (int t = 0; t < 128; ++t) {
            int l2, k1;
            tcu_role_b(u.out_kind, t, l2, k1);
            const float g = tcu_pow2(e1[l2]) * fscale;
            const float gi = a.conj_out ? -g : g;
            for (int q = 0; q < 16; ++q) {
                const float2 v = make_float2(D2[t][2 * q] * g, D2[t][2 * q + 1] * gi);
                const int off = u.out_kind == TCU_OUT_ROW ? l2 * 2048 + (k1 + 16 * q) * 8 : tcu_st_off(k1 + 16 * q, l2);
                memcpy(Ah + off, &v, 8);
            }
        }
        for (int l = 0; l < TCU_J; ++l)
            for (int p = 0; p < 256; ++p) {
                const int lin = u.out_kind == TCU_OUT_ROW ? (l * 256 + p) * 8 : emu_swz64((p * TCU_J + l) * 8);
                float2 v;
                memcpy(&v, Ah + lin, 8);
                NFFT_GST(out + tcu_out_index(u, b, j0 + l, p), v);
            }
    }
    return true;
}

bool tc_lean_enabled() {
    const char* e = getenv("NOTORIOUS_FFT_TC_LEAN");
    return !e || atoi(e) != 0;
}

bool launch_tc_lean(const PassArgs& a, int, cudaStream_t) {
    if (sizeof(real_t) != 4) {
        set_error(6, "the split tensor-core form exists in the float library only");
        return false;
    }
    if constexpr (sizeof(real_t) == 4) {
        using TL = TcLean<256>;
        g_launches++;
        const TwTables<float>* tw = (const TwTables<float>*)a.tw;
        std::vector<TL::Consts> c(32);
        TcA A[32];
        for (int lane = 0; lane < 32; ++lane) {
            TL::setup(tw, lane, c[lane]);
            A[lane] = c[lane].A;
        }
        g_smem_elems = TCL_SLOTS;
        std::vector<float2> sm(TCL_SLOTS);
        long long lin[TCL_J], lout[TCL_J], lj[TCL_J];
        TileLines tl{lin, lout, lj};
        std::vector<TL::LineRegs> st(32);
        uint32_t xb[32][2][2][2][2];
        float acc[32][2][2][4];
        const long long ntiles = (a.nlines + TCL_J - 1) >> TCL_LOGJ;
        for (long long tile = 0; tile < ntiles; ++tile) {
            for (auto& x : sm) x = make_float2(NAN, NAN);
            for (int l = 0; l < TCL_J; ++l) line_setup(a, (tile << TCL_LOGJ) + l, l, tl);
            for (int e = 0; e < TCL_SLOTS; ++e) {
                int l, r;
                tcl_walk(a.in_row, e, l, r);
                float2 v = make_float2(0.f, 0.f);
                if (lj[l] >= 0) v = NFFT_GLD((const float2*)a.in + tcl_in_off(a, lin[l], lj[l], r));
                sm[NFFT_SM(tcl_slot(r, l))] = v;
            }
            for (int l = 0; l < TCL_J; ++l) {
                if (lj[l] < 0) continue;
                float m = 0.f;
                for (int lane = 0; lane < 32; ++lane) m = fmaxf(m, TL::load(a, tw, sm.data(), l, lj[l], lane, st[lane]));
                for (int lane = 0; lane < 32; ++lane) {
                    TL::split1(m, st[lane]);
                    memcpy(xb[lane], st[lane].xb, sizeof xb[lane]);
                }
                emu_tcl_stage(A, xb, acc);
                for (int lane = 0; lane < 32; ++lane) {
                    memcpy(st[lane].acc, acc[lane], sizeof acc[lane]);
                    TL::mid(a, tw, c[lane], lj[l], lane, st[lane]);
                    memcpy(xb[lane], st[lane].xb, sizeof xb[lane]);
                }
                emu_tcl_stage(A, xb, acc);
                for (int lane = 0; lane < 32; ++lane) {
                    memcpy(st[lane].acc, acc[lane], sizeof acc[lane]);
                    TL::store(a, sm.data(), l, lane, st[lane]);
                }
            }
            for (int e = 0; e < TCL_SLOTS; ++e) {
                int l, r;
                tcl_walk(a.out_row, e, l, r);
                if (lj[l] < 0) continue;
                NFFT_GST((float2*)a.out + tcl_out_off(a, lout[l], lj[l], r), sm[NFFT_SM(tcl_slot(r, l))]);
            }
        }
    }
    return true;
}

using EmuLean = void (*)(const PassArgs&, long long, long long);
static std::map<unsigned, EmuLean>& emu_lean_table() {
    static std::map<unsigned, EmuLean> t = [] {
        std::map<unsigned, EmuLean> m;
#define X(R, T, CI, CO, LD, ST) m[lean_key(R, T, CI, CO, LD, ST)] = emu_lean<R, T, CI != 0, CO != 0, LD, ST>;
        NFFT_LEAN_ALL(X)
#undef X
        return m;
    }();
    return t;
}
bool lean_available(int logR, int logT, int ci, int co, int ld, int st) {
    return emu_lean_table().count(lean_key(logR, logT, ci, co, ld, st)) > 0;
}
static long long g_lean_launches = 0;
bool launch_lean(const PassArgs& a, int logT, int ci, int co, int ld, int st, long long ntiles, cudaStream_t) {
    auto it = emu_lean_table().find(lean_key(a.logR, logT, ci, co, ld, st));
    if (it == emu_lean_table().end()) {
        set_error(6, "no specialized pass kernel for radix 2^%d", a.logR);
        return false;
    }
    g_launches++;
    g_lean_launches++;
    if (ld == LD_FILT) {
        // the kernel's tile order for the filter-product pass (lean_batch_inner):
        // run the tiles in that order and check that it is a permutation
        const int logJ = logT + 4 - a.logR;
        std::vector<char> seen((size_t)ntiles, 0);
        for (long long k = 0; k < ntiles; ++k) {
            const long long t = lean_batch_inner(a, k, logJ);
            if (t < 0 || t >= ntiles || seen[(size_t)t]) {
                fprintf(stderr, "nfft_emu: filter-pass tile order is not a permutation (%lld -> %lld)\n", k, t);
                abort();
            }
            seen[(size_t)t] = 1;
            it->second(a, t, t + 1);
        }
        return true;
    }
    it->second(a, 0, ntiles);
    return true;
}
long long launch_count() { return g_launches; }

bool launch_post(cplx_t* post, long long n, cudaStream_t) {
    for (long long q = 0; q < n; ++q) {
        long double ang = 3.141592653589793238462643383279502884L * (long double)q / (long double)(2 * n);
        post[q] = mkc((real_t)cosl(ang), (real_t)-sinl(ang));
    }
    return true;
}

// ---- the persistent queue: items run in claim order by one virtual CTA.  In
// that order every dependency of an item has been published before the item
// is claimed, so a counter short of its target is a dependency that can never
// be published; the device kernel's bounded wait gives up on it, and so does
// this emulation (abort flag + status word).
int queue_grid(const DeviceCtx*) { return 296; }
static long long g_queue_items = 0;
bool launch_queue(const QueueArgs& q, int, cudaStream_t) {
    using T = real_t;
    static std::map<int, EmuLean> table = [] {
        std::map<int, EmuLean> m;
#define X(R, CI, CO, LD, ST) m[qop_lean(R, CI, CO, LD, ST)] = emu_lean<R, QUEUE_LOGT, CI != 0, CO != 0, LD, ST>;
        NFFT_QUEUE_LEAN(X)
#undef X
#define X(LD, ST) m[qop_gen(LD, ST)] = emu_pass<QUEUE_LOG_TILE, LD, ST>;
        NFFT_QUEUE_GENERIC(X)
#undef X
        return m;
    }();
    g_launches++;
    unsigned* ctr = q.ctr;
    for (long long i = 0; i < q.nitems; ++i) {
        const QItem it = q.items[i];
        QDesc d = q.descs[it.desc];
        if (d.flags & QD_IN_USER) d.a.in = (const char*)q.user_in + (size_t)d.a.in;
        if (d.flags & QD_OUT_USER) d.a.out = (char*)q.user_out + (size_t)d.a.out;
        if (it.wait >= 0 && ctr[it.wait] < (unsigned)it.target) {
            ctr[QCTR_ABORT] = 1;
            if (!*q.status) *q.status = (int)(i + 1);
            return true;
        }
        ++g_queue_items;
        const long long t0 = it.tile0, t1 = it.tile0 + it.ntiles;
        const TwTables<T>* tw = (const TwTables<T>*)d.a.tw;
        if (it.op == qop_unpack(ST_R) || it.op == qop_unpack(ST_T2)) {
            for (long long t = t0; t < t1; ++t) {
                long long w0, w1;
                unpack_tile_range(d.a, t, w0, w1);
                for (long long w = w0; w < w1; ++w) {
                    if (it.op == qop_unpack(ST_R)) unpack_item<T, ST_R>(d.a, tw, (const C2<T>*)d.z, d.zdist, w);
                    else unpack_item<T, ST_T2>(d.a, tw, (const C2<T>*)d.z, d.zdist, w);
                }
            }
        } else if (it.op == QOP_SCALAR) {
            const PassArgs& a = d.a;
            for (long long t = t0; t < t1; ++t)
                for (long long j = t * SCALAR_TILE; j < std::min<long long>((t + 1) * SCALAR_TILE, a.nlines); ++j) {
                    const T* x = (const T*)a.in + NFFT_GLD(&a.in_tab[j]);
                    T* y = (T*)a.out + NFFT_GLD(&a.out_tab[j]);
                    const T re = (T)(a.scale * (double)NFFT_GLD(&x[0]));
                    const T im = (a.conj_in && a.dst) ? (T)(a.scale * (double)NFFT_GLD(&x[1])) : (T)0;
                    NFFT_GST(&y[0], re);
                    if (a.conj_out) NFFT_GST(&y[1], im);
                }
        } else {
            auto f = table.find(it.op);
            if (f == table.end()) {
                fprintf(stderr, "nfft_emu: queue item %lld has unknown branch 0x%x\n", i, it.op);
                abort();
            }
            f->second(d.a, t0, t1);
        }
        if (it.done >= 0) ctr[it.done] += (unsigned)it.ntiles;
    }
    return true;
}

}  // namespace nfft

extern "C" {
// Test hooks: "device" memory of the emulator, launch counter.
void* nfft_emu_malloc(size_t bytes) {
    void* p = nullptr;
    return emu::Malloc(&p, bytes) == cudaSuccess ? p : nullptr;
}
void nfft_emu_free(void* p) { emu::Free(p); }
void nfft_emu_register_host(void* p, size_t bytes) {
    std::lock_guard<std::mutex> lk(emu::mu);
    emu::host_ok[(uintptr_t)p] = bytes;
}
void nfft_emu_unregister_host(void* p) {
    std::lock_guard<std::mutex> lk(emu::mu);
    emu::host_ok.erase((uintptr_t)p);
}
long long nfft_emu_launches(void) { return nfft::g_launches; }
long long nfft_emu_lean_launches(void) { return nfft::g_lean_launches; }
long long nfft_emu_checks(void) { return emu::n_checks; }
long long nfft_emu_queue_items(void) { return nfft::g_queue_items; }
long long nfft_emu_umma_launches(void) { return nfft::g_umma_launches; }
long long nfft_emu_umma_kind_launches(int k) { return (k >= 0 && k < 3) ? nfft::g_umma_kind[k] : -1; }
}

// nfft_kernels.cu -- instantiation and launch of the pass kernels, the
// unpack epilogue, the size-1 kernel, and the plan-time kernels (twiddle
// tables from FP64 sincospi; Bluestein chirp from exact k^2 mod 2n).
#include "nfft_engine.h"

#include <atomic>

namespace nfft {

// Kernels launched by this library in this process (all devices).
static std::atomic<long long> g_launches{0};
long long launch_count() { return g_launches.load(); }
void note_launch() { g_launches++; }

using PassFn = void (*)(const PassArgs);

// Valid (load, store) operator pairs.  Others are never planned.
#define NFFT_PAIRS(X)          \
    X(LD_C, ST_C)              \
    X(LD_C, ST_R)              \
    X(LD_C, ST_T2)             \
    X(LD_C, ST_T3)             \
    X(LD_C, ST_T4)             \
    X(LD_C, ST_BLUE)           \
    X(LD_T2, ST_C)             \
    X(LD_T2, ST_T2)            \
    X(LD_T3, ST_C)             \
    X(LD_T3, ST_T3)            \
    X(LD_IR, ST_C)             \
    X(LD_T4, ST_C)             \
    X(LD_T4, ST_T4)            \
    X(LD_BLUE, ST_C)           \
    X(LD_BLUE, ST_BLUE)        \
    X(LD_R2C, ST_C)            \
    X(LD_R2C, ST_R)            \
    X(LD_C, ST_C2R)            \
    X(LD_IR, ST_C2R)           \
    X(LD_FILT, ST_C)

constexpr int NLOAD = NUM_LOAD_OPS, NSTORE = NUM_STORE_OPS;

static PassFn pass_table(int log_tile, int ld, int st) {
    static PassFn t12[NLOAD][NSTORE] = {};
    static PassFn t13[NLOAD][NSTORE] = {};
    static bool filled = false;
    if (!filled) {
#define X(L, S)                                          \
    t12[L][S] = pass_kernel<real_t, 12, L, S>;           \
    t13[L][S] = pass_kernel<real_t, 13, L, S>;
        NFFT_PAIRS(X)
#undef X
        filled = true;
    }
    if (ld < 0 || ld >= NLOAD || st < 0 || st >= NSTORE) return nullptr;
    return log_tile == 13 ? t13[ld][st] : (log_tile == 12 ? t12[ld][st] : nullptr);
}

void lean_register_slice_0(LeanRegistry&);
void lean_register_slice_1(LeanRegistry&);
void lean_register_slice_2(LeanRegistry&);
void lean_register_slice_3(LeanRegistry&);
void lean_register_slice_4(LeanRegistry&);
void lean_register_slice_5(LeanRegistry&);
void lean_register_slice_6(LeanRegistry&);
void lean_register_slice_7(LeanRegistry&);

const LeanRegistry& lean_registry() {
    static LeanRegistry reg = [] {
        LeanRegistry r;
        lean_register_slice_0(r);
        lean_register_slice_1(r);
        lean_register_slice_2(r);
        lean_register_slice_3(r);
        lean_register_slice_4(r);
        lean_register_slice_5(r);
        lean_register_slice_6(r);
        lean_register_slice_7(r);
        return r;
    }();
    return reg;
}

bool lean_available(int logR, int logT, int ci, int co, int ld, int st) {
    return lean_registry().find(lean_key(logR, logT, ci, co, ld, st)) != nullptr;
}

bool launch_lean(const PassArgs& a, int logT, int ci, int co, int ld, int st, long long ntiles, cudaStream_t s) {
    const LeanEntry* e = lean_registry().find(lean_key(a.logR, logT, ci, co, ld, st));
    if (!e) {
        set_error(6, "no specialized pass kernel for radix 2^%d", a.logR);
        return false;
    }
    if (ntiles <= 0) return true;
    dim3 grid;
    if (ntiles <= 0x7fffffffll) grid = dim3((unsigned)ntiles, 1, 1);
    else grid = dim3(0x7fffffffu, (unsigned)((ntiles + 0x7fffffffll - 1) / 0x7fffffffll), 1);
    void* args[] = {(void*)&a};
    cudaError_t err = cudaLaunchKernel(e->fn, grid, dim3(e->threads, 1, 1), args, e->smem, s);
    g_launches++;
    return cuda_ok(err, "specialized pass kernel launch");
}

bool set_kernel_attributes() {
    for (auto& kv : lean_registry().entries) {
        if (!cuda_ok(cudaFuncSetAttribute(kv.second.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kv.second.smem),
                     "cudaFuncSetAttribute(lean pass)"))
            return false;
    }
    for (int lt = 12; lt <= 13; ++lt) {
        size_t smem = pass_smem_bytes<real_t>(lt);
        for (int ld = 0; ld < NLOAD; ++ld)
            for (int st = 0; st < NSTORE; ++st) {
                PassFn f = pass_table(lt, ld, st);
                if (!f) continue;
                if (!cuda_ok(cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                             "cudaFuncSetAttribute(pass)"))
                    return false;
            }
    }
    return true;
}

bool launch_pass(const PassArgs& a, int load_op, int store_op, int log_tile, long long ntiles, cudaStream_t s) {
    PassFn f = pass_table(log_tile, load_op, store_op);
    if (!f) {
        set_error(6, "no pass kernel for load op %d / store op %d / tile %d", load_op, store_op, log_tile);
        return false;
    }
    if (ntiles <= 0) return true;
    const int threads = (1 << log_tile) / 16;
    dim3 grid;
    if (ntiles <= 0x7fffffffll) grid = dim3((unsigned)ntiles, 1, 1);
    else {
        long long gy = (ntiles + 0x7fffffffll - 1) / 0x7fffffffll;
        grid = dim3(0x7fffffffu, (unsigned)gy, 1);
    }
    f<<<grid, threads, pass_smem_bytes<real_t>(log_tile), s>>>(a);
    g_launches++;
    return cuda_ok(cudaGetLastError(), "pass kernel launch");
}

bool launch_unpack(const PassArgs& a, int store_op, const cplx_t* Z, long long zdist, long long nlines, cudaStream_t s) {
    long long per = (a.N / 2) >= 2 ? (a.N / 4) : 1;
    long long total = per * nlines;
    int threads = 256;
    long long blocks = (total + threads - 1) / threads;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (blocks < 1) blocks = 1;
    if (store_op == ST_R) unpack_kernel<real_t, ST_R><<<(unsigned)blocks, threads, 0, s>>>(a, Z, zdist, nlines);
    else unpack_kernel<real_t, ST_T2><<<(unsigned)blocks, threads, 0, s>>>(a, Z, zdist, nlines);
    g_launches++;
    return cuda_ok(cudaGetLastError(), "unpack kernel launch");
}

bool launch_tiny(const real_t* x, real_t* y, long long howmany, long long inner, long long idist, long long odist,
                 int in_cplx, int out_cplx, double factor, cudaStream_t s) {
    int threads = 256;
    long long total = howmany * inner;
    long long blocks = (total + threads - 1) / threads;
    if (blocks > 148 * 64) blocks = 148 * 64;
    tiny_kernel<real_t><<<(unsigned)blocks, threads, 0, s>>>(x, y, howmany, inner, idist, odist, in_cplx, out_cplx, factor);
    g_launches++;
    return cuda_ok(cudaGetLastError(), "tiny kernel launch");
}

// Tk[m] = exp(-2 pi i m / 2^(12 (k+1))), from FP64 sincospi of the exact
// fraction 2m / 2^(12(k+1)).
__global__ void init_tables_kernel(TwTables<real_t>* tw) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    int level = blockIdx.y;
    if (m >= TW_SIZE) return;
    double frac = ldexp((double)m, 1 - TW_BITS * (level + 1));
    double s, c;
    sincospi(frac, &s, &c);
    tw->t[level][m] = mkc((real_t)c, (real_t)-s);
}

bool launch_init_tables(TwTables<real_t>* tw, cudaStream_t s) {
    init_tables_kernel<<<dim3(TW_SIZE / 256, 3, 1), 256, 0, s>>>(tw);
    return cuda_ok(cudaGetLastError(), "table init launch");
}

// chirp[k] = e^{-i pi k^2 / n} for k < n, with the phase index k^2 mod 2n
// formed exactly in 64-bit integers and the angle pi r / n evaluated by FP64
// sincospi.  bwrap (length M) receives conj(chirp) at k and M-k, zeros
// elsewhere: the Bluestein convolution kernel before its FFT.
__global__ void chirp_kernel(cplx_t* chirp, cplx_t* bwrap, long long n, long long M) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    if (k < n) {
        unsigned long long r = ((unsigned long long)k * (unsigned long long)k) % (unsigned long long)(2 * n);
        double s, c;
        sincospi((double)r / (double)n, &s, &c);
        chirp[k] = mkc((real_t)c, (real_t)-s);
        bwrap[k] = mkc((real_t)c, (real_t)s);
        if (k > 0) bwrap[M - k] = mkc((real_t)c, (real_t)s);
    } else if (k <= M - n) {
        bwrap[k] = mkc((real_t)0, (real_t)0);
    }
}

// post[q] = e^{-i pi q / 2n}, q < n: FP64 sincospi of the fraction q / 2n
// (the DCT-2 post-twiddle for lengths that are not powers of two).
__global__ void post_kernel(cplx_t* post, long long n) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    double s, c;
    sincospi((double)q / (double)(2 * n), &s, &c);
    post[q] = mkc((real_t)c, (real_t)-s);
}

bool launch_post(cplx_t* post, long long n, cudaStream_t s) {
    int threads = 256;
    long long blocks = (n + threads - 1) / threads;
    post_kernel<<<(unsigned)blocks, threads, 0, s>>>(post, n);
    return cuda_ok(cudaGetLastError(), "post-twiddle kernel launch");
}

bool launch_chirp(cplx_t* chirp, cplx_t* bwrap, long long n, long long M, cudaStream_t s) {
    int threads = 256;
    long long blocks = (M + threads - 1) / threads;
    chirp_kernel<<<(unsigned)blocks, threads, 0, s>>>(chirp, bwrap, n, M);
    return cuda_ok(cudaGetLastError(), "chirp kernel launch");
}

}  // namespace nfft

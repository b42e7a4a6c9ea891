// nfft_plan.cu -- device contexts, error state, pass schedules, plan
// construction and execution.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

#include "nfft_engine.h"
#include "nfft_queue.h"

namespace nfft {

// ---------------------------------------------------------------------------
// errors (per calling thread)
// ---------------------------------------------------------------------------
static thread_local int t_err = 0;
static thread_local char t_errmsg[512] = "";

void set_error(int code, const char* fmt, ...) {
    t_err = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_errmsg, sizeof t_errmsg, fmt, ap);
    va_end(ap);
}
int last_error() { return t_err; }
const char* last_error_string() { return t_errmsg; }
void clear_error() {
    t_err = 0;
    t_errmsg[0] = 0;
}
bool cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? 3 : 4, "%s: %s", what, cudaGetErrorString(e));
    return false;
}

// ---------------------------------------------------------------------------
// per-device contexts
// ---------------------------------------------------------------------------
static std::mutex g_ctx_mu;
static DeviceCtx g_ctx[64];

DeviceCtx* device_ctx(int device) {
    if (device < 0 || device >= 64) {
        set_error(2, "device %d out of range", device);
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    DeviceCtx& c = g_ctx[device];
    if (c.ready) return &c;
    int prev = -1;
    cudaGetDevice(&prev);
    if (!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return nullptr;
    cudaDeviceProp prop;
    if (!cuda_ok(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties")) return nullptr;
    if (prop.major < 10) {
        set_error(2, "device %d (%s, sm_%d%d) is not an sm_100 GPU", device, prop.name, prop.major, prop.minor);
        return nullptr;
    }
    c.device = device;
    c.sm_count = prop.multiProcessorCount;
    c.l2_bytes = (size_t)prop.l2CacheSize;
    if (!cuda_ok(cudaMalloc((void**)&c.tw, sizeof(TwTables<real_t>)), "cudaMalloc(twiddle tables)")) return nullptr;
    if (!launch_init_tables(c.tw, 0)) return nullptr;
    if (!set_kernel_attributes()) return nullptr;
    if (!cuda_ok(cudaDeviceSynchronize(), "twiddle table init")) return nullptr;
    c.ready = true;
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    return &c;
}

DeviceCtx* current_ctx() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        set_error(2, "no CUDA device available");
        return nullptr;
    }
    return device_ctx(dev);
}

Family family_of(int kind) {
    switch (kind) {
    case K_DFT: case K_INVDFT: return FAM_DFT;
    case K_REALDFT: case K_INVREALDFT: return FAM_REAL;
    case K_DCT4: case K_DST4: return FAM_T4;
    default: return FAM_T2T3;
    }
}

size_t in_elem_bytes(int kind) {
    return (kind == K_DFT || kind == K_INVDFT || kind == K_INVREALDFT) ? sizeof(cplx_t) : sizeof(real_t);
}
size_t out_elem_bytes(int kind) {
    return (kind == K_DFT || kind == K_INVDFT || kind == K_REALDFT) ? sizeof(cplx_t) : sizeof(real_t);
}

// ---------------------------------------------------------------------------
// schedules
// ---------------------------------------------------------------------------
static int ilog2(long long n) {
    int l = 0;
    while ((1ll << l) < n) ++l;
    return l;
}
static bool is_pow2(long long n) { return n > 0 && (n & (n - 1)) == 0; }

// Minimum lines per tile in column mode: 64 contiguous bytes per row.
static int log_jmin() { return sizeof(real_t) == 8 ? 2 : 3; }

static void split_sub(int logR, int* nsub, int* sub) {
    int n = 0;
    if (logR == 0) {
        *nsub = 0;
        return;
    }
    int n4 = logR / 4, rem = logR % 4;
    if (rem == 1 && n4 >= 1) {
        for (int i = 0; i < n4 - 1; ++i) sub[n++] = 4;
        sub[n++] = 3;
        sub[n++] = 2;
    } else {
        for (int i = 0; i < n4; ++i) sub[n++] = 4;
        if (rem) sub[n++] = rem;
    }
    *nsub = n;
}

FftSchedule make_schedule(int logL, bool strided, int max_tile, int max_pass_log) {
    FftSchedule s;
    s.logL = logL;
    const int jmin = log_jmin();
    if (!strided && logL <= max_tile) {
        s.npass = 1;
        s.plog[0] = logL;
        s.tile[0] = logL <= 12 ? 12 : 13;
    } else {
        // largest pass radix: the tile must keep jmin lines.  Contiguous axes of
        // 2^19..2^24 points run passes of radix <= 2^8 (three instead of two
        // for 2^19..2^22): the extra sweep costs less than the 64-byte rows of
        // the big radices (B200, 1 GiB batches: FP64 +13% / +15% / +30% / +37%
        // at 2^19 / 2^20 / 2^21 / 2^22, FP32 +26% / +27% at 2^19 / 2^20 and
        // the same schedule as before above).  NOTORIOUS_FFT_MAX_PASS_LOG sets
        // the cap for every size.
        static const int cap_env = [] {
            const char* e = getenv("NOTORIOUS_FFT_MAX_PASS_LOG");
            return e ? atoi(e) : 0;
        }();
        const int cap = max_pass_log >= 0 ? max_pass_log
                        : cap_env ? cap_env : ((!strided && logL >= 19 && logL <= 24 && max_tile == 13) ? 8 : 0);
        int maxr = max_tile - jmin;
        if (cap >= 4 && cap < maxr) maxr = std::max(cap, (logL + 3) / 4);   // at most 4 passes
        int np = (logL + maxr - 1) / maxr;
        if (np < 1) np = 1;
        s.npass = np;
        int base = logL / np, extra = logL % np;
        for (int i = 0; i < np; ++i) s.plog[i] = base + (i < extra ? 1 : 0);
        for (int i = 0; i < np; ++i) s.tile[i] = std::min(max_tile, (s.plog[i] + jmin + 1 <= 12) ? 12 : 13);
    }
    for (int i = 0; i < s.npass; ++i) split_sub(s.plog[i], &s.nsub[i], s.sub[i]);
    return s;
}

bool make_split_schedule(int logL, const int* plog, int npass, FftSchedule* out) {
    if (npass < 1 || npass > 4) return false;
    FftSchedule s;
    s.logL = logL;
    s.npass = npass;
    int sum = 0;
    for (int i = 0; i < npass; ++i) {
        const int lim = npass == 1 ? 12 : 12 - log_jmin();   // column passes keep >= jmin lines per tile
        if (plog[i] < 1 || plog[i] > lim) return false;
        s.plog[i] = plog[i];
        s.tile[i] = 12;
        split_sub(plog[i], &s.nsub[i], s.sub[i]);
        sum += plog[i];
    }
    if (sum != logL) return false;
    *out = s;
    return true;
}

FftSchedule reversed(const FftSchedule& s) {
    FftSchedule r = s;
    for (int i = 0; i < s.npass; ++i) {
        int k = s.npass - 1 - i;
        r.plog[i] = s.plog[k];
        r.tile[i] = s.tile[k];
        r.nsub[i] = s.nsub[k];
        for (int j = 0; j < MAX_SUB; ++j) r.sub[i][j] = s.sub[k][j];
    }
    return r;
}

// ---------------------------------------------------------------------------
// scratch
// ---------------------------------------------------------------------------
static void* get_scratch(notorious_fft_plan* p, int slot, size_t bytes) {
    if (p->scratch_bytes[slot] >= bytes && p->scratch[slot]) return p->scratch[slot];
    if (p->scratch[slot]) {
        cudaFree(p->scratch[slot]);
        p->scratch[slot] = nullptr;
        p->scratch_bytes[slot] = 0;
    }
    void* ptr = nullptr;
    if (!cuda_ok(cudaMalloc(&ptr, bytes), "cudaMalloc(scratch)")) return nullptr;
    p->scratch[slot] = ptr;
    p->scratch_bytes[slot] = bytes;
    return ptr;
}

// NOTORIOUS_FFT_GENERIC_PASSES=1 routes every pass through pass_kernel (the
// runtime-shaped kernel), e.g. to compare it with the specialized kernels.
static bool lean_disabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("NOTORIOUS_FFT_GENERIC_PASSES");
        v = (e && atoi(e) != 0) ? 1 : 0;
    }
    return v == 1;
}

Recorder*& recorder() {
    static thread_local Recorder* r = nullptr;
    return r;
}

bool queue_has_lean(int logR, int ci, int co, int ld, int st) {
    const int k = qop_lean(logR, ci, co, ld, st);
#define X(R, CI, CO, LD, ST) \
    if (k == qop_lean(R, CI, CO, LD, ST)) return true;
    NFFT_QUEUE_LEAN(X)
#undef X
    return false;
}

// Inter-pass scratch per chunk of the outermost batch dimension
// (NOTORIOUS_FFT_SCRATCH_MB, default 2048).  B200, FP64 2^16 x 4096 dft +
// invdft: 32 MB chunks 2179 GB/s, 128 MB 2788, 512 MB 3187, 2048 MB 3309,
// 4096 MB 3330 -- fewer, larger launches win; chunks small enough to keep the
// scratch in L2 lose more to launch count than they save in DRAM traffic.
static size_t scratch_cap_bytes() {
    // a recorded (queue) bucket runs in one piece: its scratch is its own
    if (recorder()) return (size_t)1 << 62;
    static size_t cap = 0;
    if (!cap) {
        const char* e = getenv("NOTORIOUS_FFT_SCRATCH_MB");
        long mb = e ? atol(e) : 2048;
        if (mb < 1) mb = 1;
        cap = (size_t)mb << 20;
    }
    return cap;
}

// ---------------------------------------------------------------------------
// pass construction
// ---------------------------------------------------------------------------


static void fill_common(PassArgs& a, const DeviceCtx* c) {
    memset(&a, 0, sizeof a);
    a.tw = c->tw;
    a.scale = 1.0;
    a.jpos = -1;
}

// Line dims of a pass.  Contiguous lines: j innermost then the batch dims;
// strided lines: the view's first (unit-stride) batch dim innermost, then j.
static void set_lines(PassArgs& a, const View& src, const View& dst, long long nj, bool j_inner) {
    int nd = 0;
    auto add_batch = [&](int d) {
        a.cnt[nd] = src.cnt[d];
        a.istr[nd] = src.str[d];
        a.ostr[nd] = dst.str[d];
        ++nd;
    };
    auto add_j = [&]() {
        if (nj > 1) {
            a.cnt[nd] = nj;
            a.istr[nd] = 0;
            a.ostr[nd] = 0;
            a.jpos = nd;
            ++nd;
        }
    };
    if (j_inner) {
        add_j();
        for (int d = 0; d < src.nb; ++d) add_batch(d);
    } else {
        if (src.nb > 0) add_batch(0);
        add_j();
        for (int d = 1; d < src.nb; ++d) add_batch(d);
    }
    if (nd == 0) {
        a.cnt[0] = 1;
        a.istr[0] = a.ostr[0] = 0;
        nd = 1;
    }
    a.ndims = nd;
    long long n = 1;
    for (int i = 0; i < nd; ++i) n *= a.cnt[i];
    a.nlines = n;
}

// L2 policy of multi-pass transforms: every pass that touches scratch
// streams its user data (evict first) and keeps its scratch (evict_last
// stores, discard after the last read).  NOTORIOUS_FFT_CACHE_HINTS: 0 never;
// 1 always; 2 (default) while the chunk's scratch fits in half of L2.  B200,
// batched c2c: the policy gains 3-5% when the scratch fits (FP64 2^14 x 256,
// 2^17 x 24, 2^20 x 4) and loses 7-16% when it does not (1 GiB batches,
// 2^14 .. 2^20, FP64 and FP32) -- the kept lines cannot be reused there and
// only push other data out.
static int cache_mode() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("NOTORIOUS_FFT_CACHE_HINTS");
        v = e ? atoi(e) : 2;
        if (v < 0 || v > 2) v = 2;
    }
    return v;
}
static bool cache_hints() { return cache_mode() != 0; }

static int env_int(const char* name, int dflt) {
    const char* e = getenv(name);
    return e ? atoi(e) : dflt;
}
// Tuning knobs (defaults chosen from measurements on B200):
//   NOTORIOUS_FFT_LEAN_LOGT  threads (log2) of the complex pass kernels: 128
//       (2048-point tiles) by default, 256 for the radix-2^9 passes of 2^17 /
//       2^18 axes (and 2^16 in float), where 4096-point tiles keep 128-byte
//       rows (B200: +7% / +19% FP64, +5..31% FP32)
//   NOTORIOUS_FFT_TW_MODE    pre-twiddle generation (0 tree, 1 chains, 2 tables)
static int lean_logt_pref(int logL) {
    static int v = env_int("NOTORIOUS_FFT_LEAN_LOGT", 0);
    if (v) return v;
    return (logL == 17 || logL == 18 || (sizeof(real_t) == 4 && logL == 16)) ? 8 : 7;
}
static int tw_mode() {
    static int v = env_int("NOTORIOUS_FFT_TW_MODE", 1);
    return v;
}

// Arguments of one pass (everything but the tile shape and the kernel).
// in_scratch / out_scratch: the pass reads / writes an inter-pass scratch buffer.
static void make_pass_args(const DeviceCtx* c, const View& src, const View& dst, int logL, int logNs, int logR,
                           int nsub, const int* sub, const OpSpec& op, bool first, bool last, int mid, int logNs_out,
                           const cplx_t* chirp, const cplx_t* filt, bool in_scratch, bool out_scratch, PassArgs& a) {
    fill_common(a, c);
    a.tw_mode = tw_mode();
    if (cache_hints() && (in_scratch || out_scratch)) {
        bool on = cache_mode() == 1;
        if (!on) {
            const View& sv = in_scratch ? src : dst;
            long long n = 1ll << logL;
            for (int d = 0; d < sv.nb; ++d) n *= sv.cnt[d];
            on = (double)n * sizeof(cplx_t) <= 0.5 * (double)c->l2_bytes;
        }
        if (on) {
            a.hint_in = in_scratch ? 2 : 1;
            a.hint_out = out_scratch ? 2 : 1;
            a.discard_in = in_scratch ? 1 : 0;
        }
    }
    a.in = src.ptr;
    a.out = dst.ptr;
    a.logR = logR;
    a.logNs = logNs;
    a.logNj = logL - logR;
    a.logNs_out = logNs_out;
    a.nsub = nsub;
    for (int i = 0; i < nsub; ++i) a.sublog[i] = sub[i];
    a.in_estride = src.estride;
    a.out_estride = dst.estride;
    const long long nj = 1ll << (logL - logR);
    // Strided source axis with a unit-stride batch dim: that dim goes innermost
    // so consecutive lines are consecutive addresses; otherwise j goes innermost.
    const bool j_inner = !(src.estride != 1 && src.nb > 0 && src.str[0] == 1);
    set_lines(a, src, dst, nj, j_inner);
    a.in_row = (nj == 1 && src.estride == 1) ? 1 : 0;
    a.out_row = (logNs_out == 0 && dst.estride == 1 && (nj == 1 || j_inner)) ? 1 : 0;
    a.conj_in = first ? op.conj_in : 0;
    a.conj_out = last ? op.conj_out : 0;
    a.scale = last ? op.scale : 1.0;
    a.N = op.N;
    a.logN = op.logN;
    a.dst = op.dst;
    a.chirp = chirp;
    a.filt = filt;
    a.mid = mid;
    a.vjp = op.vjp;
    a.post = op.post;
}

bool run_pass(const DeviceCtx* c, const View& src, const View& dst, int logL, int logNs, int logR, int tile,
              int nsub, const int* sub, const OpSpec& op, bool first, bool last, int mid, int logNs_out,
              const cplx_t* chirp, const cplx_t* filt, cudaStream_t s, bool in_scratch, bool out_scratch) {
    PassArgs a;
    make_pass_args(c, src, dst, logL, logNs, logR, nsub, sub, op, first, last, mid, logNs_out, chirp, filt, in_scratch,
                   out_scratch, a);
    int ldop = first ? op.ld : LD_C;
    int stop = last ? op.st : ST_C;
    int logE_max = tile;
    int logJ = logE_max - logR;
    if (logJ > 8) logJ = 8;
    int lines_log = ilog2(a.nlines);
    if (logJ > lines_log) logJ = lines_log;
    if (logJ < 0) {
        set_error(6, "pass radix 2^%d exceeds tile 2^%d", logR, tile);
        return false;
    }
    if (Recorder* rec = recorder()) {
        // queue form: a branch of the persistent 256-thread kernel.  Scratch
        // written earlier in the same launch is read through L2 (hint 3, for
        // coherence); NOTORIOUS_FFT_QUEUE_KEEP=0 drops the keep-in-L2 policy
        // (evict_last scratch stores, discard after the read).
        static const int keep = env_int("NOTORIOUS_FFT_QUEUE_KEEP", 1);
        if (in_scratch || out_scratch) {
            a.hint_in = in_scratch ? 3 : 1;
            a.hint_out = out_scratch ? (keep ? 2 : 0) : 1;
            a.discard_in = in_scratch && keep ? 1 : 0;
        }
        const int ci = a.in_row ? 0 : 1, co = a.out_row ? 0 : 1;
        RecLaunch r;
        if (!mid && logR >= 4 && !lean_disabled() && queue_has_lean(logR, ci, co, ldop, stop)) {
            a.logJ = QUEUE_LOGT + 4 - logR;
            r.op = qop_lean(logR, ci, co, ldop, stop);
        } else {
            if (tile != QUEUE_LOG_TILE) {
                set_error(6, "queue pass of radix 2^%d needs a 2^%d tile", logR, tile);
                return false;
            }
            a.logJ = logJ;
            r.op = qop_gen(ldop, stop);
        }
        r.a = a;
        r.ntiles = (a.nlines + (1ll << a.logJ) - 1) >> a.logJ;
        rec->launches.push_back(r);
        return true;
    }
    // split tensor-core form: radix-256 passes on tcgen05 where the layout
    // allows (unit-stride lines, aligned strides), else in the warp-level
    // specialized kernel; other radices with the radix-16 sub-stages of the
    // generic pass on the tensor cores
    if (op.tc && !mid && ldop == LD_C && stop == ST_C && logR == 8 && logNs + 8 <= 24) {
        if (tc_umma_enabled()) {
            bool launched = false;
            if (!try_launch_tc_umma(a, c->sm_count, s, launched)) return false;
            if (launched) return true;
        }
        if (tc_lean_enabled()) {
            a.logJ = 4;
            return launch_tc_lean(a, c->sm_count, s);
        }
    }
    if (op.tc && !mid && ldop == LD_C && stop == ST_C && logR >= 4 && tile == 12 && logJ == 12 - logR) {
        a.logJ = logJ;
        long long nt = (a.nlines + (1ll << logJ) - 1) >> logJ;
        return launch_tc_pass(a, tile, nt, s);
    }
    // specialized kernel for this pass shape when one is instantiated
    if (!mid && logR >= 4 && !lean_disabled()) {
        const int ci = a.in_row ? 0 : 1, co = a.out_row ? 0 : 1;
        const bool rr = !ci && !co;
        int logT = (logR <= 12 && (rr || logR <= 10)) ? 8 : 9;
        // 2048-point tiles where preferred, unless a column tile would keep
        // fewer than 64 contiguous bytes per row (FP32 radix >= 2^9)
        if (lean_logt_pref(logL) == 7 && lean_available(logR, 7, ci, co, ldop, stop) &&
            (rr || 7 + 4 - logR >= log_jmin()))
            logT = 7;
        if (op.logt && lean_available(logR, op.logt, ci, co, ldop, stop)) logT = op.logt;   // tuned
        if (lean_available(logR, logT, ci, co, ldop, stop)) {
            a.logJ = logT + 4 - logR;
            long long nt = (a.nlines + (1ll << a.logJ) - 1) >> a.logJ;
            return launch_lean(a, logT, ci, co, ldop, stop, nt, s);
        }
    }
    a.logJ = logJ;
    long long ntiles = (a.nlines + (1ll << logJ) - 1) >> logJ;
    return launch_pass(a, ldop, stop, tile, ntiles, s);
}

// Scratch view with the same lines as `like` and a contiguous (or, for
// strided lines, unit-stride-batch-innermost) layout of axis length L.
View scratch_view(void* ptr, const View& like, long long L, bool strided) {
    View v;
    v.ptr = ptr;
    v.nb = like.nb;
    for (int d = 0; d < like.nb; ++d) v.cnt[d] = like.cnt[d];
    if (!strided || like.nb == 0) {
        v.estride = 1;
        long long s = L;
        for (int d = 0; d < like.nb; ++d) {
            v.str[d] = s;
            s *= like.cnt[d];
        }
    } else {
        v.str[0] = 1;
        v.estride = like.cnt[0];
        long long s = like.cnt[0] * L;
        for (int d = 1; d < like.nb; ++d) {
            v.str[d] = s;
            s *= like.cnt[d];
        }
    }
    return v;
}

// Run a power-of-two FFT of complex length 2^logL over the lines of src ->
// dst with the fused operators of `op`.  Multi-pass runs go through plan
// scratch slots 0/1, in chunks of the outermost batch dim sized to the
// scratch cap.
static bool run_pow2_axis(notorious_fft_plan* p, const DeviceCtx* c, const AxisPlan& ax, View src, View dst,
                          const OpSpec& op, cudaStream_t s) {
    const int logL = ax.fft_contig.logL;
    const bool strided = !(src.estride == 1 && dst.estride == 1);
    const FftSchedule& sch = strided ? ax.fft_strided : ax.fft_contig;
    const long long L = 1ll << logL;
    const int np = sch.npass;
    if (np == 1 && !(op.paired && strided)) {
        OpSpec o1 = op;
        o1.logt = sch.logt;
        return run_pass(c, src, dst, logL, 0, sch.plog[0], sch.tile[0], sch.nsub[0], sch.sub[0], o1, true, true, 0, 0,
                        nullptr, nullptr, s);
    }
    // multi-pass (or a paired op on strided lines): chunk the outermost batch dim
    long long lines = src.lines();
    long long outer = src.nb > 0 ? src.cnt[src.nb - 1] : 1;
    long long inner_lines = outer > 0 ? lines / outer : lines;
    size_t per_outer = (size_t)inner_lines * (size_t)L * sizeof(cplx_t);
    long long chunk = (long long)(scratch_cap_bytes() / std::max<size_t>(per_outer, 1));
    if (chunk < 1) chunk = 1;
    if (chunk > outer) chunk = outer;
    // realdft / DCT-2 / DST-2 over several passes: the last pass unpacks in
    // mirror tiles when that kernel exists (the same choice run_pass makes);
    // otherwise an unpack epilogue reads the packed spectrum back
    bool mirror = false;
    if (op.paired && np >= 2 && !strided && !lean_disabled()) {
        const int lr = sch.plog[np - 1];
        mirror = recorder() ? queue_has_lean(lr, 1, 1, LD_C, op.st)
                            : (lr >= 4 && lean_available(lr, (lr <= 12 && lr <= 10) ? 8 : 9, 1, 1, LD_C, op.st));
    }
    const bool paired_epilogue = op.paired && !mirror;
    const int nbuf = paired_epilogue ? (np >= 2 ? 2 : 1) : (np >= 3 ? 2 : 1);
    void* buf[2] = {nullptr, nullptr};
    for (int i = 0; i < nbuf; ++i) {
        buf[i] = get_scratch(p, i, (size_t)chunk * per_outer);
        if (!buf[i]) return false;
    }
    for (long long o0 = 0; o0 < outer; o0 += chunk) {
        long long cn = std::min(chunk, outer - o0);
        View vs = src, vd = dst;
        if (src.nb > 0) {
            vs.ptr = (char*)src.ptr + (size_t)(o0 * src.str[src.nb - 1]) * (op.ld == LD_C || op.ld == LD_BLUE || op.ld == LD_IR ? sizeof(cplx_t) : sizeof(real_t));
            vs.cnt[src.nb - 1] = cn;
            vd.ptr = (char*)dst.ptr + (size_t)(o0 * dst.str[dst.nb - 1]) *
                                          ((op.st == ST_C || op.st == ST_R || op.st == ST_BLUE) ? sizeof(cplx_t) : sizeof(real_t));
            vd.cnt[dst.nb - 1] = cn;
        }
        View cur = vs;
        int logNs = 0;
        for (int i = 0; i < np; ++i) {
            bool first = i == 0, last = i == np - 1;
            View out;
            bool to_user = last && !paired_epilogue;
            if (to_user) out = vd;
            else out = scratch_view(buf[i % nbuf], vs, L, strided && !paired_epilogue);
            OpSpec o = op;
            o.logt = sch.logt;
            if (last && paired_epilogue) {
                o.st = ST_C;
                o.scale = 1.0;
                o.conj_out = 0;
            }
            int logR = sch.plog[i];
            if (!run_pass(c, cur, out, logL, logNs, logR, sch.tile[i], sch.nsub[i], sch.sub[i], o, first, last, 0, logNs,
                          nullptr, nullptr, s, /*in_scratch=*/!first, /*out_scratch=*/!to_user))
                return false;
            logNs += logR;
            cur = out;
        }
        if (paired_epilogue) {
            PassArgs a;
            fill_common(a, c);
            a.out = vd.ptr;
            a.out_estride = vd.estride;
            a.N = op.N;
            a.logN = op.logN;
            a.dst = op.dst;
            a.vjp = op.vjp;
            a.ndims = vd.nb > 0 ? vd.nb : 1;
            for (int d = 0; d < vd.nb; ++d) {
                a.cnt[d] = vd.cnt[d];
                a.ostr[d] = vd.str[d];
            }
            if (vd.nb == 0) {
                a.cnt[0] = 1;
                a.ostr[0] = 0;
            }
            if (Recorder* rec = recorder()) {
                RecLaunch r;
                r.op = qop_unpack(op.st);
                a.nlines = vs.lines();
                r.a = a;
                r.ntiles = a.nlines * unpack_tiles_per_line(a);
                r.z = cur.ptr;
                r.zdist = L;
                rec->launches.push_back(r);
                continue;
            }
            if (!launch_unpack(a, op.st, (const cplx_t*)cur.ptr, L, vs.lines(), s)) return false;
        }
    }
    return true;
}

// Bluestein for a complex axis of length n (not a power of two).
// ld / st: LD_BLUE / ST_BLUE for complex data; the real-input operators
// (LD_BLUE_R, LD_BLUE_T2 / ST_BLUE_R, ST_BLUE_T2) give realdft and DCT-2 of
// any length (queue plans).
static bool run_bluestein_axis(notorious_fft_plan* p, const DeviceCtx* c, const AxisPlan& ax, View src, View dst,
                               int inverse, double scale, cudaStream_t s, int ld = LD_BLUE, int st = ST_BLUE) {
    const int logM = ax.logM;
    const long long M = 1ll << logM;
    OpSpec op;
    op.ld = ld;
    op.st = st;
    op.post = ax.post;
    op.conj_in = inverse;
    op.conj_out = inverse;
    op.scale = scale;
    op.N = ax.n;
    const FftSchedule& f = ax.mfwd;
    const FftSchedule& g = ax.minv;
    const int np = f.npass;
    if (np == 1) {
        return run_pass(c, src, dst, logM, 0, f.plog[0], f.tile[0], f.nsub[0], f.sub[0], op, true, true, 1, 0, ax.chirp,
                        ax.filt, s);
    }
    long long lines = src.lines();
    long long outer = src.nb > 0 ? src.cnt[src.nb - 1] : 1;
    long long inner_lines = outer > 0 ? lines / outer : lines;
    size_t per_outer = (size_t)inner_lines * (size_t)M * sizeof(cplx_t);
    long long chunk = (long long)(scratch_cap_bytes() / std::max<size_t>(per_outer, 1));
    if (chunk < 1) chunk = 1;
    if (chunk > outer) chunk = outer;
    void* buf[2];
    for (int i = 0; i < 2; ++i) {
        buf[i] = get_scratch(p, i, (size_t)chunk * per_outer);
        if (!buf[i]) return false;
    }
    for (long long o0 = 0; o0 < outer; o0 += chunk) {
        long long cn = std::min(chunk, outer - o0);
        View vs = src, vd = dst;
        if (src.nb > 0) {
            const size_t ib = ld == LD_BLUE ? sizeof(cplx_t) : sizeof(real_t);
            const size_t ob = st == ST_BLUE_T2 ? sizeof(real_t) : sizeof(cplx_t);
            vs.ptr = (char*)src.ptr + (size_t)(o0 * src.str[src.nb - 1]) * ib;
            vs.cnt[src.nb - 1] = cn;
            vd.ptr = (char*)dst.ptr + (size_t)(o0 * dst.str[dst.nb - 1]) * ob;
            vd.cnt[dst.nb - 1] = cn;
        }
        View cur = vs;
        int bi = 0;
        int logNs = 0;
        // forward passes 0 .. np-2
        for (int i = 0; i < np - 1; ++i) {
            View out = scratch_view(buf[bi], vs, M, false);
            if (!run_pass(c, cur, out, logM, logNs, f.plog[i], f.tile[i], f.nsub[i], f.sub[i], op, i == 0, false, 0,
                          logNs, ax.chirp, ax.filt, s))
                return false;
            logNs += f.plog[i];
            cur = out;
            bi ^= 1;
        }
        {
            // the last forward pass and the first inverse pass as separate
            // specialized passes; the filter product and conjugation are the
            // inverse pass's load operator.  (Fusing the two into one tile, the
            // product never leaving shared memory, measured slower on B200:
            // 1,000,003 x 4 0.360 vs 0.349 ms -- the fused tile does two passes'
            // arithmetic at the SMs' tile rate.)
            View out = scratch_view(buf[bi], vs, M, false);
            if (!run_pass(c, cur, out, logM, logNs, f.plog[np - 1], f.tile[np - 1], f.nsub[np - 1], f.sub[np - 1], op,
                          false, false, 0, logNs, ax.chirp, ax.filt, s))
                return false;
            cur = out;
            bi ^= 1;
            View out2 = scratch_view(buf[bi], vs, M, false);
            OpSpec o = op;
            o.ld = LD_FILT;
            o.conj_in = 0;
            if (!run_pass(c, cur, out2, logM, 0, g.plog[0], g.tile[0], g.nsub[0], g.sub[0], o, true, false, 0, 0,
                          ax.chirp, ax.filt, s))
                return false;
            cur = out2;
            bi ^= 1;
        }
        // remaining inverse passes (the first one ran above)
        int logNs_inv = g.plog[0];
        for (int i = 1; i < np; ++i) {
            bool last = i == np - 1;
            View out = last ? vd : scratch_view(buf[bi], vs, M, false);
            if (!run_pass(c, cur, out, logM, logNs_inv, g.plog[i], g.tile[i], g.nsub[i], g.sub[i], op, false, last, 0,
                          logNs_inv, ax.chirp, ax.filt, s))
                return false;
            logNs_inv += g.plog[i];
            cur = out;
            bi ^= 1;
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// plans
// ---------------------------------------------------------------------------
PlanOverride*& plan_override() {
    thread_local PlanOverride* o = nullptr;
    return o;
}

static bool build_axis(notorious_fft_plan* p, const DeviceCtx* c, AxisPlan& ax, int n, int family, int max_tile = 13) {
    ax.n = n;
    ax.pow2 = is_pow2(n);
    ax.logn = ilog2(n);
    if (ax.pow2) {
        int logL = (family == FAM_DFT) ? ax.logn : std::max(0, ax.logn - 1);
        ax.fft_contig = make_schedule(logL, false, max_tile);
        ax.fft_strided = make_schedule(logL, true, max_tile);
        // standalone plans: an autotuner trial, else the tune cache's split and
        // thread count for (family, n) on this GPU (a split this build cannot
        // run keeps the default schedule)
        if (!recorder() && logL >= 1) {
            std::vector<int> split;
            int logt = 0;
            bool have = false;
            if (PlanOverride* o = plan_override()) {
                split = o->split;
                logt = o->logt;
                have = true;
            } else {
                have = tune_get_plan(family, n, split, logt);
            }
            if (have) {
                FftSchedule t;
                if (split.empty()) t = ax.fft_contig;
                else if (!make_split_schedule(logL, split.data(), (int)split.size(), &t)) t = ax.fft_contig;
                t.logt = (logt == 7 || logt == 8 || logt == 9) ? logt : 0;
                ax.fft_contig = t;
            }
        }
        return true;
    }
    if (family != FAM_DFT) {
        set_error(1, "length %d is not a power of two", n);
        return false;
    }
    long long M = 1;
    while (M < 2ll * n - 1) M <<= 1;
    ax.logM = ilog2(M);
    ax.mfwd = make_schedule(ax.logM, false, max_tile);
    ax.minv = reversed(ax.mfwd);
    if (!cuda_ok(cudaMalloc((void**)&ax.chirp, sizeof(cplx_t) * (size_t)n), "cudaMalloc(chirp)")) return false;
    if (!cuda_ok(cudaMalloc((void**)&ax.filt, sizeof(cplx_t) * (size_t)M), "cudaMalloc(filter)")) return false;
    cplx_t* bwrap = nullptr;
    if (!cuda_ok(cudaMalloc((void**)&bwrap, sizeof(cplx_t) * (size_t)M), "cudaMalloc(bluestein kernel)")) return false;
    bool ok = launch_chirp(ax.chirp, bwrap, n, M, 0);
    if (ok) {
        // filt = FFT_M(bwrap) / M with the library's own passes
        AxisPlan mp;
        mp.n = (int)M;
        mp.logn = ax.logM;
        mp.fft_contig = make_schedule(ax.logM, false);
        mp.fft_strided = mp.fft_contig;
        View vs, vd;
        vs.ptr = bwrap;
        vd.ptr = ax.filt;
        OpSpec op;
        op.scale = 1.0 / (double)M;
        ok = run_pow2_axis(p, c, mp, vs, vd, op, 0);
    }
    ok = ok && cuda_ok(cudaDeviceSynchronize(), "Bluestein filter");
    cudaFree(bwrap);
    return ok;
}

notorious_fft_plan* plan_create(int family, int d, const int* Ns) {
    if (d < 1 || !Ns) {
        set_error(1, "invalid rank %d", d);
        return nullptr;
    }
    long long total = 1;
    for (int i = 0; i < d; ++i) {
        if (Ns[i] <= 0) {
            set_error(1, "invalid dimension %d", Ns[i]);
            return nullptr;
        }
        if (family != FAM_DFT && !is_pow2(Ns[i])) {
            set_error(1, "dimension %d is not a power of two", Ns[i]);
            return nullptr;
        }
        total *= Ns[i];
        if (total > 0x7fffffffll) {
            set_error(1, "transform size exceeds the int range of the API");
            return nullptr;
        }
    }
    DeviceCtx* c = current_ctx();
    if (!c) return nullptr;
    notorious_fft_plan* p = new notorious_fft_plan();
    p->family = family;
    p->device = c->device;
    p->dims.assign(Ns, Ns + d);
    p->axes.resize(d);
    for (int i = 0; i < d; ++i) {
        // a real plan transforms only its last axis as real; the leading axes
        // are full-length complex DFTs of the half spectrum (FFTW layout)
        int fam_i = (family == FAM_REAL && i < d - 1) ? FAM_DFT : family;
        if (!build_axis(p, c, p->axes[i], Ns[i], fam_i)) {
            plan_destroy(p);
            return nullptr;
        }
    }
    return p;
}

void plan_destroy(notorious_fft_plan* p) {
    if (!p) return;
    int prev = -1;
    cudaGetDevice(&prev);
    if (p->device >= 0 && prev != p->device) cudaSetDevice(p->device);
    for (auto& ax : p->axes) {
        if (ax.chirp) cudaFree(ax.chirp);
        if (ax.filt) cudaFree(ax.filt);
        if (ax.post) cudaFree(ax.post);
    }
    for (int i = 0; i < 2; ++i)
        if (p->scratch[i]) cudaFree(p->scratch[i]);
    if (p->stage_in) cudaFree(p->stage_in);
    for (int i = 0; i < 2; ++i) {
        if (p->ev_h[i]) cudaEventDestroy(p->ev_h[i]);
        if (p->ev_c[i]) cudaEventDestroy(p->ev_c[i]);
        if (p->ev_d[i]) cudaEventDestroy(p->ev_d[i]);
    }
    if (p->ev_last) cudaEventDestroy(p->ev_last);
    if (p->s_h2d) cudaStreamDestroy(p->s_h2d);
    if (p->s_d2h) cudaStreamDestroy(p->s_d2h);
    if (p->nd_tmp) cudaFree(p->nd_tmp);
    if (p->stage_out) cudaFree(p->stage_out);
    if (p->host_in) cudaFreeHost(p->host_in);
    if (p->host_out) cudaFreeHost(p->host_out);
    if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
    delete p;
}

static long long prod(const std::vector<int>& v, int a, int b) {
    long long r = 1;
    for (int i = a; i < b; ++i) r *= v[i];
    return r;
}

long long plan_in_elems(const notorious_fft_plan* p, int kind) {
    long long total = prod(p->dims, 0, (int)p->dims.size());
    if (kind == K_INVREALDFT) return total / p->dims.back() * (p->dims.back() / 2 + 1);
    return total;
}
long long plan_out_elems(const notorious_fft_plan* p, int kind) {
    long long total = prod(p->dims, 0, (int)p->dims.size());
    if (kind == K_REALDFT) return total / p->dims.back() * (p->dims.back() / 2 + 1);
    return total;
}

// View of axis `a` of a row-major array with dims D (elements of the view
// type), batched `howmany` times at distance `dist`.
static View axis_view(void* ptr, const std::vector<long long>& D, int a, long long howmany, long long dist) {
    View v;
    v.ptr = ptr;
    long long inner = 1, outer = 1;
    for (size_t i = a + 1; i < D.size(); ++i) inner *= D[i];
    for (int i = 0; i < a; ++i) outer *= D[i];
    v.estride = inner;
    int nb = 0;
    if (inner > 1) { v.cnt[nb] = inner; v.str[nb] = 1; ++nb; }
    if (outer > 1) { v.cnt[nb] = outer; v.str[nb] = D[a] * inner; ++nb; }
    if (howmany > 1) { v.cnt[nb] = howmany; v.str[nb] = dist; ++nb; }
    v.nb = nb;
    return v;
}

static OpSpec real_op(int kind, int n) {
    OpSpec op;
    op.N = n;
    op.logN = ilog2(n);
    switch (kind) {
    case K_REALDFT: op.ld = LD_R2C; op.st = ST_R; op.paired = true; break;
    case K_INVREALDFT: op.ld = LD_IR; op.st = ST_C2R; op.conj_out = 1; break;
    case K_DCT2: op.ld = LD_T2; op.st = ST_T2; op.paired = true; break;
    case K_DST2: op.ld = LD_T2; op.st = ST_T2; op.paired = true; op.dst = 1; break;
    case K_DCT3: op.ld = LD_T3; op.st = ST_T3; break;
    case K_DST3: op.ld = LD_T3; op.st = ST_T3; op.dst = 1; break;
    case K_DCT4: op.ld = LD_T4; op.st = ST_T4; break;
    case K_DST4: op.ld = LD_T4; op.st = ST_T4; op.dst = 1; break;
    }
    return op;
}

// Size-1 factor of the real families (the reference's N = 1 cases).
static double tiny_factor(int kind) {
    switch (kind) {
    case K_DCT2: case K_DST2: return 2.0;
    case K_DCT4: case K_DST4: return 1.41421356237309504880;
    default: return 1.0;
    }
}

// One real-family 1-D transform along axis `a` (src -> dst views).
static bool run_real_axis(notorious_fft_plan* p, const DeviceCtx* c, const AxisPlan& ax, int kind, const View& src,
                          const View& dst, int vjp, double unit_factor, cudaStream_t s) {
    if (ax.n == 1) {
        // every line is one element: y = factor * x (complex in/out for the realdft pair)
        long long lines = src.lines();
        if (src.nb > 1 || dst.nb > 1) {
            // N-D size-1 axes are skipped by the caller; only 1-D batches reach here
            set_error(6, "size-1 axis inside a multi-dimensional real transform");
            return false;
        }
        long long idist = src.nb ? src.str[0] : 1, odist = dst.nb ? dst.str[0] : 1;
        int in_c = kind == K_INVREALDFT, out_c = kind == K_REALDFT;
        return launch_tiny((const real_t*)src.ptr, (real_t*)dst.ptr, lines, 1, idist, odist, in_c, out_c, unit_factor, s);
    }
    OpSpec op = real_op(kind, ax.n);
    op.vjp = vjp;
    return run_pow2_axis(p, c, ax, src, dst, op, s);
}

// Adjoint pipelines: the transposed transform of each family (complex data
// treated as pairs of reals).  dft <-> unnormalized inverse; realdft <->
// invrealdft with interior-bin weights; DCT-2 <-> DCT-3 and DST-2 <-> DST-3
// with the first / last coefficient weighted; DCT-4 and DST-4 are symmetric.
static int adjoint_kind(int kind) {
    switch (kind) {
    case K_REALDFT: return K_INVREALDFT;
    case K_INVREALDFT: return K_REALDFT;
    case K_DCT2: return K_DCT3;
    case K_DST2: return K_DST3;
    case K_DCT3: return K_DCT2;
    case K_DST3: return K_DST2;
    default: return kind;
    }
}

int plan_execute(notorious_fft_plan* p, int okind, const void* in, void* out, long long howmany, long long idist,
                 long long odist, cudaStream_t stream, int vjp) {
    const int kind = vjp ? adjoint_kind(okind) : okind;
    const double unit_factor = tiny_factor(okind);
    DeviceCtx* c = device_ctx(p->device);
    if (!c) return last_error();
    const int d = (int)p->dims.size();
    std::vector<long long> D(p->dims.begin(), p->dims.end());
    if (howmany < 1) return 0;
    const int fam = family_of(kind);
    if (fam != p->family) {
        set_error(1, "transform kind %d does not match the aux family %d", kind, p->family);
        return 1;
    }
    bool ok = true;
    if (fam == FAM_DFT) {
        // forward / inverse direction; the Bluestein 1/n factor belongs to invdft
        // and is kept by the adjoint of invdft (a forward pass scaled by 1/n)
        const int inverse = (okind == K_INVDFT) != (vjp != 0);
        const bool scale_blue = okind == K_INVDFT;
        for (int step = 0; step < d && ok; ++step) {
            int a = d - 1 - step;
            const void* sp = step == 0 ? in : out;
            View src = axis_view((void*)sp, D, a, howmany, step == 0 ? idist : odist);
            View dst = axis_view(out, D, a, howmany, odist);
            const AxisPlan& ax = p->axes[a];
            if (ax.n == 1) {
                if (step == 0 && in != out) {
                    // identity axis: the data still has to reach `out`
                    if (d == 1) {
                        ok = cuda_ok(cudaMemcpy2DAsync(out, (size_t)odist * sizeof(cplx_t), in, (size_t)idist * sizeof(cplx_t),
                                                       sizeof(cplx_t), (size_t)howmany, cudaMemcpyDeviceToDevice, stream),
                                     "copy of size-1 transform");
                    } else {
                        OpSpec op;
                        AxisPlan one;
                        one.fft_contig = make_schedule(0, false);
                        one.fft_strided = make_schedule(0, true);
                        ok = run_pow2_axis(p, c, one, src, dst, op, stream);
                    }
                }
                continue;
            }
            if (ax.pow2) {
                OpSpec op;
                op.conj_in = op.conj_out = inverse;
                op.tc = p->form == 1 ? 1 : 0;
                ok = run_pow2_axis(p, c, ax, src, dst, op, stream);
            } else {
                ok = run_bluestein_axis(p, c, ax, src, dst, inverse, scale_blue ? 1.0 / (double)ax.n : 1.0, stream);
            }
        }
    } else if (fam == FAM_REAL) {
        std::vector<long long> H = D;
        H.back() = D.back() / 2 + 1;
        if (kind == K_REALDFT) {
            View src = axis_view((void*)in, D, d - 1, howmany, idist);
            View dst = axis_view(out, H, d - 1, howmany, odist);
            ok = run_real_axis(p, c, p->axes[d - 1], kind, src, dst, vjp, unit_factor, stream);
            for (int a = d - 2; a >= 0 && ok; --a) {
                if (p->axes[a].n == 1) continue;
                View v = axis_view(out, H, a, howmany, odist);
                OpSpec op;
                AxisPlan ax = p->axes[a];
                ok = run_pow2_axis(p, c, ax, v, v, op, stream);
            }
        } else {
            // complex inverse DFTs along the leading axes into a temporary (the
            // caller's input is left untouched), then invrealdft along the last axis
            const void* src_ptr = in;
            long long sdist = idist;
            if (d > 1) {
                long long per = prod(p->dims, 0, d - 1) * H.back();
                size_t bytes = (size_t)per * (size_t)howmany * sizeof(cplx_t);
                if (p->nd_tmp == nullptr || p->nd_tmp_bytes < bytes) {
                    if (p->nd_tmp) cudaFree(p->nd_tmp);
                    p->nd_tmp = nullptr;
                    p->nd_tmp_bytes = 0;
                    if (!cuda_ok(cudaMalloc(&p->nd_tmp, bytes), "cudaMalloc(N-D temporary)")) return last_error();
                    p->nd_tmp_bytes = bytes;
                }
                bool firstc = true;
                for (int a = d - 2; a >= 0 && ok; --a) {
                    if (p->axes[a].n == 1) continue;
                    View vs = axis_view(firstc ? (void*)in : p->nd_tmp, H, a, howmany, firstc ? idist : per);
                    View vd = axis_view(p->nd_tmp, H, a, howmany, per);
                    OpSpec op;
                    op.conj_in = op.conj_out = 1;
                    ok = run_pow2_axis(p, c, p->axes[a], vs, vd, op, stream);
                    firstc = false;
                }
                if (!firstc) {
                    src_ptr = p->nd_tmp;
                    sdist = per;
                }
            }
            View src = axis_view((void*)src_ptr, H, d - 1, howmany, sdist);
            View dst = axis_view(out, D, d - 1, howmany, odist);
            ok = ok && run_real_axis(p, c, p->axes[d - 1], kind, src, dst, vjp, unit_factor, stream);
        }
    } else {
        // real-to-real families: the reference transforms axis k only while the
        // product of the axes after it exceeds 1 (src/07_legacy.h:822-861), so
        // trailing length-1 axes are skipped; length-1 axes before that scale by
        // the 1-D N=1 factor.
        int last = 0;
        for (int i = 0; i < d; ++i)
            if (p->dims[i] != 1) last = i;
        if (d == 1) {
            View src = axis_view((void*)in, D, 0, howmany, idist);
            View dst = axis_view(out, D, 0, howmany, odist);
            ok = run_real_axis(p, c, p->axes[0], kind, src, dst, vjp, unit_factor, stream);
        } else {
            const long long total = prod(p->dims, 0, d);
            bool first = true;
            for (int a = last; a >= 0 && ok; --a) {
                const void* sp = first ? in : out;
                long long sdist = first ? idist : odist;
                if (p->axes[a].n == 1) {
                    ok = launch_tiny((const real_t*)sp, (real_t*)out, howmany, total, sdist, odist, 0, 0,
                                     unit_factor, stream);
                } else {
                    View src = axis_view((void*)sp, D, a, howmany, sdist);
                    View dst = axis_view(out, D, a, howmany, odist);
                    ok = run_real_axis(p, c, p->axes[a], kind, src, dst, vjp, unit_factor, stream);
                }
                first = false;
            }
        }
    }
    if (!ok) return last_error() ? last_error() : 4;
    return 0;
}

// ---------------------------------------------------------------------------
// ragged-batch queue plans (nfft_queue_build.cu)
// ---------------------------------------------------------------------------
notorious_fft_plan* plan_create_queue(int kind, int n, const int* plog, int npass) {
    if (n < 2) {
        set_error(1, "queue plans need n >= 2 (got %d)", n);
        return nullptr;
    }
    const bool pow2 = is_pow2(n);
    if (!pow2 && kind != K_DFT && kind != K_INVDFT && kind != K_REALDFT && kind != K_DCT2) {
        set_error(6, "kind %d of length %d: only dft, invdft, realdft and dct2 accept lengths that are not powers of two",
                  kind, n);
        return nullptr;
    }
    DeviceCtx* c = current_ctx();
    if (!c) return nullptr;
    notorious_fft_plan* p = new notorious_fft_plan();
    p->family = pow2 ? family_of(kind) : FAM_DFT;
    p->device = c->device;
    p->dims.assign(1, n);
    p->axes.resize(1);
    AxisPlan& ax = p->axes[0];
    if (!build_axis(p, c, ax, n, p->family, 12)) {
        plan_destroy(p);
        return nullptr;
    }
    if (npass > 0 && pow2) {
        FftSchedule sch;
        if (!make_split_schedule(ax.fft_contig.logL, plog, npass, &sch)) {
            set_error(1, "pass split does not fit a 2^%d transform", ax.fft_contig.logL);
            plan_destroy(p);
            return nullptr;
        }
        ax.fft_contig = sch;
    }
    if (!pow2 && kind == K_DCT2) {
        bool ok = cuda_ok(cudaMalloc((void**)&ax.post, sizeof(cplx_t) * (size_t)n), "cudaMalloc(post-twiddle)") &&
                  launch_post(ax.post, n, 0) && cuda_ok(cudaDeviceSynchronize(), "post-twiddle table");
        if (!ok) {
            plan_destroy(p);
            return nullptr;
        }
    }
    return p;
}

int plan_record(notorious_fft_plan* p, int kind, const void* in, void* out, long long count, long long idist,
                long long odist) {
    if (!recorder()) {
        set_error(1, "plan_record needs an active recorder");
        return 1;
    }
    const AxisPlan& ax = p->axes[0];
    if (ax.pow2 || kind == K_DFT || kind == K_INVDFT) return plan_execute(p, kind, in, out, count, idist, odist, 0, 0);
    // realdft / DCT-2 of a length that is not a power of two: N-point complex
    // Bluestein of the (reordered) real input with the real-output epilogue
    DeviceCtx* c = device_ctx(p->device);
    if (!c) return last_error();
    std::vector<long long> Din(1, ax.n), Dout(1, kind == K_REALDFT ? ax.n / 2 + 1 : ax.n);
    View src = axis_view((void*)in, Din, 0, count, idist);
    View dst = axis_view(out, Dout, 0, count, odist);
    const int ld = kind == K_REALDFT ? LD_BLUE_R : LD_BLUE_T2;
    const int st = kind == K_REALDFT ? ST_BLUE_R : ST_BLUE_T2;
    if (!run_bluestein_axis(p, c, ax, src, dst, 0, 1.0, 0, ld, st)) return last_error() ? last_error() : 4;
    return 0;
}

}  // namespace nfft

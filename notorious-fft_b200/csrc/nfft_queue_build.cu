// nfft_queue_build.cu -- ragged batches of 1-D transforms run by one
// persistent launch (nfft_queue.h): bucket planning, dependency groups, queue
// order, execution through a CUDA graph, and the autotuner's split cache.
//
// Building a batch:
//  1. transforms with equal (kind, length) form a bucket; each bucket gets a
//     table of its members' input / output offsets (elements of the array type);
//  2. every bucket is planned with the ordinary planner in recording mode
//     (plan_record): the passes it would launch become pass descriptors, with
//     pointers into the caller's buffers stored as offsets (patched per launch)
//     and the batch dim of the lines read from the offset tables;
//  3. a bucket's transforms are split into dependency groups whose tiles never
//     straddle a group boundary; pass k+1 of a group waits on one counter that
//     pass k of the same group publishes;
//  4. the items (runs of tiles) are ordered so that a group's next pass comes
//     `lag` items after its previous one (enough for the earlier pass to have
//     finished on the resident CTAs, few enough that its output is still in L2),
//     with other groups' work in between.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <queue>
#include <string>
#include <vector>

#include "nfft_engine.h"
#include "nfft_queue.h"

namespace nfft {

namespace {

// Recorded pointers in [base, base + span) are offsets into the caller's
// input (IN_BASE) or output (OUT_BASE) buffer.
const uintptr_t IN_BASE = (uintptr_t)1 << 46;
const uintptr_t OUT_BASE = (uintptr_t)1 << 47;
const uintptr_t SPAN = (uintptr_t)1 << 45;

bool pow2(long long n) { return n > 0 && (n & (n - 1)) == 0; }
bool kind_in_cplx(int k) { return k == K_DFT || k == K_INVDFT || k == K_INVREALDFT; }
bool kind_out_cplx(int k) { return k == K_DFT || k == K_INVDFT || k == K_REALDFT; }
long long in_reals_of(int k, long long n) {
    if (k == K_INVREALDFT) return 2 * (n / 2 + 1);
    return kind_in_cplx(k) ? 2 * n : n;
}
long long out_reals_of(int k, long long n) {
    if (k == K_REALDFT) return 2 * (n / 2 + 1);
    return kind_out_cplx(k) ? 2 * n : n;
}
// Length-1 transforms: y = factor * x (the reference's N = 1 cases).
double unit_factor(int k) {
    if (k == K_DCT2 || k == K_DST2) return 2.0;
    if (k == K_DCT4 || k == K_DST4) return 1.41421356237309504880;
    return 1.0;
}
const char* kind_name(int k) {
    static const char* names[10] = {"dft", "invdft", "realdft", "invrealdft", "dct2",
                                    "dst2", "dct3", "dst3", "dct4", "dst4"};
    return (k >= 0 && k < 10) ? names[k] : "?";
}
long long gcd_ll(long long a, long long b) {
    while (b) {
        long long t = a % b;
        a = b;
        b = t;
    }
    return a;
}
long long env_ll(const char* name, long long dflt) {
    const char* e = getenv(name);
    return e ? atoll(e) : dflt;
}

}  // namespace

struct BucketPlan {
    int kind = 0, n = 0;
    std::vector<int> members;
    notorious_fft_plan* plan = nullptr;
    long long* d_tab = nullptr;   // input offsets, then output offsets
};

// Build options (defaults from the environment, see batch_default_options).
struct BatchOptions {
    int use_tuned = 1;           // take pass splits from the tune cache
    // Tiles per item.  Every item is one call of a branch function (a register
    // save / restore of ~350 bytes per thread), so longer runs of tiles amortize
    // it: on B200 the 20,000-transform uneven batch (FP64) took 20.65 ms at 4 / 8,
    // 19.30 at 8 / 8, 18.76 at 16 / 16, 19.08 at 16 / 64, 19.04 at 24 / 24; the
    // 2,000-transform batch 2.48 / 2.45 / 2.99 ms at 4 / 8, 16 / 16, 24 / 24.
    int tiles_multi = 16;        // tiles per item of multi-pass transforms
    int tiles_single = 16;       // tiles per item of single-pass transforms
    long long group_bytes = 4ll << 20;
    long long lag = -1;          // items between dependent passes (-1: 3 x resident CTAs)
    long long spin_limit = 1ll << 22;
    std::vector<int> force_split;   // every power-of-two bucket uses this split (tuner)
};

BatchOptions batch_default_options() {
    BatchOptions o;
    o.tiles_multi = (int)std::max(1ll, env_ll("NOTORIOUS_FFT_QUEUE_TILES_MULTI", 16));
    o.tiles_single = (int)std::max(1ll, env_ll("NOTORIOUS_FFT_QUEUE_TILES_SINGLE", 16));
    o.group_bytes = std::max(1ll, env_ll("NOTORIOUS_FFT_QUEUE_GROUP_KB", 4096)) << 10;
    o.lag = env_ll("NOTORIOUS_FFT_QUEUE_LAG", -1);
    o.spin_limit = std::max(1ll, env_ll("NOTORIOUS_FFT_QUEUE_SPIN", 1ll << 22));
    return o;
}

bool tune_get(int kind, int n, std::vector<int>& split);

}  // namespace nfft

using namespace nfft;

struct notorious_fft_batch {
    int device = -1;
    int count = 0;
    long long in_reals = 0, out_reals = 0;
    bool inplace_ok = false;
    std::vector<BucketPlan> buckets;
    QItem* d_items = nullptr;
    QDesc* d_descs = nullptr;
    unsigned* d_ctr = nullptr;   // counters, then the status word
    std::vector<QItem> items;    // host copy (the test hook edits one item)
    long long nitems = 0, tiles = 0;
    int ndescs = 0, nctr = 0;
    int grid = 0;
    long long spin_limit = 0;
    size_t scratch_bytes = 0;
    long long withhold_spin = 0;   // > 0: the next execution withholds one dependency
    bool use_graph = true;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* g_in = nullptr;
    void* g_out = nullptr;
    long long g_spin = -1;
    void* st_in = nullptr;
    void* st_out = nullptr;
    size_t st_in_bytes = 0, st_out_bytes = 0;
    cudaStream_t last_stream = nullptr;
    std::mutex mu;
};

namespace nfft {

void batch_destroy(notorious_fft_batch* b) {
    if (!b) return;
    int prev = -1;
    cudaGetDevice(&prev);
    if (b->device >= 0 && prev != b->device) cudaSetDevice(b->device);
    for (auto& bk : b->buckets) {
        if (bk.plan) plan_destroy(bk.plan);
        if (bk.d_tab) cudaFree(bk.d_tab);
    }
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_descs) cudaFree(b->d_descs);
    if (b->d_ctr) cudaFree(b->d_ctr);
    if (b->st_in) cudaFree(b->st_in);
    if (b->st_out) cudaFree(b->st_out);
#ifndef NFFT_EMULATE
    if (b->exec) cudaGraphExecDestroy(b->exec);
#endif
    if (b->cap) cudaStreamDestroy(b->cap);
    if (prev >= 0 && prev != b->device) cudaSetDevice(prev);
    delete b;
}

namespace {

// Tiles [a, b) of recorded launch r that belong to transforms [t0, t1) of a
// bucket of `count` transforms.
void tile_range(const RecLaunch& r, long long count, long long t0, long long t1, long long& a, long long& b) {
    if (r.op == QOP_SCALAR) {
        a = t0 / SCALAR_TILE;
        b = (t1 + SCALAR_TILE - 1) / SCALAR_TILE;
        return;
    }
    if (r.op >= QOP_UNPACK_BASE && r.op < QOP_SCALAR) {
        const long long tpl = unpack_tiles_per_line(r.a);
        a = t0 * tpl;
        b = t1 * tpl;
        return;
    }
    const long long lpt = r.a.nlines / count;
    const long long J = 1ll << r.a.logJ;
    a = (t0 * lpt) / J;
    b = (t1 * lpt + J - 1) / J;
}

struct Chain {
    std::vector<std::vector<QItem>> stages;
    long long bytes = 0;
};

void add_items(std::vector<QItem>& out, int op, int desc, long long a, long long b, int per, int wait, int target,
               int done) {
    for (long long t = a; t < b; t += per) {
        QItem it;
        it.op = op;
        it.desc = desc;
        it.tile0 = t;
        it.ntiles = (int)std::min<long long>(per, b - t);
        it.wait = wait;
        it.target = target;
        it.done = done;
        out.push_back(it);
    }
}

bool upload(void** dptr, const void* src, size_t bytes, const char* what) {
    if (!bytes) return true;
    if (!cuda_ok(cudaMalloc(dptr, bytes), what)) return false;
    return cuda_ok(cudaMemcpy(*dptr, src, bytes, cudaMemcpyHostToDevice), what);
}

}  // namespace

notorious_fft_batch* batch_create(int count, const int* kinds, const int* Ns, const long long* ioff,
                                  const long long* ooff, const BatchOptions& opt) {
    if (count < 0 || (count > 0 && (!kinds || !Ns))) {
        set_error(1, "invalid batch description (count %d)", count);
        return nullptr;
    }
    DeviceCtx* c = current_ctx();
    if (!c) return nullptr;
    notorious_fft_batch* b = new notorious_fft_batch();
    b->device = c->device;
    b->count = count;
    b->spin_limit = opt.spin_limit;
    auto fail = [&]() -> notorious_fft_batch* {
        batch_destroy(b);
        return nullptr;
    };
    // ---- offsets and validation
    std::vector<long long> in_off(count), out_off(count);
    long long ip = 0, op = 0;
    b->inplace_ok = true;
    for (int i = 0; i < count; ++i) {
        const int k = kinds[i];
        const long long n = Ns[i];
        if (k < 0 || k > 9 || n < 1) {
            set_error(1, "transform %d: invalid kind %d or length %lld", i, k, n);
            return fail();
        }
        if (n > 1 && !pow2(n) && k != K_DFT && k != K_INVDFT && k != K_REALDFT && k != K_DCT2) {
            set_error(6, "transform %d: %s of length %lld (not a power of two) is not supported", i, kind_name(k), n);
            return fail();
        }
        const long long ni = in_reals_of(k, n), no = out_reals_of(k, n);
        in_off[i] = ioff ? ioff[i] : ip;
        out_off[i] = ooff ? ooff[i] : op;
        ip = in_off[i] + ni + ((in_off[i] + ni) & 1);
        op = out_off[i] + no + ((out_off[i] + no) & 1);
        if (in_off[i] < 0 || out_off[i] < 0 || (kind_in_cplx(k) && (in_off[i] & 1)) ||
            (kind_out_cplx(k) && (out_off[i] & 1))) {
            set_error(1, "transform %d: offsets must be >= 0 and even for complex data", i);
            return fail();
        }
        b->in_reals = std::max(b->in_reals, in_off[i] + ni);
        b->out_reals = std::max(b->out_reals, out_off[i] + no);
        if (in_off[i] != out_off[i] || ni != no) b->inplace_ok = false;
    }
    if (count == 0) return b;
    b->grid = queue_grid(c);
    if (b->grid <= 0) return fail();
    // ---- buckets
    std::map<std::pair<int, int>, int> index;
    for (int i = 0; i < count; ++i) {
        auto key = std::make_pair(kinds[i], Ns[i]);
        auto it = index.find(key);
        if (it == index.end()) {
            index[key] = (int)b->buckets.size();
            BucketPlan bp;
            bp.kind = kinds[i];
            bp.n = Ns[i];
            b->buckets.push_back(bp);
            b->buckets.back().members.push_back(i);
        } else {
            b->buckets[it->second].members.push_back(i);
        }
    }
    std::vector<QDesc> descs;
    std::vector<Chain> chains;
    int nctr = QCTR_FIRST;
    for (auto& bk : b->buckets) {
        const int k = bk.kind;
        const long long cnt = (long long)bk.members.size();
        const bool scalar = bk.n == 1;
        // offset tables: elements of the array type (reals for the size-1 branch)
        const long long iu = (!scalar && kind_in_cplx(k)) ? 2 : 1, ou = (!scalar && kind_out_cplx(k)) ? 2 : 1;
        std::vector<long long> tab(2 * cnt);
        for (long long j = 0; j < cnt; ++j) {
            tab[j] = in_off[bk.members[j]] / iu;
            tab[cnt + j] = out_off[bk.members[j]] / ou;
        }
        if (!upload((void**)&bk.d_tab, tab.data(), tab.size() * sizeof(long long), "offset table upload")) return fail();
        Recorder rec;
        if (scalar) {
            RecLaunch r;
            memset(&r.a, 0, sizeof r.a);
            r.op = QOP_SCALAR;
            r.a.in = (const void*)IN_BASE;
            r.a.out = (void*)OUT_BASE;
            r.a.nlines = cnt;
            r.a.conj_in = kind_in_cplx(k);
            r.a.conj_out = kind_out_cplx(k);
            r.a.dst = (k == K_DFT || k == K_INVDFT) ? 1 : 0;
            r.a.scale = unit_factor(k);
            r.ntiles = (cnt + SCALAR_TILE - 1) / SCALAR_TILE;
            rec.launches.push_back(r);
        } else {
            std::vector<int> split = opt.force_split;
            bool tuned = false;
            if (split.empty() && opt.use_tuned && pow2(bk.n)) tuned = tune_get(k, bk.n, split);
            bk.plan = plan_create_queue(k, bk.n, split.empty() ? nullptr : split.data(), (int)split.size());
            if (!bk.plan && tuned) {
                // a cached split this build cannot execute: use the default schedule
                clear_error();
                bk.plan = plan_create_queue(k, bk.n, nullptr, 0);
            }
            if (!bk.plan) return fail();
            const long long e0 = cnt == 1 ? 1 : 0;   // a single transform: its offset goes into the pointer
            const void* inp = (const void*)(IN_BASE + (uintptr_t)(e0 * in_off[bk.members[0]] * (long long)sizeof(real_t)));
            void* outp = (void*)(OUT_BASE + (uintptr_t)(e0 * out_off[bk.members[0]] * (long long)sizeof(real_t)));
            recorder() = &rec;
            const int rc = plan_record(bk.plan, k, inp, outp, cnt, in_reals_of(k, bk.n) / iu, out_reals_of(k, bk.n) / ou);
            recorder() = nullptr;
            if (rc) return fail();
            b->scratch_bytes += bk.plan->scratch_bytes[0] + bk.plan->scratch_bytes[1];
        }
        // descriptors
        const int desc0 = (int)descs.size();
        for (auto& r : rec.launches) {
            QDesc d;
            memset(&d, 0, sizeof d);
            d.a = r.a;
            d.z = r.z;
            d.zdist = r.zdist;
            const uintptr_t ui = (uintptr_t)r.a.in, uo = (uintptr_t)r.a.out;
            if (ui >= IN_BASE && ui < IN_BASE + SPAN) {
                d.flags |= QD_IN_USER;
                d.a.in = (const void*)(ui - IN_BASE);
            } else if (ui >= OUT_BASE && ui < OUT_BASE + SPAN) {
                set_error(6, "queue plan of %s %d reads its output buffer", kind_name(k), bk.n);
                return fail();
            }
            if (uo >= OUT_BASE && uo < OUT_BASE + SPAN) {
                d.flags |= QD_OUT_USER;
                d.a.out = (void*)(uo - OUT_BASE);
            } else if (uo >= IN_BASE && uo < IN_BASE + SPAN) {
                set_error(6, "queue plan of %s %d writes its input buffer", kind_name(k), bk.n);
                return fail();
            }
            if (r.op == QOP_SCALAR) {
                d.a.in_tab = bk.d_tab;
                d.a.out_tab = bk.d_tab + cnt;
            } else if (cnt > 1 && (d.flags & (QD_IN_USER | QD_OUT_USER))) {
                const int bd = d.a.ndims - 1;
                if (bd < 0 || d.a.cnt[bd] != cnt || d.a.jpos == bd) {
                    set_error(6, "unexpected line layout in the queue plan of %s %d", kind_name(k), bk.n);
                    return fail();
                }
                d.a.tab_dim = bd;
                if (d.flags & QD_IN_USER) d.a.in_tab = bk.d_tab;
                if (d.flags & QD_OUT_USER) d.a.out_tab = bk.d_tab + cnt;
            }
            if (r.op != QOP_SCALAR && !(r.op >= QOP_UNPACK_BASE && r.op < QOP_SCALAR) && r.a.nlines % cnt) {
                set_error(6, "queue plan of %s %d: lines do not divide into transforms", kind_name(k), bk.n);
                return fail();
            }
            descs.push_back(d);
        }
        // dependency groups: multiples of g0 transforms keep tiles inside a group
        const int K = (int)rec.launches.size();
        long long g0 = 1;
        for (auto& r : rec.launches) {
            if (r.op == QOP_SCALAR || (r.op >= QOP_UNPACK_BASE && r.op < QOP_SCALAR)) continue;
            const long long J = 1ll << r.a.logJ, lpt = r.a.nlines / cnt;
            const long long need = J / gcd_ll(J, lpt);
            g0 = g0 / gcd_ll(g0, need) * need;
        }
        long long G = cnt;
        if (K > 1) {
            const long long per = std::max(1ll, (long long)bk.n * (long long)sizeof(cplx_t));
            G = std::max(g0, opt.group_bytes / per / g0 * g0);
            if (G > cnt) G = cnt;
        }
        const int per_item = K > 1 ? opt.tiles_multi : opt.tiles_single;
        for (long long t0 = 0; t0 < cnt; t0 += G) {
            const long long t1 = std::min(cnt, t0 + G);
            Chain ch;
            ch.bytes = (t1 - t0) * (long long)bk.n;
            int prev_ctr = -1, prev_tiles = 0;
            for (int kk = 0; kk < K; ++kk) {
                long long a, e;
                tile_range(rec.launches[kk], cnt, t0, t1, a, e);
                const int done = kk + 1 < K ? nctr++ : -1;
                std::vector<QItem> st;
                add_items(st, rec.launches[kk].op, desc0 + kk, a, e, per_item, prev_ctr, prev_tiles, done);
                b->tiles += e - a;
                ch.stages.push_back(std::move(st));
                prev_ctr = done;
                prev_tiles = (int)(e - a);
            }
            chains.push_back(std::move(ch));
        }
    }
    // ---- queue order: multi-pass chains first (largest first), then the
    // single-pass ones; a chain's pass k+1 is released `lag` items after pass k
    std::stable_sort(chains.begin(), chains.end(), [](const Chain& x, const Chain& y) {
        if (x.stages.size() != y.stages.size()) return x.stages.size() > y.stages.size();
        return x.bytes > y.bytes;
    });
    const long long lag = opt.lag >= 0 ? opt.lag : 3ll * b->grid;
    struct Pending {
        long long release, seq;
        int chain, stage;
        bool operator>(const Pending& o) const { return release != o.release ? release > o.release : seq > o.seq; }
    };
    std::priority_queue<Pending, std::vector<Pending>, std::greater<Pending>> pend;
    long long seq = 0;
    size_t next = 0;
    while (next < chains.size() || !pend.empty()) {
        int ci, si;
        if (!pend.empty() && (pend.top().release <= (long long)b->items.size() || next >= chains.size())) {
            ci = pend.top().chain;
            si = pend.top().stage;
            pend.pop();
        } else {
            ci = (int)next++;
            si = 0;
        }
        auto& st = chains[ci].stages[si];
        b->items.insert(b->items.end(), st.begin(), st.end());
        if (si + 1 < (int)chains[ci].stages.size())
            pend.push(Pending{(long long)b->items.size() + lag, seq++, ci, si + 1});
    }
    b->nitems = (long long)b->items.size();
    b->ndescs = (int)descs.size();
    b->nctr = nctr;
    if (b->nitems >= (1ll << 31)) {
        set_error(6, "ragged batch of %lld items exceeds the queue's claim counter", b->nitems);
        return fail();
    }
    if (!upload((void**)&b->d_items, b->items.data(), b->items.size() * sizeof(QItem), "queue item upload") ||
        !upload((void**)&b->d_descs, descs.data(), descs.size() * sizeof(QDesc), "queue descriptor upload"))
        return fail();
    if (!cuda_ok(cudaMalloc((void**)&b->d_ctr, sizeof(unsigned) * (size_t)(nctr + 1)), "cudaMalloc(queue counters)"))
        return fail();
    if (!cuda_ok(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking), "cudaStreamCreate")) return fail();
    return b;
}

// ---- execution ---------------------------------------------------------------

static QueueArgs batch_args(notorious_fft_batch* b, const void* din, void* dout, long long spin) {
    QueueArgs q;
    q.items = b->d_items;
    q.nitems = b->nitems;
    q.descs = b->d_descs;
    q.ctr = b->d_ctr;
    q.status = (int*)(b->d_ctr + b->nctr);
    q.user_in = din;
    q.user_out = dout;
    q.spin_limit = spin;
    return q;
}

static bool batch_enqueue(notorious_fft_batch* b, const QueueArgs& q, cudaStream_t s) {
    return cuda_ok(cudaMemsetAsync(b->d_ctr, 0, sizeof(unsigned) * (size_t)(b->nctr + 1), s), "queue counter reset") &&
           launch_queue(q, b->grid, s);
}

// Device pointers, asynchronous on s.
int batch_run(notorious_fft_batch* b, const void* din, void* dout, cudaStream_t s) {
    if (b->nitems == 0) return 0;
    const size_t ib = (size_t)b->in_reals * sizeof(real_t), ob = (size_t)b->out_reals * sizeof(real_t);
    const char *i0 = (const char*)din, *o0 = (const char*)dout;
    if (din == dout ? !b->inplace_ok : (i0 < o0 + ob && o0 < i0 + ib)) {
        set_error(1, "batch input and output overlap (in place needs every transform to map onto itself)");
        return 1;
    }
    long long spin = b->spin_limit;
    bool withhold = b->withhold_spin > 0;
    long long witem = -1;
    if (withhold) {
        spin = b->withhold_spin;
        for (long long i = 0; i < b->nitems; ++i)
            if (b->items[i].wait >= 0) {
                witem = i;
                break;
            }
        if (witem < 0) {
            set_error(6, "the batch has no dependent item to withhold");
            return 6;
        }
        QItem it = b->items[witem];
        it.target += 1;   // a count that is never reached
        if (!cuda_ok(cudaMemcpy(&b->d_items[witem], &it, sizeof it, cudaMemcpyHostToDevice), "queue item edit")) return 4;
    }
    const QueueArgs q = batch_args(b, din, dout, spin);
    bool ok = true;
#ifndef NFFT_EMULATE
    if (b->use_graph && !withhold) {
        if (!b->exec || b->g_in != din || b->g_out != dout || b->g_spin != spin) {
            if (b->exec) cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
            cudaGraph_t g = nullptr;
            ok = cuda_ok(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
            if (ok) {
                bool rec = batch_enqueue(b, q, b->cap);
                ok = cuda_ok(cudaStreamEndCapture(b->cap, &g), "cudaStreamEndCapture") && rec;
            }
            ok = ok && cuda_ok(cudaGraphInstantiate(&b->exec, g, 0), "cudaGraphInstantiate");
            if (g) cudaGraphDestroy(g);
            if (!ok) return last_error() ? last_error() : 4;
            b->g_in = din;
            b->g_out = dout;
            b->g_spin = spin;
        }
        ok = cuda_ok(cudaGraphLaunch(b->exec, s), "cudaGraphLaunch");
    } else {
        ok = batch_enqueue(b, q, s);
    }
#else
    ok = batch_enqueue(b, q, s);
#endif
    if (ok) note_launch();
    b->last_stream = s;
    if (withhold) {
        // restore the item once the launch is over
        ok = cuda_ok(cudaStreamSynchronize(s), "stream synchronize") && ok;
        ok = cuda_ok(cudaMemcpy(&b->d_items[witem], &b->items[witem], sizeof(QItem), cudaMemcpyHostToDevice),
                     "queue item restore") && ok;
        b->withhold_spin = 0;
    }
    return ok ? 0 : (last_error() ? last_error() : 4);
}

// Wait for the last launch; TIMEOUT if one of its waits gave up.
int batch_status(notorious_fft_batch* b) {
    if (b->nitems == 0) return 0;
    if (!cuda_ok(cudaStreamSynchronize(b->last_stream), "stream synchronize")) return last_error();
    int st = 0;
    if (!cuda_ok(cudaMemcpy(&st, b->d_ctr + b->nctr, sizeof st, cudaMemcpyDeviceToHost), "queue status read"))
        return last_error();
    if (st) {
        set_error(5, "ragged batch: a dependency wait of item %d gave up; the launch was abandoned", st - 1);
        return 5;
    }
    return 0;
}

static bool grow_dev(void** buf, size_t* have, size_t need) {
    if (*have >= need && *buf) return true;
    if (*buf) cudaFree(*buf);
    *buf = nullptr;
    *have = 0;
    if (!cuda_ok(cudaMalloc(buf, need), "cudaMalloc(batch staging)")) return false;
    *have = need;
    return true;
}

// Host pointers: staged through device buffers, synchronous.
int batch_run_host(notorious_fft_batch* b, const void* hin, void* hout, cudaStream_t s) {
    if (b->nitems == 0) return 0;
    const size_t ib = (size_t)b->in_reals * sizeof(real_t), ob = (size_t)b->out_reals * sizeof(real_t);
    if (!grow_dev(&b->st_in, &b->st_in_bytes, std::max<size_t>(ib, 16)) ||
        !grow_dev(&b->st_out, &b->st_out_bytes, std::max<size_t>(ob, 16)))
        return last_error();
    if (!cuda_ok(cudaMemcpyAsync(b->st_in, hin, ib, cudaMemcpyHostToDevice, s), "H2D copy")) return last_error();
    int rc = batch_run(b, b->st_in, b->st_out, s);
    if (rc) return rc;
    if (!cuda_ok(cudaMemcpyAsync(hout, b->st_out, ob, cudaMemcpyDeviceToHost, s), "D2H copy")) return last_error();
    return batch_status(b);
}

// ---- autotuner cache -----------------------------------------------------------

namespace {
std::mutex g_tune_mu;
bool g_tune_loaded = false;
std::map<std::string, std::vector<int>> g_tune;   // key -> split
std::map<std::string, int> g_tune_logt;           // key -> threads (log2) of standalone plans, 0: default
std::map<std::string, std::string> g_tune_lines;  // key -> file line of this device (kept on save)
std::vector<std::string> g_tune_foreign;          // lines of other devices (kept verbatim)

std::string tune_path() {
    const char* e = getenv("NOTORIOUS_FFT_TUNE_CACHE");
    if (e && *e) return e;
    const char* h = getenv("HOME");
    return std::string(h && *h ? h : ".") + "/.cache/notorious_fft/tune.json";
}

std::string device_tag() {
    int dev = 0, drv = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    memset(&prop, 0, sizeof prop);
    cudaGetDeviceProperties(&prop, dev);
    cudaDriverGetVersion(&drv);
    char buf[320];
    snprintf(buf, sizeof buf, "%s sm_%d%d driver %d", prop.name, prop.major, prop.minor, drv);
    for (char* p = buf; *p; ++p)
        if (*p == '"' || *p == '\\') *p = '_';
    return buf;
}

std::string tune_key(int kind, int n) {
    return std::string(sizeof(real_t) == 8 ? "f64:" : "f32:") + kind_name(kind) + ":" + std::to_string(n);
}

// Standalone plans are keyed by transform family: the inner FFT schedule of a
// power-of-two axis is shared by the kinds of a family.
const char* family_name(int fam) {
    switch (fam) {
    case FAM_DFT: return "dft";
    case FAM_REAL: return "realdft";
    case FAM_T2T3: return "t2t3";
    default: return "t4";
    }
}
std::string tune_key_plan(int fam, int n) {
    return std::string(sizeof(real_t) == 8 ? "f64:plan:" : "f32:plan:") + family_name(fam) + ":" + std::to_string(n);
}

// The string value of "name": "..." in line, or "".
std::string json_str(const std::string& line, const char* name) {
    std::string pat = std::string("\"") + name + "\": \"";
    size_t p = line.find(pat);
    if (p == std::string::npos) return "";
    p += pat.size();
    size_t q = line.find('"', p);
    return q == std::string::npos ? "" : line.substr(p, q - p);
}

void tune_load_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    FILE* f = fopen(tune_path().c_str(), "r");
    if (!f) return;
    const std::string tag = device_tag();
    char buf[1024];
    while (fgets(buf, sizeof buf, f)) {
        std::string line(buf);
        while (!line.empty() && (line.back() == '\n' || line.back() == '\r' || line.back() == ',')) line.pop_back();
        std::string key = json_str(line, "key"), dev = json_str(line, "device");
        if (key.empty()) continue;
        if (dev != tag) {
            g_tune_foreign.push_back(line);
            continue;
        }
        size_t p = line.find("\"split\": [");
        if (p == std::string::npos) continue;
        std::vector<int> split;
        const char* s = line.c_str() + p + 10;
        while (*s && *s != ']') {
            char* end = nullptr;
            long v = strtol(s, &end, 10);
            if (end == s) break;
            split.push_back((int)v);
            s = end;
            while (*s == ',' || *s == ' ') ++s;
        }
        // plan entries may carry an empty split (the default schedule) and a
        // thread count; queue entries always name a split
        const bool plan = key.find(":plan:") != std::string::npos;
        if (!split.empty() || plan) {
            g_tune[key] = split;
            g_tune_lines[key] = line;
            size_t q = line.find("\"logt\": ");
            g_tune_logt[key] = q == std::string::npos ? 0 : atoi(line.c_str() + q + 8);
        }
    }
    fclose(f);
}

bool tune_save_locked() {
    const std::string path = tune_path();
    // create the parent directories (existing ones make mkdir fail harmlessly)
    for (size_t p = path.find('/', 1); p != std::string::npos; p = path.find('/', p + 1))
        mkdir(path.substr(0, p).c_str(), 0755);
    std::string tmp = path + ".tmp";
    FILE* f = fopen(tmp.c_str(), "w");
    if (!f) return false;
    fprintf(f, "{\"format\": \"notorious_fft tune cache 1\", \"entries\": [\n");
    bool first = true;
    for (auto& l : g_tune_foreign) {
        fprintf(f, "%s%s", first ? "" : ",\n", l.c_str());
        first = false;
    }
    for (auto& kv : g_tune_lines) {
        fprintf(f, "%s%s", first ? "" : ",\n", kv.second.c_str());
        first = false;
    }
    fprintf(f, "\n]}\n");
    fclose(f);
    return rename(tmp.c_str(), path.c_str()) == 0;
}

}  // namespace

bool tune_get(int kind, int n, std::vector<int>& split) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    auto it = g_tune.find(tune_key(kind, n));
    if (it == g_tune.end()) return false;
    split = it->second;
    return true;
}

bool tune_get_plan(int fam, int n, std::vector<int>& split, int& logt) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    const std::string key = tune_key_plan(fam, n);
    auto it = g_tune.find(key);
    if (it == g_tune.end()) return false;
    split = it->second;
    auto lt = g_tune_logt.find(key);
    logt = lt == g_tune_logt.end() ? 0 : lt->second;
    return true;
}

static void tune_put_plan(int fam, int n, const std::vector<int>& split, int logt, double us) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    const std::string key = tune_key_plan(fam, n);
    std::string sp;
    for (size_t i = 0; i < split.size(); ++i) sp += (i ? ", " : "") + std::to_string(split[i]);
    char buf[768];
    snprintf(buf, sizeof buf, "{\"device\": \"%s\", \"key\": \"%s\", \"split\": [%s], \"logt\": %d, \"us\": %.2f}",
             device_tag().c_str(), key.c_str(), sp.c_str(), logt, us);
    g_tune[key] = split;
    g_tune_logt[key] = logt;
    g_tune_lines[key] = buf;
    tune_save_locked();
}

static void tune_put(int kind, int n, const std::vector<int>& split, double us) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    const std::string key = tune_key(kind, n);
    std::string sp;
    for (size_t i = 0; i < split.size(); ++i) sp += (i ? ", " : "") + std::to_string(split[i]);
    char buf[768];
    snprintf(buf, sizeof buf, "{\"device\": \"%s\", \"key\": \"%s\", \"split\": [%s], \"us\": %.2f}",
             device_tag().c_str(), key.c_str(), sp.c_str(), us);
    g_tune[key] = split;
    g_tune_lines[key] = buf;
    tune_save_locked();
}

// Executable splits of a 2^logL inner FFT, most balanced first.
static std::vector<std::vector<int>> tune_candidates(int logL) {
    const int lim = 12 - (sizeof(real_t) == 8 ? 2 : 3);
    std::vector<std::vector<int>> c;
    if (logL <= 12) c.push_back({logL});
    for (int r1 = 1; r1 < logL; ++r1) {
        const int r2 = logL - r1;
        if (r1 <= lim && r2 <= lim && r1 >= 4 && r2 >= 4) c.push_back({r1, r2});
    }
    if (c.empty()) c.push_back({});   // default schedule (three or more passes)
    std::stable_sort(c.begin(), c.end(), [](const std::vector<int>& x, const std::vector<int>& y) {
        auto spread = [](const std::vector<int>& v) { return v.size() < 2 ? 0 : std::abs(v[0] - v[1]); };
        if (x.size() != y.size()) return x.size() < y.size();
        return spread(x) < spread(y);
    });
    if (c.size() > 5) c.resize(5);
    return c;
}

// Standalone plans of (family of kind, n): time the default schedule and the
// executable pass splits, each with the default thread rule and with 128- and
// 256-thread pass kernels, on a ~256 MB batch of `kind`; store the fastest.
static int autotune_plan(int kind, int n, cudaStream_t s) {
    const int fam = family_of(kind);
    int logn = 0;
    while ((1 << logn) < n) ++logn;
    const int logL = fam == FAM_DFT ? logn : logn - 1;
    std::vector<std::vector<int>> splits = {{}};   // {} = the default schedule
    for (auto& c : tune_candidates(logL))
        if (!c.empty()) splits.push_back(c);
    const int logts[3] = {0, 7, 8};
    const long long bytes = (in_reals_of(kind, n) + out_reals_of(kind, n)) * (long long)sizeof(real_t);
    const long long cnt = std::max(1ll, (256ll << 20) / bytes);
    void *din = nullptr, *dout = nullptr;
    const size_t ib = (size_t)cnt * (size_t)in_reals_of(kind, n) * sizeof(real_t);
    const size_t ob = (size_t)cnt * (size_t)out_reals_of(kind, n) * sizeof(real_t);
    if (!cuda_ok(cudaMalloc(&din, ib), "cudaMalloc(tune input)")) return last_error();
    if (!cuda_ok(cudaMalloc(&dout, ob), "cudaMalloc(tune output)")) {
        cudaFree(din);
        return last_error();
    }
    cudaMemsetAsync(din, 0, ib, s);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e30;
    std::vector<int> best_split;
    int best_logt = 0, rc = 0;
    for (auto& split : splits) {
        for (int lt : logts) {
            PlanOverride o;
            o.split = split;
            o.logt = lt;
            plan_override() = &o;
            notorious_fft_plan* p = plan_create(fam, 1, &n);
            plan_override() = nullptr;
            if (!p) {
                clear_error();
                continue;
            }
            const long long ie = plan_in_elems(p, kind), oe = plan_out_elems(p, kind);
            std::vector<float> ms;
            bool ok = true;
            for (int it = 0; it < 7 && ok; ++it) {
                cudaEventRecord(e0, s);
                ok = plan_execute(p, kind, din, dout, cnt, ie, oe, s, 0) == 0;
                cudaEventRecord(e1, s);
                ok = ok && cuda_ok(cudaEventSynchronize(e1), "tune timing");
                float t = 0;
                cudaEventElapsedTime(&t, e0, e1);
                if (it >= 2) ms.push_back(t);
            }
            plan_destroy(p);
            if (!ok) {
                rc = last_error() ? last_error() : 4;
                break;
            }
            std::sort(ms.begin(), ms.end());
            const double med = ms.empty() ? 1e30 : ms[ms.size() / 2];
            if (med < best) {
                best = med;
                best_split = split;
                best_logt = lt;
            }
        }
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(din);
    cudaFree(dout);
    if (rc) return rc;
    if (best < 1e30) tune_put_plan(fam, n, best_split, best_logt, best * 1000.0 / (double)cnt);
    return 0;
}

int tune_lookup_plan(int kind, int n, int* plog, int max_passes, int* logt) {
    std::vector<int> split;
    int lt = 0;
    if (kind < 0 || kind > 9 || !tune_get_plan(family_of(kind), n, split, lt)) return -1;
    for (int i = 0; i < (int)split.size() && i < max_passes; ++i) plog[i] = split[i];
    if (logt) *logt = lt;
    return (int)split.size();
}

int autotune(int kind, int n, cudaStream_t s) {
    if (kind < 0 || kind > 9 || n < 2 || !pow2(n)) {
        set_error(1, "autotune needs a power-of-two length >= 2 and a valid kind");
        return 1;
    }
    int logn = 0;
    while ((1 << logn) < n) ++logn;
    const int logL = (kind == K_DFT || kind == K_INVDFT) ? logn : logn - 1;
    auto cands = tune_candidates(logL);
    const long long bytes = (in_reals_of(kind, n) + out_reals_of(kind, n)) * (long long)sizeof(real_t);
    const long long cnt = std::max(1ll, (256ll << 20) / bytes);
    std::vector<int> kinds((size_t)cnt, kind), Ns((size_t)cnt, n);
    void *din = nullptr, *dout = nullptr;
    const size_t ib = (size_t)cnt * (size_t)(in_reals_of(kind, n) + 1) * sizeof(real_t);
    const size_t ob = (size_t)cnt * (size_t)(out_reals_of(kind, n) + 1) * sizeof(real_t);
    if (!cuda_ok(cudaMalloc(&din, ib), "cudaMalloc(tune input)")) return last_error();
    if (!cuda_ok(cudaMalloc(&dout, ob), "cudaMalloc(tune output)")) {
        cudaFree(din);
        return last_error();
    }
    cudaMemsetAsync(din, 0, ib, s);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e30;
    std::vector<int> best_split;
    int rc = 0;
    for (auto& cand : cands) {
        BatchOptions o = batch_default_options();
        o.use_tuned = 0;
        o.force_split = cand;
        notorious_fft_batch* b = batch_create((int)cnt, kinds.data(), Ns.data(), nullptr, nullptr, o);
        if (!b) {
            clear_error();
            continue;
        }
        b->use_graph = false;
        std::vector<float> ms;
        bool ok = true;
        for (int it = 0; it < 7 && ok; ++it) {
            cudaEventRecord(e0, s);
            ok = batch_run(b, din, dout, s) == 0;
            cudaEventRecord(e1, s);
            ok = ok && batch_status(b) == 0;
            float t = 0;
            cudaEventElapsedTime(&t, e0, e1);
            if (it >= 2) ms.push_back(t);
        }
        batch_destroy(b);
        if (!ok) {
            rc = last_error() ? last_error() : 4;
            break;
        }
        std::sort(ms.begin(), ms.end());
        const double med = ms.empty() ? 1e30 : ms[ms.size() / 2];
        if (med < best) {
            best = med;
            best_split = cand;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(din);
    cudaFree(dout);
    if (rc) return rc;
    if (!best_split.empty()) tune_put(kind, n, best_split, best * 1000.0 / (double)cnt);
    // (the queue has no other choice than the default schedule otherwise)
    return autotune_plan(kind, n, s);
}

int tune_lookup(int kind, int n, int* plog, int max_passes) {
    std::vector<int> split;
    if (!tune_get(kind, n, split)) return 0;
    for (int i = 0; i < (int)split.size() && i < max_passes; ++i) plog[i] = split[i];
    return (int)split.size();
}

notorious_fft_batch* batch_create_default(int count, const int* kinds, const int* Ns, const long long* in_off,
                                          const long long* out_off) {
    return batch_create(count, kinds, Ns, in_off, out_off, batch_default_options());
}
long long batch_in_reals(const notorious_fft_batch* b) { return b->in_reals; }
long long batch_out_reals(const notorious_fft_batch* b) { return b->out_reals; }
void batch_info(const notorious_fft_batch* b, long long* items, long long* tiles, long long* scratch, int* ctas) {
    if (items) *items = b->nitems;
    if (tiles) *tiles = b->tiles;
    if (scratch) *scratch = (long long)b->scratch_bytes;
    if (ctas) *ctas = b->grid;
}
void batch_set_graph(notorious_fft_batch* b, int enable) { b->use_graph = enable != 0; }
void batch_withhold(notorious_fft_batch* b, long long spin_limit) { b->withhold_spin = std::max(1ll, spin_limit); }

}  // namespace nfft

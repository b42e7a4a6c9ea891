// nfft_queue.h -- the persistent work queue for ragged batches (internal).
//
// A ragged batch is a list of independent 1-D transforms of mixed kinds and
// lengths.  The builder (nfft_queue_build.cu) groups equal (kind, length)
// transforms into buckets, plans every bucket with the ordinary pass planner
// in recording mode (256-thread tiles), and turns each recorded launch into
// queue items: runs of tiles of one pass for one dependency group of
// transforms.  One persistent kernel (nfft_queue_kernel.cu) executes all
// items: each CTA claims items in queue order with an atomic counter, waits
// (bounded) until the previous pass of the same group has published all its
// tiles, runs the tiles, and publishes them.  Items only ever wait on items
// earlier in the queue, so a claimed item always makes progress.
#pragma once

#include "nfft_pass.cuh"

namespace nfft {

// One claimable unit of work.
struct QItem {
    int op;          // branch of the queue kernel (QOP_* key)
    int desc;        // pass descriptor
    long long tile0; // first tile of the run
    int ntiles;
    int wait;        // counter that must reach `target` first (-1: none)
    int target;
    int done;        // counter that receives ntiles when the run is finished (-1: none)
};

// One recorded pass.  flags: QD_IN_USER / QD_OUT_USER mark a.in / a.out as
// byte offsets from the caller's input / output buffer (patched per launch).
enum { QD_IN_USER = 1, QD_OUT_USER = 2 };
struct QDesc {
    PassArgs a;
    const void* z;       // unpack: packed spectrum (scratch), line distance zdist
    long long zdist;
    int flags;
    int pad;
};

// Counters: [0] next item to claim, [1] abort flag; per-group counters follow.
constexpr int QCTR_NEXT = 0, QCTR_ABORT = 1, QCTR_FIRST = 2;

struct QueueArgs {
    const QItem* items;
    long long nitems;
    const QDesc* descs;
    unsigned int* ctr;
    int* status;           // item + 1 of the first wait that gave up; 0 when none did
    const void* user_in;
    void* user_out;
    long long spin_limit;  // polls of one wait before the launch is abandoned
};

// Tile shape of every queue branch: 256 threads, 4096 points.
constexpr int QUEUE_LOGT = 8;
constexpr int QUEUE_THREADS = 1 << QUEUE_LOGT;
constexpr int QUEUE_LOG_TILE = 12;

// Specialized (lean) branches: X(LOGR, COL_IN, COL_OUT, LOAD, STORE), in four
// families (each compiled in its own translation unit, nfft_queue_b*.cu).
// Complex passes: single-pass rows, first (column in / row out) passes.
#define NFFT_QUEUE_LEAN_A(X)                                                                        \
    X(4, 0, 0, LD_C, ST_C) X(5, 0, 0, LD_C, ST_C) X(6, 0, 0, LD_C, ST_C) X(7, 0, 0, LD_C, ST_C)     \
    X(8, 0, 0, LD_C, ST_C) X(9, 0, 0, LD_C, ST_C) X(10, 0, 0, LD_C, ST_C) X(11, 0, 0, LD_C, ST_C)   \
    X(12, 0, 0, LD_C, ST_C)                                                                         \
    X(5, 1, 0, LD_C, ST_C) X(6, 1, 0, LD_C, ST_C) X(7, 1, 0, LD_C, ST_C) X(8, 1, 0, LD_C, ST_C)     \
    X(9, 1, 0, LD_C, ST_C) X(10, 1, 0, LD_C, ST_C)
// Complex column/column passes; first and last (mirror-tile unpack) passes of
// multi-pass realdft and DCT-2.
#define NFFT_QUEUE_LEAN_B(X)                                                                        \
    X(4, 1, 1, LD_C, ST_C) X(5, 1, 1, LD_C, ST_C) X(6, 1, 1, LD_C, ST_C) X(7, 1, 1, LD_C, ST_C)     \
    X(8, 1, 1, LD_C, ST_C) X(9, 1, 1, LD_C, ST_C) X(10, 1, 1, LD_C, ST_C)                           \
    X(5, 1, 0, LD_R2C, ST_C) X(6, 1, 0, LD_R2C, ST_C) X(7, 1, 0, LD_R2C, ST_C)                      \
    X(8, 1, 0, LD_R2C, ST_C) X(9, 1, 0, LD_R2C, ST_C) X(10, 1, 0, LD_R2C, ST_C)                     \
    X(5, 1, 0, LD_T2, ST_C) X(6, 1, 0, LD_T2, ST_C) X(7, 1, 0, LD_T2, ST_C)                         \
    X(8, 1, 0, LD_T2, ST_C) X(9, 1, 0, LD_T2, ST_C) X(10, 1, 0, LD_T2, ST_C)                         \
    X(4, 1, 1, LD_C, ST_R) X(5, 1, 1, LD_C, ST_R) X(6, 1, 1, LD_C, ST_R) X(7, 1, 1, LD_C, ST_R)     \
    X(8, 1, 1, LD_C, ST_R) X(9, 1, 1, LD_C, ST_R) X(10, 1, 1, LD_C, ST_R)                           \
    X(4, 1, 1, LD_C, ST_T2) X(5, 1, 1, LD_C, ST_T2) X(6, 1, 1, LD_C, ST_T2) X(7, 1, 1, LD_C, ST_T2) \
    X(8, 1, 1, LD_C, ST_T2) X(9, 1, 1, LD_C, ST_T2) X(10, 1, 1, LD_C, ST_T2)
// Single-pass realdft and DCT-2 / DST-2.
#define NFFT_QUEUE_LEAN_C(X)                                                                        \
    X(4, 0, 0, LD_R2C, ST_R) X(5, 0, 0, LD_R2C, ST_R) X(6, 0, 0, LD_R2C, ST_R)                      \
    X(7, 0, 0, LD_R2C, ST_R) X(8, 0, 0, LD_R2C, ST_R) X(9, 0, 0, LD_R2C, ST_R)                      \
    X(10, 0, 0, LD_R2C, ST_R) X(11, 0, 0, LD_R2C, ST_R) X(12, 0, 0, LD_R2C, ST_R)                   \
    X(4, 0, 0, LD_T2, ST_T2) X(5, 0, 0, LD_T2, ST_T2) X(6, 0, 0, LD_T2, ST_T2)                      \
    X(7, 0, 0, LD_T2, ST_T2) X(8, 0, 0, LD_T2, ST_T2) X(9, 0, 0, LD_T2, ST_T2)                      \
    X(10, 0, 0, LD_T2, ST_T2) X(11, 0, 0, LD_T2, ST_T2) X(12, 0, 0, LD_T2, ST_T2)
// Multi-pass Bluestein: chirp-premultiplied first forward passes, the filter
// product fused into the first inverse pass, window + chirp in the last one.
#define NFFT_QUEUE_LEAN_D(X)                                                                        \
    X(6, 1, 0, LD_BLUE, ST_C) X(7, 1, 0, LD_BLUE, ST_C) X(8, 1, 0, LD_BLUE, ST_C)                   \
    X(9, 1, 0, LD_BLUE, ST_C) X(10, 1, 0, LD_BLUE, ST_C)                                            \
    X(6, 1, 0, LD_BLUE_R, ST_C) X(7, 1, 0, LD_BLUE_R, ST_C) X(8, 1, 0, LD_BLUE_R, ST_C)             \
    X(9, 1, 0, LD_BLUE_R, ST_C) X(10, 1, 0, LD_BLUE_R, ST_C)                                        \
    X(6, 1, 0, LD_BLUE_T2, ST_C) X(7, 1, 0, LD_BLUE_T2, ST_C) X(8, 1, 0, LD_BLUE_T2, ST_C)          \
    X(9, 1, 0, LD_BLUE_T2, ST_C) X(10, 1, 0, LD_BLUE_T2, ST_C)                                      \
    X(5, 1, 0, LD_FILT, ST_C) X(6, 1, 0, LD_FILT, ST_C) X(7, 1, 0, LD_FILT, ST_C)                   \
    X(8, 1, 0, LD_FILT, ST_C) X(9, 1, 0, LD_FILT, ST_C) X(10, 1, 0, LD_FILT, ST_C)                  \
    X(6, 1, 1, LD_C, ST_BLUE) X(7, 1, 1, LD_C, ST_BLUE) X(8, 1, 1, LD_C, ST_BLUE)                   \
    X(9, 1, 1, LD_C, ST_BLUE) X(10, 1, 1, LD_C, ST_BLUE)                                            \
    X(6, 1, 1, LD_C, ST_BLUE_R) X(7, 1, 1, LD_C, ST_BLUE_R) X(8, 1, 1, LD_C, ST_BLUE_R)             \
    X(9, 1, 1, LD_C, ST_BLUE_R) X(10, 1, 1, LD_C, ST_BLUE_R)                                        \
    X(6, 1, 1, LD_C, ST_BLUE_T2) X(7, 1, 1, LD_C, ST_BLUE_T2) X(8, 1, 1, LD_C, ST_BLUE_T2)          \
    X(9, 1, 1, LD_C, ST_BLUE_T2) X(10, 1, 1, LD_C, ST_BLUE_T2)
#define NFFT_QUEUE_LEAN(X) NFFT_QUEUE_LEAN_A(X) NFFT_QUEUE_LEAN_B(X) NFFT_QUEUE_LEAN_C(X) NFFT_QUEUE_LEAN_D(X)

// Generic branches (4096-point tile, any pass radix): X(LOAD, STORE).
#define NFFT_QUEUE_GENERIC(X)                                                                       \
    X(LD_C, ST_C) X(LD_C, ST_T3) X(LD_C, ST_T4) X(LD_C, ST_BLUE) X(LD_T2, ST_C) X(LD_T2, ST_T2)     \
    X(LD_T3, ST_C) X(LD_T3, ST_T3) X(LD_IR, ST_C) X(LD_T4, ST_C) X(LD_T4, ST_T4) X(LD_BLUE, ST_C)   \
    X(LD_BLUE, ST_BLUE) X(LD_R2C, ST_C) X(LD_R2C, ST_R) X(LD_C, ST_C2R) X(LD_IR, ST_C2R)            \
    X(LD_BLUE_R, ST_C) X(LD_BLUE_R, ST_BLUE_R) X(LD_C, ST_BLUE_R) X(LD_BLUE_T2, ST_C)               \
    X(LD_BLUE_T2, ST_BLUE_T2) X(LD_C, ST_BLUE_T2) X(LD_FILT, ST_C)

// Branch keys.
constexpr int QOP_LEAN_BASE = 0x100000, QOP_GEN_BASE = 0x200000, QOP_UNPACK_BASE = 0x300000;
constexpr int QOP_SCALAR = 0x400000;
NFFT_HD constexpr int qop_lean(int logR, int ci, int co, int ld, int st) {
    return QOP_LEAN_BASE | logR | (ci << 5) | (co << 6) | (ld << 8) | (st << 12);
}
NFFT_HD constexpr int qop_gen(int ld, int st) { return QOP_GEN_BASE | (ld << 8) | (st << 12); }
NFFT_HD constexpr int qop_unpack(int st) { return QOP_UNPACK_BASE | st; }

// Size-1 transforms (QOP_SCALAR): tile t covers transforms [t*SCALAR_TILE, ...)
// of the descriptor; a.in_tab / a.out_tab give each one's offsets (elements of
// T), a.conj_in / a.conj_out say whether input / output are complex, a.dst
// that the imaginary part is copied (complex to complex), a.scale the factor.
constexpr int SCALAR_TILE = 2048;

}  // namespace nfft

// nfft_cluster.cuh -- single-pass complex DFT of one transform per thread-block
// cluster, exchanging the intermediate through distributed shared memory.
//
// The length N = R1 * R2 transform is the two-pass Stockham FFT (pass 1:
// radix R1 over the R2 lines j, reading x[j + r R2]; pass 2: radix R2 over
// the R1 lines j', reading A[j' + r' R1] times W_N^{r' j'}), with the C = 2^LOGC
// CTAs of a cluster splitting each pass's lines: CTA c runs pass-1 lines
// [c R2/C, (c+1) R2/C) and keeps their outputs in its own shared memory;
// after a cluster barrier, CTA c runs pass-2 lines [c R1/C, (c+1) R1/C),
// reading each point A[j' + r' R1] (= output j' of pass-1 line r') from the
// shared memory of the CTA that owns line r'.  A second cluster barrier keeps
// every CTA's shared memory alive until all remote reads are done.  The
// intermediate therefore never touches HBM: the transform reads its input and
// writes its output once.
//
// Both passes reuse the specialized pass building blocks (nfft_lean.cuh) in
// column mode; the tile of each CTA is N / C points (16 per thread).
#pragma once

#include <cooperative_groups.h>

#include "nfft_lean.cuh"

namespace nfft {

namespace cg = cooperative_groups;

template <typename T, int LOGR1, int LOGR2, int LOGC, int LOGT>
struct ClusterFFT {
    static constexpr int LOGN = LOGR1 + LOGR2;
    static constexpr int C = 1 << LOGC;
    static constexpr int THREADS = 1 << LOGT;
    static_assert(LOGT + 4 + LOGC == LOGN, "cluster tile must be 16 points per thread");
    static constexpr int LOGJA = LOGR2 - LOGC;   // pass-1 lines per CTA
    static constexpr int LOGJC = LOGR1 - LOGC;   // pass-2 lines per CTA
    using P1 = Lean<T, LOGR1, LOGT, true, true, LD_C, ST_C>;
    using P2 = Lean<T, LOGR2, LOGT, true, true, LD_C, ST_C>;
    static_assert(P1::LOGJ == LOGJA && P2::LOGJ == LOGJC, "tile shapes");
    static constexpr int SMEM_ELEMS = P1::SMEM_ELEMS > P2::SMEM_ELEMS ? P1::SMEM_ELEMS : P2::SMEM_ELEMS;
    static constexpr int MAXJ = (1 << LOGJA) > (1 << LOGJC) ? (1 << LOGJA) : (1 << LOGJC);

    // pass-1 / pass-2 line tables of CTA c of transform b
    static NFFT_HD void lines1(const PassArgs& a, long long b, int c, int l, LeanLine* lines) {
        lines[l] = LeanLine{b * a.istr[0], 0, ((long long)c << LOGJA) + l};
    }
    static NFFT_HD void lines2(const PassArgs& a, long long b, int c, int l, LeanLine* lines) {
        lines[l] = LeanLine{0, b * a.ostr[0], ((long long)c << LOGJC) + l};
    }

    // Pass 2, first sub-stage, gather: thread t's 16 points A[j' + r' R1],
    // r' = i + m R2/16, from the CTA owning pass-1 line r' (shared memories of
    // the cluster in `cta_sm`), then the pass pre-twiddle and the radix 16.
    template <typename SmemOf>
    static NFFT_HD void gather(const PassArgs& a2, const TwTables<T>* tw, int c, int t, SmemOf cta_sm, C2<T>* v, int& l,
                               int& i) {
        lean_map<true, LOGJC>(t, LOGR2 - 4, l, i);
        const int jp = (c << LOGJC) + l;   // pass-2 line = pass-1 output position
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int rp = i + (m << (LOGR2 - 4));          // pass-1 line holding the point
            const C2<T>* sm = cta_sm(rp >> LOGJA);
            v[m] = sm[NFFT_SM((lean_idx<true, LOGR1, LOGJA>(rp & ((1 << LOGJA) - 1), jp)))];
        }
        // W_N^{r' j'} = W_N^{i j'} (W_{16 R1}^{j'})^m, as in the lean first sub-stage
        if (jp) {
            C2<T> w = twiddle<T>(tw, (uint64_t)i * (uint64_t)jp, LOGN);
            const C2<T> s = twiddle<T>(tw, (uint64_t)jp, LOGR1 + 4);
            const C2<T> s4 = cmul(cmul(s, s), cmul(s, s));
            C2<T> c0 = w, c1 = cmul(w, s);
            C2<T> c2 = cmul(c1, s), c3 = cmul(c2, s);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                v[4 * q + 0] = cmul(v[4 * q + 0], c0);
                v[4 * q + 1] = cmul(v[4 * q + 1], c1);
                v[4 * q + 2] = cmul(v[4 * q + 2], c2);
                v[4 * q + 3] = cmul(v[4 * q + 3], c3);
                if (q < 3) { c0 = cmul(c0, s4); c1 = cmul(c1, s4); c2 = cmul(c2, s4); c3 = cmul(c3, s4); }
            }
        }
        dft16<T>(v);
    }
};

template <typename T, int LOGR1, int LOGR2, int LOGC, int LOGT>
constexpr size_t cluster_smem_bytes() {
    using K = ClusterFFT<T, LOGR1, LOGR2, LOGC, LOGT>;
    return sizeof(C2<T>) * (size_t)K::SMEM_ELEMS + sizeof(LeanLine) * (size_t)K::MAXJ;
}

// Middle and last sub-stages of a lean pass whose first sub-stage already
// left its outputs in shared memory (P = the Lean instantiation).  The last
// one writes to global memory (TO_GLOBAL) or back to shared memory.
template <typename P, bool TO_GLOBAL, typename T>
__device__ __forceinline__ void lean_tail(const PassArgs& a, const TwTables<T>* tw, C2<T>* sm, const LeanLine* lines,
                                          int t) {
    using V = C2<T>;
    if constexpr (P::NS >= 3) {
        constexpr int S = 1;
        constexpr int RHO = 1 << LeanSched<P::LOGR_>::lr[S];
        V w[16];
        int ls[16 / RHO], is[16 / RHO];
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) P::template read<S, P::COLL>(sm, t, q, &w[q * RHO], ls[q], is[q]);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) {
            P::template twiddle_dft<S>(tw, is[q], &w[q * RHO]);
            P::template write_smem<S>(sm, ls[q], is[q], &w[q * RHO]);
        }
        __syncthreads();
    }
    if constexpr (P::NS >= 4) {
        constexpr int S = 2;
        constexpr int RHO = 1 << LeanSched<P::LOGR_>::lr[S];
        V w[16];
        int ls[16 / RHO], is[16 / RHO];
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) P::template read<S, P::COLL>(sm, t, q, &w[q * RHO], ls[q], is[q]);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) {
            P::template twiddle_dft<S>(tw, is[q], &w[q * RHO]);
            P::template write_smem<S>(sm, ls[q], is[q], &w[q * RHO]);
        }
        __syncthreads();
    }
    {
        constexpr int S = P::NS - 1;
        constexpr int RHO = 1 << LeanSched<P::LOGR_>::lr[S];
        V w[16];
        int ls[16 / RHO], is[16 / RHO];
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) P::template read<S, true>(sm, t, q, &w[q * RHO], ls[q], is[q]);
        if constexpr (!TO_GLOBAL) __syncthreads();
#pragma unroll
        for (int q = 0; q < 16 / RHO; ++q) {
            P::template twiddle_dft<S>(tw, is[q], &w[q * RHO]);
            if constexpr (TO_GLOBAL) P::template write_global<S>(a, tw, lines, ls[q], is[q], &w[q * RHO]);
            else P::template write_smem<S>(sm, ls[q], is[q], &w[q * RHO]);
        }
    }
}

// One transform per cluster of C CTAs; a1 / a2 describe pass 1 / pass 2
// (radix, strides, batch distance in istr[0] / ostr[0], conjugation).
template <typename T, int LOGR1, int LOGR2, int LOGC, int LOGT>
__global__ void __launch_bounds__(1 << LOGT, (LOGT <= 7 ? 4 : (LOGT == 8 ? 2 : 1)))
cluster_fft_kernel(const PassArgs a1, const PassArgs a2, long long ntransforms) {
    using K = ClusterFFT<T, LOGR1, LOGR2, LOGC, LOGT>;
    using V = C2<T>;
    extern __shared__ __align__(16) unsigned char smraw[];
    V* sm = (V*)smraw;
    LeanLine* lines = (LeanLine*)(sm + K::SMEM_ELEMS);
    const TwTables<T>* tw = (const TwTables<T>*)a1.tw;
    cg::cluster_group cluster = cg::this_cluster();
    const int c = (int)cluster.block_rank();
    const long long b = (long long)blockIdx.x >> LOGC;
    const bool live = b < ntransforms;   // uniform over the cluster
    const int t = threadIdx.x;

    // ---- pass 1 into this CTA's shared memory ----
    if (live) {
        if (t < (1 << K::LOGJA)) K::lines1(a1, b, c, t, lines);
        __syncthreads();
        V v[16];
        int l, i;
        K::P1::first(a1, tw, lines, t, v, l, i);
        K::P1::template write_smem<0>(sm, l, i, v);
        __syncthreads();
        lean_tail<typename K::P1, false, T>(a1, tw, sm, lines, t);
    }
    cluster.sync();
    // ---- pass 2: gather from the cluster, then finish and store ----
    V v[16];
    int l = 0, i = 0;
    if (live) {
        K::gather(a2, tw, c, t, [&](int rank) { return (const V*)cluster.map_shared_rank(sm, rank); }, v, l, i);
    }
    cluster.sync();   // every remote read of this CTA's shared memory is done
    if (live) {
        if (t < (1 << K::LOGJC)) K::lines2(a2, b, c, t, lines);
        K::P2::template write_smem<0>(sm, l, i, v);
        __syncthreads();
        lean_tail<typename K::P2, true, T>(a2, tw, sm, lines, t);
    }
}

}  // namespace nfft

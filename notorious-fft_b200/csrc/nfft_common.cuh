// nfft_common.cuh -- device-side building blocks of the B200 FFT engine:
// complex arithmetic, the three-level twiddle table, and the radix-2/4/8/16
// in-register DFT butterflies (forward sign; inverse transforms run through
// conjugation at the load/store boundaries).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Host+device helpers.  The library is built for the GPU only; the host
// side of these helpers is compiled solely by the test-only emulator build
// (tests/emu), which defines NFFT_EMULATE to bounds-check every global access.
#define NFFT_HD __host__ __device__ __forceinline__
#ifdef NFFT_EMULATE
__host__ __device__ void nfft_emu_check(const void* p, size_t bytes, int write);
#define NFFT_GLD(ptr) (nfft_emu_check((ptr), sizeof(*(ptr)), 0), *(ptr))
#define NFFT_GST(ptr, val) (nfft_emu_check((ptr), sizeof(*(ptr)), 1), *(ptr) = (val))
#else
#define NFFT_GLD(ptr) (*(ptr))
#define NFFT_GST(ptr, val) (*(ptr) = (val))
#endif

namespace nfft {

template <typename T> struct cvec;
template <> struct cvec<double> { using type = double2; };
template <> struct cvec<float> { using type = float2; };
template <typename T> using C2 = typename cvec<T>::type;

NFFT_HD double2 mkc(double a, double b) { return make_double2(a, b); }
NFFT_HD float2 mkc(float a, float b) { return make_float2(a, b); }

template <typename V> NFFT_HD V cadd(V a, V b) { return mkc(a.x + b.x, a.y + b.y); }
template <typename V> NFFT_HD V csub(V a, V b) { return mkc(a.x - b.x, a.y - b.y); }
// a * b
template <typename V> NFFT_HD V cmul(V a, V b) {
    return mkc(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * conj(b)
template <typename V> NFFT_HD V cmulc(V a, V b) {
    return mkc(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
template <typename V> NFFT_HD V cconj(V a) { return mkc(a.x, -a.y); }
// a * (-i)
template <typename V> NFFT_HD V mul_mi(V a) { return mkc(a.y, -a.x); }
template <typename V, typename S> NFFT_HD V cscale(V a, S s) { return mkc(a.x * s, a.y * s); }

// ---------------------------------------------------------------------------
// Global accesses with L2 policy.  hint 0: default; 1: streaming (user data
// read or written once: evict first); 2: inter-pass scratch (stores kept in L2
// with evict_last priority; the last read is followed by discard_l2); 3: data
// written earlier in the same launch by other CTAs (loaded at L2, the point of
// coherence, never from a possibly stale L1 line; stores as hint 2).
// ---------------------------------------------------------------------------
template <typename V>
NFFT_HD V gload(const V* p, int hint) {
#if defined(__CUDA_ARCH__)
    if (hint == 1 || hint == 2) return __ldcs(p);
    if (hint == 3) return __ldcg(p);
    return *p;
#else
    (void)hint;
    return NFFT_GLD(p);
#endif
}

NFFT_HD void gstore(double2* p, double2 v, int hint) {
#if defined(__CUDA_ARCH__)
    if (hint == 1) { __stcs(p, v); return; }
    if (hint >= 2) {
        uint64_t pol;
        asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
        asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(v.x), "d"(v.y), "l"(pol)
                     : "memory");
        return;
    }
    *p = v;
#else
    (void)hint;
    NFFT_GST(p, v);
#endif
}

NFFT_HD void gstore(float2* p, float2 v, int hint) {
#if defined(__CUDA_ARCH__)
    if (hint == 1) { __stcs(p, v); return; }
    if (hint >= 2) {
        uint64_t pol;
        asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
        asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x), "f"(v.y), "l"(pol)
                     : "memory");
        return;
    }
    *p = v;
#else
    (void)hint;
    NFFT_GST(p, v);
#endif
}

// Load of a table every transform of a batch reads again (Bluestein chirp and
// filter spectrum): kept in L2 with evict_last priority.
NFFT_HD double2 gload_keep(const double2* p) {
#if defined(__CUDA_ARCH__)
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    double2 v;
    asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
    return v;
#else
    return NFFT_GLD(p);
#endif
}
NFFT_HD float2 gload_keep(const float2* p) {
#if defined(__CUDA_ARCH__)
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    float2 v;
    asm volatile("ld.global.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(pol));
    return v;
#else
    return NFFT_GLD(p);
#endif
}

// Drop a 128-byte line from L2 without writing it back (dead scratch data).
NFFT_HD void discard_l2(const void* p) {
#if defined(__CUDA_ARCH__)
    asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
#else
    (void)p;
#endif
}

// ---------------------------------------------------------------------------
// Twiddle tables.  W_P^q = exp(-2 pi i q / P) for any power of two P <= 2^36
// is assembled from three 4096-entry tables that split a 36-bit fraction of a
// turn into 12-bit digits:  u = q * 2^(36 - log2 P),
//   W = T0[u >> 24] * T1[(u >> 12) & 4095] * T2[u & 4095],
//   Tk[m] = exp(-2 pi i m / 2^(12 (k+1))).
// Roots of order <= 4096 are a single exact table entry; larger orders cost one
// or two extra complex products (each ~1 ulp).  The tables are filled once per
// device from FP64 sincospi (rounded to float for the float library).
// ---------------------------------------------------------------------------
constexpr int TW_BITS = 12;
constexpr int TW_SIZE = 1 << TW_BITS;

template <typename T> struct TwTables { C2<T> t[3][TW_SIZE]; };

template <typename T>
NFFT_HD C2<T> tw_load(const TwTables<T>* tw, int level, uint32_t idx) {
#if defined(__CUDA_ARCH__)
    return __ldg(&tw->t[level][idx]);
#else
    return NFFT_GLD(&tw->t[level][idx]);
#endif
}

// W_{2^logP}^q, q < 2^logP, logP <= 12: one table entry.
template <typename T>
NFFT_HD C2<T> twiddle_small(const TwTables<T>* tw, uint32_t q, int logP) {
    return tw_load<T>(tw, 0, (q << (TW_BITS - logP)) & (TW_SIZE - 1));
}

// W_{2^logP}^q for any logP <= 36.
template <typename T>
NFFT_HD C2<T> twiddle(const TwTables<T>* tw, uint64_t q, int logP) {
    uint64_t u = (q << (36 - logP)) & ((1ull << 36) - 1);
    C2<T> w = tw_load<T>(tw, 0, (uint32_t)(u >> 24));
    uint32_t i1 = (uint32_t)(u >> 12) & (TW_SIZE - 1);
    uint32_t i2 = (uint32_t)u & (TW_SIZE - 1);
    if (i1) w = cmul(w, tw_load<T>(tw, 1, i1));
    if (i2) w = cmul(w, tw_load<T>(tw, 2, i2));
    return w;
}

// ---------------------------------------------------------------------------
// In-register DFTs, natural order in and out, forward sign.
// ---------------------------------------------------------------------------
template <typename V> NFFT_HD void dft2(V& a0, V& a1) {
    V t = a0;
    a0 = cadd(t, a1);
    a1 = csub(t, a1);
}

template <typename V> NFFT_HD void dft4(V& a0, V& a1, V& a2, V& a3) {
    V b0 = cadd(a0, a2), b1 = csub(a0, a2);
    V b2 = cadd(a1, a3), b3 = mul_mi(csub(a1, a3));
    a0 = cadd(b0, b2);
    a2 = csub(b0, b2);
    a1 = cadd(b1, b3);
    a3 = csub(b1, b3);
}

template <typename T> struct K {
    // cos(pi/8), sin(pi/8), sqrt(1/2)
    static constexpr T c8 = (T)0.92387953251128675612818318939678828682L;
    static constexpr T s8 = (T)0.38268343236508977172845998403039886676L;
    static constexpr T r2 = (T)0.70710678118654752440084436210484903928L;
};

// x * W8^1 = x * (1 - i)/sqrt2
template <typename T> NFFT_HD C2<T> mul_w8_1(C2<T> x) {
    return mkc((x.x + x.y) * K<T>::r2, (x.y - x.x) * K<T>::r2);
}
// x * W8^3 = x * (-1 - i)/sqrt2
template <typename T> NFFT_HD C2<T> mul_w8_3(C2<T> x) {
    return mkc((x.y - x.x) * K<T>::r2, -(x.x + x.y) * K<T>::r2);
}

template <typename T> NFFT_HD void dft8(C2<T>* a) {
    C2<T> e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6];
    C2<T> o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
    dft4(e0, e1, e2, e3);
    dft4(o0, o1, o2, o3);
    o1 = mul_w8_1<T>(o1);
    o2 = mul_mi(o2);
    o3 = mul_w8_3<T>(o3);
    a[0] = cadd(e0, o0); a[4] = csub(e0, o0);
    a[1] = cadd(e1, o1); a[5] = csub(e1, o1);
    a[2] = cadd(e2, o2); a[6] = csub(e2, o2);
    a[3] = cadd(e3, o3); a[7] = csub(e3, o3);
}

// 16 = 4 x 4: n = 4 n1 + n2, k = k1 + 4 k2.
template <typename T> NFFT_HD void dft16(C2<T>* a) {
    using V = C2<T>;
    V b[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        V x0 = a[n2], x1 = a[4 + n2], x2 = a[8 + n2], x3 = a[12 + n2];
        dft4(x0, x1, x2, x3);
        b[n2][0] = x0; b[n2][1] = x1; b[n2][2] = x2; b[n2][3] = x3;
    }
    const T c = K<T>::c8, s = K<T>::s8;
    // W16^{n2 k1}
    b[1][1] = cmul(b[1][1], mkc(c, -s));
    b[1][2] = mul_w8_1<T>(b[1][2]);
    b[1][3] = cmul(b[1][3], mkc(s, -c));
    b[2][1] = mul_w8_1<T>(b[2][1]);
    b[2][2] = mul_mi(b[2][2]);
    b[2][3] = mul_w8_3<T>(b[2][3]);
    b[3][1] = cmul(b[3][1], mkc(s, -c));
    b[3][2] = mul_w8_3<T>(b[3][2]);
    b[3][3] = cmul(b[3][3], mkc(-c, s));
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        V x0 = b[0][k1], x1 = b[1][k1], x2 = b[2][k1], x3 = b[3][k1];
        dft4(x0, x1, x2, x3);
        a[k1] = x0; a[k1 + 4] = x1; a[k1 + 8] = x2; a[k1 + 12] = x3;
    }
}

template <typename T, int RHO> NFFT_HD void dft_radix(C2<T>* a) {
    if constexpr (RHO == 2) dft2(a[0], a[1]);
    else if constexpr (RHO == 4) dft4(a[0], a[1], a[2], a[3]);
    else if constexpr (RHO == 8) dft8<T>(a);
    else if constexpr (RHO == 16) dft16<T>(a);
}

}  // namespace nfft

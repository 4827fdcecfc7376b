// hop.cuh — the hopping-term arithmetic shared by the solver kernels and the
// standalone Dslash: complex 3x3 matrix-vector products as FMA chains, with
// the hop's scalar factor (eta_mu / 2, the anti-periodic time sign, the
// per-site scale of the 16-bit storages) applied to the input vector; and
// for FP16 links and vectors the products in packed half2.
#pragma once

#include <cuda_fp16.h>

#include "sfh_core.cuh"

namespace sfh {
namespace {

template <typename To, typename From>
__device__ __forceinline__ Vec3<To> vcvt(const Vec3<From>& v)
{
    Vec3<To> o;
#pragma unroll
    for (int k = 0; k < 3; ++k) o.c[k] = {(To)v.c[k].re, (To)v.c[k].im};
    return o;
}

// w = U v (FIRST) or w += U v, as FMA chains
template <bool FIRST, typename R>
__device__ __forceinline__ void mv_add(Vec3<R>& w, const Mat3<R>& U, const Vec3<R>& v)
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const Cx<R>* u = &U.e[3 * i];
        R re = FIRST ? u[0].re * v.c[0].re : fma(u[0].re, v.c[0].re, w.c[i].re);
        R im = FIRST ? u[0].re * v.c[0].im : fma(u[0].re, v.c[0].im, w.c[i].im);
        re = fma(-u[0].im, v.c[0].im, re);
        im = fma(u[0].im, v.c[0].re, im);
#pragma unroll
        for (int k = 1; k < 3; ++k) {
            re = fma(u[k].re, v.c[k].re, re);
            re = fma(-u[k].im, v.c[k].im, re);
            im = fma(u[k].re, v.c[k].im, im);
            im = fma(u[k].im, v.c[k].re, im);
        }
        w.c[i] = {re, im};
    }
}

// w -= U^dag v, as FMA chains: (U^dag v)_i = sum_k conj(U_ki) v_k
template <typename R>
__device__ __forceinline__ void mdv_sub(Vec3<R>& w, const Mat3<R>& U, const Vec3<R>& v)
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R re = w.c[i].re, im = w.c[i].im;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const Cx<R> u = U.e[3 * k + i];
            re = fma(-u.re, v.c[k].re, re);
            re = fma(-u.im, v.c[k].im, re);
            im = fma(-u.re, v.c[k].im, im);
            im = fma(u.im, v.c[k].re, im);
        }
        w.c[i] = {re, im};
    }
}

// acc += s w
template <typename R>
__device__ __forceinline__ void vfma(Vec3<R>& acc, R s, const Vec3<R>& w)
{
#pragma unroll
    for (int k = 0; k < 3; ++k) acc.c[k] = {fma(s, w.c[k].re, acc.c[k].re), fma(s, w.c[k].im, acc.c[k].im)};
}

template <typename R>
__device__ __forceinline__ Vec3<R> vneg_if(const Vec3<R>& v, bool neg, R scale = R(1))
{
    const R s = neg ? -scale : scale;
    Vec3<R> o;
#pragma unroll
    for (int k = 0; k < 3; ++k) o.c[k] = {s * v.c[k].re, s * v.c[k].im};
    return o;
}

// a neighbour spinor with the hop's scalar factor applied: the eta / 2 and
// time-wrap sign, and for the 16-bit storages the per-site scale (one multiply)
template <int SP, typename R, bool COH = false>
__device__ __forceinline__ Vec3<R> hop_input(const void* in, int nq, int j, int Vh, bool neg, R s)
{
    if constexpr (SpinorFmt<SP>::scaled) {
        float sc;
        Vec3<R> v = SpinorFmt<SP>::template load_unscaled<COH>(in, nq, j, Vh, &sc);
        return vneg_if(v, neg, s * sc);
    } else {
        return vneg_if(vcvt<R>(SpinorFmt<SP>::template load<COH>(in, nq, j, Vh)), neg, s);
    }
}

// hop_input for a stored word of a scaled 16-bit vector format
template <int SP, typename R>
__device__ __forceinline__ Vec3<R> hop_input_word(const uint4 w, bool neg, R s)
{
    float sc;
    const Vec3<R> v = SpinorFmt<SP>::unscaled(w, &sc);
    return vneg_if(v, neg, s * sc);
}

// ---------------------------------------------------------------------------
// FP16 links and vectors: the products in packed half2 arithmetic
// ---------------------------------------------------------------------------
// Complex numbers are half2 pairs (re, im).  With b_perp = (-b.im, b.re),
// a b = a.re (b.re, b.im) + a.im b_perp: two packed FMAs whose first
// operand is one half of a broadcast to both (free in the instruction), so
// a 3x3 complex matrix-vector product is 18 packed FMAs and the links and
// vectors are used as stored.  Each neighbour's product (|entries| <= 3:
// link entries and the site-normalised vector entries are at most 1) is
// converted to FP32 and accumulated there with its scalar factor (eta / 2,
// the time-wrap sign, the neighbour's site scale).

__device__ __forceinline__ __half2 h2_bits(uint32_t w) { return *reinterpret_cast<__half2*>(&w); }

__device__ __forceinline__ __half2 h2_perp(__half2 b)  // (-b.im, b.re)
{
    return __hmul2(__lowhigh2highlow(b), __halves2half2(__ushort_as_half(0xBC00u), __ushort_as_half(0x3C00u)));
}

// 12-real FP16 link -> nine half2, row 2 = conj(row0 x row1)
__device__ __forceinline__ void hlink_unpack(const uint2 (&w)[3], __half2 (&e)[9])
{
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        e[2 * k] = h2_bits(w[k].x);
        e[2 * k + 1] = h2_bits(w[k].y);
    }
    const __half2* a = &e[0];
    const __half2* b = &e[3];
    __half2 bp[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) bp[k] = h2_perp(b[k]);
    const __half2 conj = __halves2half2(__ushort_as_half(0x3C00u), __ushort_as_half(0xBC00u));  // (1, -1)
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const int j = (m + 1) % 3, k = (m + 2) % 3;
        // a_j b_k - a_k b_j
        __half2 d = __hmul2(__low2half2(a[j]), b[k]);
        d = __hfma2(__high2half2(a[j]), bp[k], d);
        d = __hfma2(__hneg2(__low2half2(a[k])), b[j], d);
        d = __hfma2(__hneg2(__high2half2(a[k])), bp[j], d);
        e[6 + m] = __hmul2(d, conj);
    }
}

// the link of direction slot d staged in shared memory ([d][k][thread],
// `tile` threads; STG) or of (p, mu, i) in global memory
template <bool STG>
__device__ __forceinline__ void hlink_load(const uint2* s, int tile, const void* Ulo, int d, int p, int mu, int i,
                                           int Vh, __half2 (&e)[9])
{
    uint2 w[3];
    if constexpr (STG) {
#pragma unroll
        for (int k = 0; k < 3; ++k) w[k] = s[(d * 3 + k) * tile + threadIdx.x];
    } else {
        const uint2* b = (const uint2*)Ulo + ((size_t)(p * 4 + mu) * 3) * Vh + i;
#pragma unroll
        for (int k = 0; k < 3; ++k) w[k] = __ldg(b + (size_t)k * Vh);
    }
    hlink_unpack(w, e);
}

// f broadcast to both halves of a packed FP32 pair
__device__ __forceinline__ unsigned long long f32x2_bcast(float f)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(f));
    return r;
}

// (acc.re, acc.im) += f2 * (y.x, y.y) as one packed FP32 FMA (fma.rn.f32x2,
// sm_100 and later): each half rounds as fmaf does
__device__ __forceinline__ void acc_f32x2(Cx<float>& acc, unsigned long long f2, float2 y)
{
    unsigned long long b, c, d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(b) : "f"(y.x), "f"(y.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(c) : "f"(acc.re), "f"(acc.im));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2), "l"(b), "l"(c));
    asm("mov.b64 {%0, %1}, %2;" : "=f"(acc.re), "=f"(acc.im) : "l"(d));
}

// acc += f (U v) (ADJ false) or acc += f (U^dag v) (ADJ true) for the
// stored FP16 vector word w (three half2 pairs and the site scale sc):
// f = s sc, products in half2
template <bool ADJ>
__device__ __forceinline__ void hop_half_word(Vec3<float>& acc, const __half2 (&U)[9], const uint4 w, float f)
{
    const __half2 v[3] = {h2_bits(w.x), h2_bits(w.y), h2_bits(w.z)};
    const unsigned long long f2 = f32x2_bcast(f * __uint_as_float(w.w));
    __half2 vp[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) vp[k] = ADJ ? __hneg2(h2_perp(v[k])) : h2_perp(v[k]);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        // row r of U (U_rk) or column r (conj(U_kr)); conj(u) v = u.re v - u.im v_perp
        __half2 y = __hmul2(__low2half2(U[ADJ ? r : 3 * r]), v[0]);
        y = __hfma2(__high2half2(U[ADJ ? r : 3 * r]), vp[0], y);
#pragma unroll
        for (int k = 1; k < 3; ++k) {
            const __half2 u = U[ADJ ? 3 * k + r : 3 * r + k];
            y = __hfma2(__low2half2(u), v[k], y);
            y = __hfma2(__high2half2(u), vp[k], y);
        }
        acc_f32x2(acc.c[r], f2, __half22float2(y));
    }
}

// hop_half_word for the vector of site j of parity nq in global memory
template <bool ADJ, bool COH = false>
__device__ __forceinline__ void hop_half(Vec3<float>& acc, const __half2 (&U)[9], const void* in, int nq, int j,
                                         int Vh, float f)
{
    hop_half_word<ADJ>(acc, U, ld_vec<COH>((const uint4*)in + (size_t)nq * Vh + j), f);
}

}  // namespace
}  // namespace sfh

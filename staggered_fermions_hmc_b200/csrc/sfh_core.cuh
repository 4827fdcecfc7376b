// sfh_core.cuh — device-side geometry, even-odd indexing, storage formats and
// SU(3) algebra shared by every kernel of the library.
//
// Site ordering follows the reference: lexicographic s = ((x*Ly+y)*Lz+z)*Lt+t
// with t fastest (Fermions.cpp:42, Lattice.cpp:20).  The device keeps fields
// split by parity p = (x+y+z+t) & 1 and indexed inside a parity by the
// checkerboard index i = s >> 1 (a bijection per parity because Lt is even).
//
// HBM layouts (structure of arrays, one thread per site reads consecutive
// words across a warp):
//   spinor, FP64     : double2 [p][color 3][i]
//   spinor, FP32     : float2  [p][color 3][i]
//   spinor, FP16+scale: uint4  [p][i] = {3 x half2 (colors), float scale}
//   gauge,  FP64 18  : double2 [p][mu][entry 9][i]        (entry = row*3+col)
//   gauge,  FP32 12  : float4  [p][mu][k 3][i]            (rows 0,1; row 2 rebuilt)
//   gauge,  FP16 12  : uint2   [p][mu][k 3][i]            (rows 0,1 as 12 halves)
//   momentum / force : double2 [p][mu][entry 9][i]        (FP64, 18-real)
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sfh {

// ---------------------------------------------------------------------------
// fast integer division by a runtime constant (round-up multiply method,
// Granlund & Montgomery 1994), valid for all 32-bit unsigned numerators.
// ---------------------------------------------------------------------------
struct FastDiv {
    uint32_t d, m, l;
    FastDiv() = default;  // trivial, so that structs holding one can live in __shared__
    explicit FastDiv(uint32_t div) : d(div)
    {
        l = 0;
        while ((1ull << l) < d) ++l;
        if (l == 0) { m = 0; return; }
        uint64_t num = ((1ull << l) - d) << 32;
        m = (uint32_t)(num / d + 1);
    }
    __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const
    {
        if (l == 0) return n;
#ifdef __CUDA_ARCH__
        uint32_t t = __umulhi(m, n);
#else
        uint32_t t = (uint32_t)(((uint64_t)m * n) >> 32);
#endif
        return (t + ((n - t) >> 1)) >> (l - 1);
    }
};

struct Geom {
    int L[4];        // Lx, Ly, Lz, Lt
    int V, Vh;
    FastDiv dLt, dLz, dLy;
};

struct Coord {
    int x[4];
    int lex;
};

// coordinates of checkerboard site i of parity p
__device__ __forceinline__ Coord eo_coords(const Geom& g, int p, int i)
{
    Coord c;
    uint32_t s0 = 2u * (uint32_t)i;
    uint32_t r = g.dLt.div(s0);
    int t0 = (int)(s0 - r * (uint32_t)g.L[3]);
    uint32_t r2 = g.dLz.div(r);
    c.x[2] = (int)(r - r2 * (uint32_t)g.L[2]);
    uint32_t r3 = g.dLy.div(r2);
    c.x[1] = (int)(r2 - r3 * (uint32_t)g.L[1]);
    c.x[0] = (int)r3;
    int flip = (c.x[0] + c.x[1] + c.x[2] + p) & 1;
    c.x[3] = t0 + flip;
    c.lex = (int)s0 + flip;
    return c;
}

// lexicographic strides
__device__ __forceinline__ int lex_stride(const Geom& g, int mu)
{
    return mu == 3 ? 1 : (mu == 2 ? g.L[3] : (mu == 1 ? g.L[2] * g.L[3] : g.L[1] * g.L[2] * g.L[3]));
}

// lexicographic index of x + mu (periodic)
__device__ __forceinline__ int lex_up(const Geom& g, const Coord& c, int mu)
{
    int st = lex_stride(g, mu);
    return c.x[mu] + 1 < g.L[mu] ? c.lex + st : c.lex - (g.L[mu] - 1) * st;
}

__device__ __forceinline__ int lex_dn(const Geom& g, const Coord& c, int mu)
{
    int st = lex_stride(g, mu);
    return c.x[mu] > 0 ? c.lex - st : c.lex + (g.L[mu] - 1) * st;
}

// staggered phase eta_mu(x) = (-1)^{sum_{nu<mu} x_nu} (Fermions.cpp:46-52)
__device__ __forceinline__ int eta_sign(const Coord& c, int mu)
{
    int s = 0;
    if (mu > 0) s += c.x[0];
    if (mu > 1) s += c.x[1];
    if (mu > 2) s += c.x[2];
    return (s & 1) ? -1 : 1;
}

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
template <typename R> struct C2;
template <> struct C2<double> { typedef double2 T; };
template <> struct C2<float> { typedef float2 T; };

template <typename R>
struct Cx {
    R re, im;
};

template <typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b)
{
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R>  // conj(a) * b
__device__ __forceinline__ Cx<R> cmulc(Cx<R> a, Cx<R> b)
{
    return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}

template <typename R>
struct Mat3 {
    Cx<R> e[9];  // row-major
};

template <typename R>
struct Vec3 {
    Cx<R> c[3];
};

// out = U v
template <typename R>
__device__ __forceinline__ Vec3<R> mul_mv(const Mat3<R>& U, const Vec3<R>& v)
{
    Vec3<R> o;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R re = U.e[i * 3].re * v.c[0].re - U.e[i * 3].im * v.c[0].im;
        R im = U.e[i * 3].re * v.c[0].im + U.e[i * 3].im * v.c[0].re;
#pragma unroll
        for (int k = 1; k < 3; ++k) {
            re += U.e[i * 3 + k].re * v.c[k].re - U.e[i * 3 + k].im * v.c[k].im;
            im += U.e[i * 3 + k].re * v.c[k].im + U.e[i * 3 + k].im * v.c[k].re;
        }
        o.c[i] = {re, im};
    }
    return o;
}

// out = U^dag v
template <typename R>
__device__ __forceinline__ Vec3<R> mul_adj_mv(const Mat3<R>& U, const Vec3<R>& v)
{
    Vec3<R> o;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R re = U.e[i].re * v.c[0].re + U.e[i].im * v.c[0].im;
        R im = U.e[i].re * v.c[0].im - U.e[i].im * v.c[0].re;
#pragma unroll
        for (int k = 1; k < 3; ++k) {
            re += U.e[k * 3 + i].re * v.c[k].re + U.e[k * 3 + i].im * v.c[k].im;
            im += U.e[k * 3 + i].re * v.c[k].im - U.e[k * 3 + i].im * v.c[k].re;
        }
        o.c[i] = {re, im};
    }
    return o;
}

template <typename R>
__device__ __forceinline__ void reconstruct_row2(Mat3<R>& U)
{
    // row2 = conj(row0 x row1) for a special-unitary matrix, as FMA chains:
    // e[6+m] = conj(a_j b_k - a_k b_j) with (j, k) = (1, 2), (2, 0), (0, 1)
    const Cx<R>* a = &U.e[0];
    const Cx<R>* b = &U.e[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const int j = (m + 1) % 3, k = (m + 2) % 3;
        R re = a[j].re * b[k].re;
        re = fma(-a[j].im, b[k].im, re);
        re = fma(-a[k].re, b[j].re, re);
        re = fma(a[k].im, b[j].im, re);
        R im = -a[j].re * b[k].im;
        im = fma(-a[j].im, b[k].re, im);
        im = fma(a[k].re, b[j].im, im);
        im = fma(a[k].im, b[j].re, im);
        U.e[6 + m] = {re, im};
    }
}

// ---------------------------------------------------------------------------
// storage formats
// ---------------------------------------------------------------------------
enum SpinorPrec { SP_F64 = 0, SP_F32 = 1, SP_F16 = 2, SP_BF16 = 3 };
enum GaugePrec { GP_F64_18 = 0, GP_F32_12 = 1, GP_F16_12 = 2, GP_F32_18 = 3, GP_BF16_12 = 4, GP_F64_12 = 5 };

template <int SP> struct SpinorFmt;

// load of a vector word: through the read-only data cache (COH false; data
// not written while the kernel runs) or through L2 only (COH true: data other
// blocks of the same persistent kernel write between its phases)
template <bool COH, typename T>
__device__ __forceinline__ T ld_vec(const T* p)
{
    if constexpr (COH) return __ldcg(p);
    else return __ldg(p);
}

template <> struct SpinorFmt<SP_F64> {
    typedef double R;
    static constexpr size_t site_bytes = 48;
    static constexpr bool scaled = false;
    template <bool COH = false>
    __device__ static __forceinline__ Vec3<R> load(const void* base, int p, int i, int Vh)
    {
        const double2* b = (const double2*)base + (size_t)p * 3 * Vh;
        Vec3<R> v;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double2 w = ld_vec<COH>(b + (size_t)c * Vh + i);
            v.c[c] = {w.x, w.y};
        }
        return v;
    }
    __device__ static __forceinline__ Vec3<R> load_cg(const void* base, int p, int i, int Vh)
    {
        const double2* b = (const double2*)base + (size_t)p * 3 * Vh;
        Vec3<R> v;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double2 w = __ldcg(b + (size_t)c * Vh + i);
            v.c[c] = {w.x, w.y};
        }
        return v;
    }
    __device__ static __forceinline__ Vec3<R> quantize(const Vec3<R>& v) { return v; }
    __device__ static __forceinline__ void store(void* base, int p, int i, int Vh, const Vec3<R>& v)
    {
        double2* b = (double2*)base + (size_t)p * 3 * Vh;
#pragma unroll
        for (int c = 0; c < 3; ++c) b[(size_t)c * Vh + i] = make_double2(v.c[c].re, v.c[c].im);
    }
    // store v and return what was stored (v itself: no rounding)
    __device__ static __forceinline__ Vec3<R> store_q(void* base, int p, int i, int Vh, const Vec3<R>& v)
    {
        store(base, p, i, Vh, v);
        return v;
    }
};

template <> struct SpinorFmt<SP_F32> {
    typedef float R;
    static constexpr size_t site_bytes = 24;
    static constexpr bool scaled = false;
    template <bool COH = false>
    __device__ static __forceinline__ Vec3<R> load(const void* base, int p, int i, int Vh)
    {
        const float2* b = (const float2*)base + (size_t)p * 3 * Vh;
        Vec3<R> v;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float2 w = ld_vec<COH>(b + (size_t)c * Vh + i);
            v.c[c] = {w.x, w.y};
        }
        return v;
    }
    __device__ static __forceinline__ Vec3<R> load_cg(const void* base, int p, int i, int Vh)
    {
        const float2* b = (const float2*)base + (size_t)p * 3 * Vh;
        Vec3<R> v;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float2 w = __ldcg(b + (size_t)c * Vh + i);
            v.c[c] = {w.x, w.y};
        }
        return v;
    }
    __device__ static __forceinline__ Vec3<R> quantize(const Vec3<R>& v) { return v; }
    __device__ static __forceinline__ void store(void* base, int p, int i, int Vh, const Vec3<R>& v)
    {
        float2* b = (float2*)base + (size_t)p * 3 * Vh;
#pragma unroll
        for (int c = 0; c < 3; ++c) b[(size_t)c * Vh + i] = make_float2(v.c[c].re, v.c[c].im);
    }
    __device__ static __forceinline__ Vec3<R> store_q(void* base, int p, int i, int Vh, const Vec3<R>& v)
    {
        store(base, p, i, Vh, v);
        return v;
    }
};

// 16-bit complex pairs (re, im) in one 32-bit word: FP16 or BF16
template <int SP> struct Pair16;
template <> struct Pair16<SP_F16> {
    __device__ static __forceinline__ float2 to_float2(uint32_t w)
    {
        return __half22float2(*reinterpret_cast<__half2*>(&w));
    }
    __device__ static __forceinline__ uint32_t from_floats(float a, float b)
    {
        __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<uint32_t*>(&h);
    }
};
template <> struct Pair16<SP_BF16> {
    __device__ static __forceinline__ float2 to_float2(uint32_t w)
    {
        return __bfloat1622float2(*reinterpret_cast<__nv_bfloat162*>(&w));
    }
    __device__ static __forceinline__ uint32_t from_floats(float a, float b)
    {
        __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<uint32_t*>(&h);
    }
};

// 16-bit vectors with a per-site scale: one uint4 per site, three (re, im)
// pairs of the colour components divided by their largest magnitude, and
// that magnitude as an FP32 in the last word
template <int SP> struct ScaledSpinorFmt {
    typedef float R;
    typedef Pair16<SP> P;
    static constexpr size_t site_bytes = 16;
    static constexpr bool scaled = true;
    __device__ static __forceinline__ Vec3<R> unpack(uint4 w)
    {
        float s = __uint_as_float(w.w);
        Vec3<R> v;
        uint32_t words[3] = {w.x, w.y, w.z};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float2 f = P::to_float2(words[c]);
            v.c[c] = {f.x * s, f.y * s};
        }
        return v;
    }
    __device__ static __forceinline__ uint4 pack(const Vec3<R>& v)
    {
        float m = 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) m = fmaxf(m, fmaxf(fabsf(v.c[c].re), fabsf(v.c[c].im)));
        float inv = m > 0.f ? 1.0f / m : 0.f;
        uint32_t words[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) words[c] = P::from_floats(v.c[c].re * inv, v.c[c].im * inv);
        uint4 w;
        w.x = words[0]; w.y = words[1]; w.z = words[2]; w.w = __float_as_uint(m);
        return w;
    }
    __device__ static __forceinline__ Vec3<R> load_cg(const void* base, int p, int i, int Vh)
    {
        return unpack(__ldcg((const uint4*)base + (size_t)p * Vh + i));
    }
    __device__ static __forceinline__ Vec3<R> quantize(const Vec3<R>& v) { return unpack(pack(v)); }
    // the pairs converted, without the scale (returned in *scale)
    template <bool COH = false>
    __device__ static __forceinline__ Vec3<R> load_unscaled(const void* base, int p, int i, int Vh, float* scale)
    {
        const uint4* b = (const uint4*)base + (size_t)p * Vh;
        return unscaled(ld_vec<COH>(b + i), scale);
    }
    // the pairs of a stored word converted, without the scale (in *scale)
    __device__ static __forceinline__ Vec3<R> unscaled(uint4 w, float* scale)
    {
        *scale = __uint_as_float(w.w);
        Vec3<R> v;
        uint32_t words[3] = {w.x, w.y, w.z};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float2 f = P::to_float2(words[c]);
            v.c[c] = {f.x, f.y};
        }
        return v;
    }
    template <bool COH = false>
    __device__ static __forceinline__ Vec3<R> load(const void* base, int p, int i, int Vh)
    {
        const uint4* b = (const uint4*)base + (size_t)p * Vh;
        return unpack(ld_vec<COH>(b + i));
    }
    __device__ static __forceinline__ void store(void* base, int p, int i, int Vh, const Vec3<R>& v)
    {
        uint4* b = (uint4*)base + (size_t)p * Vh;
        b[i] = pack(v);
    }
    // store v and return the stored (rounded) value, packing once: equal to
    // quantize(v), whose packing a later store would repeat bit for bit
    __device__ static __forceinline__ Vec3<R> store_q(void* base, int p, int i, int Vh, const Vec3<R>& v)
    {
        const uint4 w = pack(v);
        ((uint4*)base + (size_t)p * Vh)[i] = w;
        return unpack(w);
    }
};

template <> struct SpinorFmt<SP_F16> : ScaledSpinorFmt<SP_F16> {};
template <> struct SpinorFmt<SP_BF16> : ScaledSpinorFmt<SP_BF16> {};

template <int GP> struct GaugeFmt;

template <> struct GaugeFmt<GP_F64_18> {
    typedef double R;
    typedef double2 E;
    static constexpr int K = 9;
    static constexpr size_t link_bytes = 144;
    __device__ static __forceinline__ Mat3<R> load(const void* base, int p, int mu, int i, int Vh)
    {
        const double2* b = (const double2*)base + ((size_t)(p * 4 + mu) * 9) * Vh + i;
        Mat3<R> U;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            double2 w = __ldg(b + (size_t)k * Vh);
            U.e[k] = {w.x, w.y};
        }
        return U;
    }
};

// FP64 12-real links (rows 0 and 1; row 2 reconstructed): six double2 per
// link, [p][mu][6][i]
template <> struct GaugeFmt<GP_F64_12> {
    typedef double R;
    typedef double2 E;
    static constexpr int K = 6;
    static constexpr size_t link_bytes = 96;
    __device__ static __forceinline__ Mat3<R> load(const void* base, int p, int mu, int i, int Vh)
    {
        const double2* b = (const double2*)base + ((size_t)(p * 4 + mu) * 6) * Vh + i;
        Mat3<R> U;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            double2 w = __ldg(b + (size_t)k * Vh);
            U.e[k] = {w.x, w.y};
        }
        reconstruct_row2(U);
        return U;
    }
};

template <> struct GaugeFmt<GP_F32_18> {
    typedef float R;
    typedef float2 E;  // storage element: K of them per link, [p][mu][k][i]
    static constexpr int K = 9;
    static constexpr size_t link_bytes = 72;
    __device__ static __forceinline__ Mat3<R> unpack(const E (&w)[K])
    {
        Mat3<R> U;
#pragma unroll
        for (int k = 0; k < 9; ++k) U.e[k] = {w[k].x, w[k].y};
        return U;
    }
    __device__ static __forceinline__ Mat3<R> load(const void* base, int p, int mu, int i, int Vh)
    {
        const E* b = (const E*)base + ((size_t)(p * 4 + mu) * K) * Vh + i;
        E w[K];
#pragma unroll
        for (int k = 0; k < K; ++k) w[k] = __ldg(b + (size_t)k * Vh);
        return unpack(w);
    }
};

template <> struct GaugeFmt<GP_F32_12> {
    typedef float R;
    typedef float4 E;
    static constexpr int K = 3;
    static constexpr size_t link_bytes = 48;
    __device__ static __forceinline__ Mat3<R> unpack(const E (&w)[K])
    {
        Mat3<R> U;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            U.e[2 * k] = {w[k].x, w[k].y};
            U.e[2 * k + 1] = {w[k].z, w[k].w};
        }
        reconstruct_row2(U);
        return U;
    }
    __device__ static __forceinline__ Mat3<R> load(const void* base, int p, int mu, int i, int Vh)
    {
        const E* b = (const E*)base + ((size_t)(p * 4 + mu) * K) * Vh + i;
        E w[K];
#pragma unroll
        for (int k = 0; k < K; ++k) w[k] = __ldg(b + (size_t)k * Vh);
        return unpack(w);
    }
};

// 16-bit 12-real links (the first two rows; the third reconstructed):
// three uint2 per link, each two (re, im) pairs
template <int SPAIR> struct Gauge16Fmt {
    typedef float R;
    typedef uint2 E;
    static constexpr int K = 3;
    static constexpr size_t link_bytes = 24;
    __device__ static __forceinline__ Mat3<R> unpack(const E (&w)[K])
    {
        Mat3<R> U;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float2 f0 = Pair16<SPAIR>::to_float2(w[k].x);
            float2 f1 = Pair16<SPAIR>::to_float2(w[k].y);
            U.e[2 * k] = {f0.x, f0.y};
            U.e[2 * k + 1] = {f1.x, f1.y};
        }
        reconstruct_row2(U);
        return U;
    }
    __device__ static __forceinline__ Mat3<R> load(const void* base, int p, int mu, int i, int Vh)
    {
        const E* b = (const E*)base + ((size_t)(p * 4 + mu) * K) * Vh + i;
        E w[K];
#pragma unroll
        for (int k = 0; k < K; ++k) w[k] = __ldg(b + (size_t)k * Vh);
        return unpack(w);
    }
};

template <> struct GaugeFmt<GP_F16_12> : Gauge16Fmt<SP_F16> {};
template <> struct GaugeFmt<GP_BF16_12> : Gauge16Fmt<SP_BF16> {};

// ---------------------------------------------------------------------------
// error flags written by kernels (never traps)
// ---------------------------------------------------------------------------
enum DeviceErr {
    DEV_OK = 0,
    DEV_ERR_DOMAIN = 1,
    DEV_ERR_BREAKDOWN = 2,
    DEV_ERR_NOT_HERMITIAN = 4,
    DEV_ERR_TIMEOUT = 8,
};

}  // namespace sfh

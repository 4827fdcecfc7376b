// su3.cuh — FP64 3x3 complex algebra, exp(iQ) and a counter-based RNG for
// device kernels.
#pragma once

#include "sfh_core.cuh"

namespace sfh {

typedef Mat3<double> M3;

__device__ __forceinline__ Cx<double> cadd(Cx<double> a, Cx<double> b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Cx<double> csub(Cx<double> a, Cx<double> b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Cx<double> cscale(Cx<double> a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ Cx<double> cconj(Cx<double> a) { return {a.re, -a.im}; }

__device__ __forceinline__ M3 m3_zero()
{
    M3 m;
#pragma unroll
    for (int k = 0; k < 9; ++k) m.e[k] = {0.0, 0.0};
    return m;
}

__device__ __forceinline__ M3 m3_id()
{
    M3 m = m3_zero();
    m.e[0].re = m.e[4].re = m.e[8].re = 1.0;
    return m;
}

// a b
__device__ __forceinline__ M3 m3_mul(const M3& a, const M3& b)
{
    M3 o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Cx<double> s = cmul(a.e[i * 3], b.e[j]);
            s = cadd(s, cmul(a.e[i * 3 + 1], b.e[3 + j]));
            s = cadd(s, cmul(a.e[i * 3 + 2], b.e[6 + j]));
            o.e[i * 3 + j] = s;
        }
    return o;
}

// a b^dag
__device__ __forceinline__ M3 m3_mul_adj(const M3& a, const M3& b)
{
    M3 o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Cx<double> s = cmul(a.e[i * 3], cconj(b.e[j * 3]));
            s = cadd(s, cmul(a.e[i * 3 + 1], cconj(b.e[j * 3 + 1])));
            s = cadd(s, cmul(a.e[i * 3 + 2], cconj(b.e[j * 3 + 2])));
            o.e[i * 3 + j] = s;
        }
    return o;
}

// a^dag b
__device__ __forceinline__ M3 m3_adj_mul(const M3& a, const M3& b)
{
    M3 o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Cx<double> s = cmul(cconj(a.e[i]), b.e[j]);
            s = cadd(s, cmul(cconj(a.e[3 + i]), b.e[3 + j]));
            s = cadd(s, cmul(cconj(a.e[6 + i]), b.e[6 + j]));
            o.e[i * 3 + j] = s;
        }
    return o;
}

__device__ __forceinline__ M3 m3_adj(const M3& a)
{
    M3 o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) o.e[i * 3 + j] = cconj(a.e[j * 3 + i]);
    return o;
}

__device__ __forceinline__ Cx<double> m3_tr(const M3& a)
{
    return {a.e[0].re + a.e[4].re + a.e[8].re, a.e[0].im + a.e[4].im + a.e[8].im};
}

__device__ __forceinline__ void m3_acc(M3& a, const M3& b)
{
#pragma unroll
    for (int k = 0; k < 9; ++k) a.e[k] = cadd(a.e[k], b.e[k]);
}

__device__ __forceinline__ void m3_axpy(M3& a, double s, const M3& b)
{
#pragma unroll
    for (int k = 0; k < 9; ++k) a.e[k] = {a.e[k].re + s * b.e[k].re, a.e[k].im + s * b.e[k].im};
}

__device__ __forceinline__ void m3_traceless(M3& a)
{
    Cx<double> t = m3_tr(a);
    Cx<double> t3 = {t.re / 3.0, t.im / 3.0};
    a.e[0] = csub(a.e[0], t3);
    a.e[4] = csub(a.e[4], t3);
    a.e[8] = csub(a.e[8], t3);
}

// FP64 18-real field access in the even-odd SoA layout
__device__ __forceinline__ M3 ld_link(const void* base, int p, int mu, int i, int Vh)
{
    const double2* b = (const double2*)base + ((size_t)(p * 4 + mu) * 9) * Vh + i;
    M3 U;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        double2 w = b[(size_t)k * Vh];
        U.e[k] = {w.x, w.y};
    }
    return U;
}

__device__ __forceinline__ void st_link(void* base, int p, int mu, int i, int Vh, const M3& U)
{
    double2* b = (double2*)base + ((size_t)(p * 4 + mu) * 9) * Vh + i;
#pragma unroll
    for (int k = 0; k < 9; ++k) b[(size_t)k * Vh] = make_double2(U.e[k].re, U.e[k].im);
}

// sin(x)/x with the reference's small-argument series (Fermions.cpp:834-841)
__device__ __forceinline__ double sinc_stable(double x)
{
    if (fabs(x) <= 0.05) {
        double x2 = x * x;
        return 1.0 - (x2 / 6.0) * (1.0 - (x2 / 20.0) * (1.0 - x2 / 42.0));
    }
    return sin(x) / x;
}

// exp(iQ) for Hermitian traceless Q by Cayley-Hamilton (Morningstar & Peardon,
// hep-lat/0311018), as numerically_stable_matrix_exponential
// (Fermions.cpp:843-902).  Returns false (and leaves out untouched) when Q is
// outside the domain the reference accepts (|Im Tr Q^3| > 1e-10 or Tr Q^2 < 0).
__device__ __forceinline__ bool expiq(const M3& Q, M3& out)
{
    M3 Q2 = m3_mul(Q, Q);
    M3 Q3 = m3_mul(Q2, Q);
    Cx<double> t3 = m3_tr(Q3);
    if (fabs(t3.im) > 1e-10) return false;
    double c0 = t3.re / 3.0;
    double c1 = 0.5 * m3_tr(Q2).re;
    if (c1 < 0.0) return false;
    if (c1 < 1e-12) {
#pragma unroll
        for (int k = 0; k < 9; ++k) out.e[k] = {-Q.e[k].im - 0.5 * Q2.e[k].re, Q.e[k].re - 0.5 * Q2.e[k].im};
        out.e[0].re += 1.0;
        out.e[4].re += 1.0;
        out.e[8].re += 1.0;
        return true;
    }
    bool neg = c0 < 0.0;
    c0 = fabs(c0);
    double c0max = 2.0 * sqrt(c1 * c1 * c1 / 27.0);
    double ratio = 1.0;
    if (c0max > 0.0) ratio = fmin(fmax(c0 / c0max, -1.0), 1.0);
    double theta = acos(ratio);
    double st3, ct3;
    sincos(theta / 3.0, &st3, &ct3);
    double w = sqrt(c1) * st3;
    double u = sqrt(c1 / 3.0) * ct3;
    double xi = sinc_stable(w), cw = cos(w);
    double s2u, c2u, su, cu;
    sincos(2.0 * u, &s2u, &c2u);
    sincos(u, &su, &cu);
    Cx<double> e2u = {c2u, s2u}, emu = {cu, -su};
    double uu = u * u, ww = w * w;
    Cx<double> a0 = {8.0 * uu * cw, 2.0 * u * (3.0 * uu + ww) * xi};
    Cx<double> h0 = cadd(cscale(e2u, uu - ww), cmul(emu, a0));
    Cx<double> a1 = {2.0 * u * cw, -(3.0 * uu - ww) * xi};
    Cx<double> h1 = csub(cscale(e2u, 2.0 * u), cmul(emu, a1));
    Cx<double> a2 = {cw, 3.0 * u * xi};
    Cx<double> h2 = csub(e2u, cmul(emu, a2));
    double den = 9.0 * uu - ww;
    Cx<double> f0 = cscale(h0, 1.0 / den), f1 = cscale(h1, 1.0 / den), f2 = cscale(h2, 1.0 / den);
    if (neg) {
        f0 = cconj(f0);
        f1 = {-f1.re, f1.im};
        f2 = cconj(f2);
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) out.e[k] = cadd(cmul(f1, Q.e[k]), cmul(f2, Q2.e[k]));
    out.e[0] = cadd(out.e[0], f0);
    out.e[4] = cadd(out.e[4], f0);
    out.e[8] = cadd(out.e[8], f0);
    return true;
}

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11) and Box-Muller normals.
// ---------------------------------------------------------------------------
struct Philox {
    __device__ static __forceinline__ uint4 round(uint4 c, uint2 k)
    {
        const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
        uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        return make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    __device__ static __forceinline__ uint4 gen(uint4 c, uint2 k)
    {
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            c = round(c, k);
            k.x += 0x9E3779B9u;
            k.y += 0xBB67AE85u;
        }
        return c;
    }
};

// two N(0,1) doubles from one Philox block (53-bit uniforms in (0,1))
__device__ __forceinline__ double2 normal2(uint4 r)
{
    const double inv53 = 1.0 / 9007199254740992.0;
    unsigned long long a = ((unsigned long long)r.x << 21) ^ (unsigned long long)(r.y >> 11);
    unsigned long long b = ((unsigned long long)r.z << 21) ^ (unsigned long long)(r.w >> 11);
    a &= (1ull << 53) - 1;
    b &= (1ull << 53) - 1;
    double u1 = ((double)a + 0.5) * inv53;
    double u2 = ((double)b + 0.5) * inv53;
    double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    return make_double2(rad * c, rad * s);
}

// n normals for object `id` of stream `stream`
template <int N>
__device__ __forceinline__ void normals(unsigned long long seed, unsigned stream, unsigned long long id,
                                        double (&z)[N])
{
    uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
#pragma unroll
    for (int k = 0; k < (N + 1) / 2; ++k) {
        uint4 ctr = make_uint4((uint32_t)id, (uint32_t)(id >> 32), (uint32_t)k, stream);
        double2 g = normal2(Philox::gen(ctr, key));
        z[2 * k] = g.x;
        if (2 * k + 1 < N) z[2 * k + 1] = g.y;
    }
}

// traceless Hermitian H with N(0,1) diagonal and off-diagonal parts, trace
// removed (the distribution of Lattice.cpp:1001-1033)
__device__ __forceinline__ M3 random_hermitian(unsigned long long seed, unsigned stream,
                                               unsigned long long id)
{
    double z[9];
    normals<9>(seed, stream, id, z);
    M3 H = m3_zero();
    double tr3 = (z[0] + z[1] + z[2]) / 3.0;
    H.e[0].re = z[0] - tr3;
    H.e[4].re = z[1] - tr3;
    H.e[8].re = z[2] - tr3;
    H.e[1] = {z[3], z[4]};
    H.e[3] = {z[3], -z[4]};
    H.e[2] = {z[5], z[6]};
    H.e[6] = {z[5], -z[6]};
    H.e[5] = {z[7], z[8]};
    H.e[7] = {z[7], -z[8]};
    return H;
}

}  // namespace sfh

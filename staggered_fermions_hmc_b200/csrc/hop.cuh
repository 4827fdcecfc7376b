// hop.cuh — the hopping-term arithmetic shared by the solver kernels and the
// standalone Dslash: complex 3x3 matrix-vector products as FMA chains, with
// the hop's scalar factor (eta_mu / 2, the anti-periodic time sign, the
// per-site scale of the 16-bit storages) applied to the input vector.
#pragma once

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
template <int SP, typename R>
__device__ __forceinline__ Vec3<R> hop_input(const void* in, int nq, int j, int Vh, bool neg, R s)
{
    if constexpr (SpinorFmt<SP>::scaled) {
        float sc;
        Vec3<R> v = SpinorFmt<SP>::load_unscaled(in, nq, j, Vh, &sc);
        return vneg_if(v, neg, s * sc);
    } else {
        return vneg_if(vcvt<R>(SpinorFmt<SP>::load(in, nq, j, Vh)), neg, s);
    }
}

}  // namespace
}  // namespace sfh

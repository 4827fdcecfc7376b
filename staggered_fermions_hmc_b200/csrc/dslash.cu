// dslash.cu — even-odd staggered hopping term (the Dslash).
//
// For output parity q the kernel computes, per checkerboard site x,
//   out(x) = a*self(x) + b * 1/2 sum_mu eta_mu(x) [ bc+ U_mu(x) in(x+mu)
//                                               - bc- U_mu(x-mu)^dag in(x-mu) ]
// which is the hopping part K of the reference operators
// D = m + K (Fermions.cpp:218-247) and D^dag = m - K (Fermions.cpp:254-283),
// restricted to one parity (K only couples even and odd sites).  bc+ / bc-
// are -1 on hops that wrap in time (anti-periodic), +1 otherwise.
//
// One thread per output site; the eight links and eight neighbour spinors
// are read with coalesced SoA loads (neighbour spinors are re-read by up to
// eight threads and are served from L1/L2).  The staggered phases and the
// boundary signs are computed from the coordinates, so links stay pure SU(3)
// and can be stored with 12 reals.  The reduced-precision storages use the
// solver's hop arithmetic (hop.cuh): for FP16 links and vectors packed-half
// products accumulated in FP32 with eta_mu / 2, the time-wrap sign and the
// site scale; for the others FMA chains with that factor on the input
// vector.
#include "hop.cuh"
#include "sfh_internal.h"
#include "tstage.cuh"

namespace sfh {

namespace {

template <typename To, typename From>
__device__ __forceinline__ Vec3<To> cvt(const Vec3<From>& v)
{
    Vec3<To> o;
#pragma unroll
    for (int k = 0; k < 3; ++k) o.c[k] = {(To)v.c[k].re, (To)v.c[k].im};
    return o;
}

template <typename R>
__device__ __forceinline__ void acc_add(Vec3<R>& acc, const Vec3<R>& w, bool neg)
{
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (neg) { acc.c[k].re -= w.c[k].re; acc.c[k].im -= w.c[k].im; }
        else     { acc.c[k].re += w.c[k].re; acc.c[k].im += w.c[k].im; }
    }
}

}  // namespace

// Hopping sum for one output site: sum_mu eta_mu [bc U in(x+mu) - bc U^dag
// in(x-mu)], times 1/2 in the FMA-chain form (every format but FP64-18),
// without it in FP64-18's own form (halved by the caller).
template <int GP> struct HopHalfInside {
    static constexpr bool v = GP != GP_F64_18;
};

template <int GP, int SPI>
__device__ __forceinline__ Vec3<typename GaugeFmt<GP>::R> hop_site(const Geom& g, const Coord& c,
                                                                   int q, int i, const void* gauge,
                                                                   const void* in)
{
    typedef typename GaugeFmt<GP>::R R;
    typedef typename SpinorFmt<SPI>::R RI;
    Vec3<R> acc;
#pragma unroll
    for (int k = 0; k < 3; ++k) acc.c[k] = {R(0), R(0)};
    if constexpr (GP == GP_F16_12 && SPI == SP_F16) {
        // FP16 links and vectors: packed-half products, FP32 accumulation
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            const float s = eta_sign(c, mu) < 0 ? -0.5f : 0.5f;
            const int lu = lex_up(g, c, mu) >> 1;
            const int ld = lex_dn(g, c, mu) >> 1;
            const bool wrap_up = (mu == 3) && (c.x[3] == g.L[3] - 1);
            const bool wrap_dn = (mu == 3) && (c.x[3] == 0);
            __half2 U[9];
            hlink_load<false>(nullptr, 0, gauge, 0, q, mu, i, g.Vh, U);
            hop_half<false>(acc, U, in, 1 - q, lu, g.Vh, wrap_up ? -s : s);
            hlink_load<false>(nullptr, 0, gauge, 0, 1 - q, mu, ld, g.Vh, U);
            hop_half<true>(acc, U, in, 1 - q, ld, g.Vh, wrap_dn ? s : -s);
        }
    } else if constexpr (HopHalfInside<GP>::v) {
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            const R s = eta_sign(c, mu) < 0 ? R(-0.5) : R(0.5);
            const int lu = lex_up(g, c, mu) >> 1;
            const int ld = lex_dn(g, c, mu) >> 1;
            const bool wrap_up = (mu == 3) && (c.x[3] == g.L[3] - 1);
            const bool wrap_dn = (mu == 3) && (c.x[3] == 0);
            mv_add<false>(acc, GaugeFmt<GP>::load(gauge, q, mu, i, g.Vh),
                          hop_input<SPI>(in, 1 - q, lu, g.Vh, wrap_up, s));
            mdv_sub(acc, GaugeFmt<GP>::load(gauge, 1 - q, mu, ld, g.Vh),
                    hop_input<SPI>(in, 1 - q, ld, g.Vh, wrap_dn, s));
        }
    } else {
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            bool eta_neg = eta_sign(c, mu) < 0;
            int lu = lex_up(g, c, mu) >> 1;
            int ld = lex_dn(g, c, mu) >> 1;
            bool wrap_up = (mu == 3) && (c.x[3] == g.L[3] - 1);
            bool wrap_dn = (mu == 3) && (c.x[3] == 0);
            Mat3<R> U = GaugeFmt<GP>::load(gauge, q, mu, i, g.Vh);
            Vec3<R> v = cvt<R, RI>(SpinorFmt<SPI>::load(in, 1 - q, lu, g.Vh));
            acc_add(acc, mul_mv(U, v), eta_neg != wrap_up);
            Mat3<R> Ud = GaugeFmt<GP>::load(gauge, 1 - q, mu, ld, g.Vh);
            Vec3<R> w = cvt<R, RI>(SpinorFmt<SPI>::load(in, 1 - q, ld, g.Vh));
            acc_add(acc, mul_adj_mv(Ud, w), !(eta_neg != wrap_dn));
        }
    }
    return acc;
}

namespace {

// five resident blocks for the FP32 arithmetic formats (at most 51
// registers; they fit in 48 without spills), the compiler's choice for FP64
template <int GP> struct HopMinBlocks {
    static constexpr int v = sizeof(typename GaugeFmt<GP>::R) == 4 ? 5 : 0;
};

template <int GP, int SPI, int SPO, bool SELF>
__global__ void __launch_bounds__(256, HopMinBlocks<GP>::v) hop_kernel(Geom g, const void* __restrict__ gauge,
                                                  const void* __restrict__ in, const void* self,
                                                  void* out, double a, double b, int q0)
{
    typedef typename GaugeFmt<GP>::R R;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int q = q0 + blockIdx.y;
    if (i >= g.Vh) return;
    Coord c = eo_coords(g, q, i);
    Vec3<R> acc = hop_site<GP, SPI>(g, c, q, i, gauge, in);
    R hb = (R)(HopHalfInside<GP>::v ? b : 0.5 * b);
    Vec3<R> res;
#pragma unroll
    for (int k = 0; k < 3; ++k) res.c[k] = {hb * acc.c[k].re, hb * acc.c[k].im};
    if (SELF) {
        Vec3<R> sv = cvt<R, typename SpinorFmt<SPO>::R>(SpinorFmt<SPO>::load(self, q, i, g.Vh));
        R ra = (R)a;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            res.c[k].re = ra * sv.c[k].re + res.c[k].re;
            res.c[k].im = ra * sv.c[k].im + res.c[k].im;
        }
    }
    SpinorFmt<SPO>::store(out, q, i, g.Vh, cvt<typename SpinorFmt<SPO>::R, R>(res));
}

// The 16-bit storages with the neighbour vectors staged along the time
// direction (tstage.cuh): the block's 256 output sites take their time and z
// neighbours from one bulk copy of [i0 - Lt/2, i0 + 256 + Lt/2) into shared
// memory, the x and y neighbours and the links from global memory.  The
// arithmetic is hop_site's, operand for operand, so the result is
// bit-identical to hop_kernel's.
// extra_tx (a test hook, normally 0): bytes announced on the barrier beyond
// the copy's, so that its phase never completes and every wait runs out.
template <int GP, int SP, bool SELF>
__global__ void __launch_bounds__(256, HopMinBlocks<GP>::v)
    hop_kernel_tstaged(Geom g, const void* __restrict__ gauge, const void* __restrict__ in, const void* self,
                       void* out, double a, double b, int q0, int* err, unsigned extra_tx)
{
    static_assert(SpinorFmt<SP>::scaled, "staging covers the one-word-per-site storages");
    extern __shared__ __align__(16) uint4 s_nb[];
    __shared__ __align__(8) unsigned long long s_bar;
    const int q = q0 + blockIdx.y, nq = 1 - q;
    const int i0 = blockIdx.x * blockDim.x, i = i0 + threadIdx.x;
    const uint4* src = (const uint4*)in + (size_t)nq * g.Vh;
    const TRange r = trange(g, i0, blockDim.x);
    if (threadIdx.x == 0) mbar_init(&s_bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&s_bar, (unsigned)r.cnt * 16u + extra_tx);
        bulk_copy_g2s(s_nb, src + r.lo, (unsigned)r.cnt * 16u, &s_bar);
    }
    if (i >= g.Vh) return;  // every block has a site of its own, whose thread waits
    const Coord c = eo_coords(g, q, i);
    bool ok = mbar_wait_bounded(&s_bar, 0);
    if (!ok) {
        atomicOr(err, DEV_ERR_TIMEOUT);
        mbar_wait_bounded(&s_bar, 0);  // the copy in flight, before the block may leave
    }
    Vec3<float> acc;
#pragma unroll
    for (int k = 0; k < 3; ++k) acc.c[k] = {0.f, 0.f};
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        const float s = eta_sign(c, mu) < 0 ? -0.5f : 0.5f;
        const uint4 wu = nbr_word(s_nb, r, ok, src, lex_up(g, c, mu) >> 1);
        const int ld = lex_dn(g, c, mu) >> 1;
        const uint4 wd = nbr_word(s_nb, r, ok, src, ld);
        const bool wrap_up = (mu == 3) && (c.x[3] == g.L[3] - 1);
        const bool wrap_dn = (mu == 3) && (c.x[3] == 0);
        if constexpr (GP == GP_F16_12) {
            __half2 U[9];
            hlink_load<false>(nullptr, 0, gauge, 0, q, mu, i, g.Vh, U);
            hop_half_word<false>(acc, U, wu, wrap_up ? -s : s);
            hlink_load<false>(nullptr, 0, gauge, 0, nq, mu, ld, g.Vh, U);
            hop_half_word<true>(acc, U, wd, wrap_dn ? s : -s);
        } else {
            mv_add<false>(acc, GaugeFmt<GP>::load(gauge, q, mu, i, g.Vh), hop_input_word<SP, float>(wu, wrap_up, s));
            mdv_sub(acc, GaugeFmt<GP>::load(gauge, nq, mu, ld, g.Vh), hop_input_word<SP, float>(wd, wrap_dn, s));
        }
    }
    const float hb = (float)b;
    Vec3<float> res;
#pragma unroll
    for (int k = 0; k < 3; ++k) res.c[k] = {hb * acc.c[k].re, hb * acc.c[k].im};
    if (SELF) {
        Vec3<float> sv = SpinorFmt<SP>::load(self, q, i, g.Vh);
        const float ra = (float)a;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            res.c[k].re = ra * sv.c[k].re + res.c[k].re;
            res.c[k].im = ra * sv.c[k].im + res.c[k].im;
        }
    }
    SpinorFmt<SP>::store(out, q, i, g.Vh, res);
}

template <int GP, int SP>
void launch_typed_tstaged(const Geom& g, const void* gauge, const void* in, void* out, const void* self, double a,
                          double b, int q0, int nq, int* err, unsigned extra_tx, cudaStream_t s)
{
    dim3 grid((g.Vh + 255) / 256, nq);
    const size_t smem = (size_t)tstage_words(256, g.L[3]) * sizeof(uint4);
    if (self)
        hop_kernel_tstaged<GP, SP, true><<<grid, 256, smem, s>>>(g, gauge, in, self, out, a, b, q0, err, extra_tx);
    else
        hop_kernel_tstaged<GP, SP, false><<<grid, 256, smem, s>>>(g, gauge, in, self, out, a, b, q0, err, extra_tx);
}

template <int GP, int SP>
void launch_typed(const Geom& g, const void* gauge, const void* in, void* out, const void* self,
                  double a, double b, int q0, int nq, cudaStream_t s)
{
    dim3 grid((g.Vh + 255) / 256, nq);
    if (self)
        hop_kernel<GP, SP, SP, true><<<grid, 256, 0, s>>>(g, gauge, in, self, out, a, b, q0);
    else
        hop_kernel<GP, SP, SP, false><<<grid, 256, 0, s>>>(g, gauge, in, self, out, a, b, q0);
}

// even-odd FP64 vectors (both parities) to storage format SP, or back
template <int SP, bool TO_FMT>
__global__ void __launch_bounds__(256) convert_spinor(Geom g, const void* __restrict__ src, void* __restrict__ dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y;
    if (i >= g.Vh) return;
    typedef typename SpinorFmt<SP>::R R;
    if (TO_FMT)
        SpinorFmt<SP>::store(dst, p, i, g.Vh, cvt<R, double>(SpinorFmt<SP_F64>::load(src, p, i, g.Vh)));
    else
        SpinorFmt<SP_F64>::store(dst, p, i, g.Vh, cvt<double, R>(SpinorFmt<SP>::load(src, p, i, g.Vh)));
}

template <int SP>
void launch_convert(const Geom& g, bool to_fmt, const void* src, void* dst, cudaStream_t s)
{
    dim3 grid((g.Vh + 255) / 256, 2);
    if (to_fmt)
        convert_spinor<SP, true><<<grid, 256, 0, s>>>(g, src, dst);
    else
        convert_spinor<SP, false><<<grid, 256, 0, s>>>(g, src, dst);
}

}  // namespace

void launch_spinor_convert(const Geom& g, int sp, bool to_fmt, const void* src, void* dst, cudaStream_t s)
{
    if (sp == SP_F32) launch_convert<SP_F32>(g, to_fmt, src, dst, s);
    else if (sp == SP_F16) launch_convert<SP_F16>(g, to_fmt, src, dst, s);
    else if (sp == SP_BF16) launch_convert<SP_BF16>(g, to_fmt, src, dst, s);
    else launch_convert<SP_F64>(g, to_fmt, src, dst, s);
}

bool hop_tstaged_fits(const Geom& g)
{
    return (size_t)tstage_words(256, g.L[3]) * sizeof(uint4) <= 48 * 1024;
}

void launch_hop_tstaged(const Geom& g, int gauge_prec, const void* gauge, const void* in, void* out,
                        const void* self, double a, double b, int q0, int nq, int* err, unsigned extra_tx,
                        cudaStream_t s)
{
    if (gauge_prec == GP_F16_12)
        launch_typed_tstaged<GP_F16_12, SP_F16>(g, gauge, in, out, self, a, b, q0, nq, err, extra_tx, s);
    else if (gauge_prec == GP_BF16_12)
        launch_typed_tstaged<GP_BF16_12, SP_BF16>(g, gauge, in, out, self, a, b, q0, nq, err, extra_tx, s);
}

void launch_hop(const Geom& g, int gauge_prec, const void* gauge, int in_prec, const void* in,
                int out_prec, void* out, const void* self, double a, double b, int q0, int nq,
                cudaStream_t s)
{
    (void)out_prec;
    if (gauge_prec == GP_F64_18 && in_prec == SP_F64)
        launch_typed<GP_F64_18, SP_F64>(g, gauge, in, out, self, a, b, q0, nq, s);
    else if (gauge_prec == GP_F32_12 && in_prec == SP_F32)
        launch_typed<GP_F32_12, SP_F32>(g, gauge, in, out, self, a, b, q0, nq, s);
    else if (gauge_prec == GP_F16_12 && in_prec == SP_F16)
        launch_typed<GP_F16_12, SP_F16>(g, gauge, in, out, self, a, b, q0, nq, s);
    else if (gauge_prec == GP_F32_18 && in_prec == SP_F32)
        launch_typed<GP_F32_18, SP_F32>(g, gauge, in, out, self, a, b, q0, nq, s);
    else if (gauge_prec == GP_BF16_12 && in_prec == SP_BF16)
        launch_typed<GP_BF16_12, SP_BF16>(g, gauge, in, out, self, a, b, q0, nq, s);
    else if (gauge_prec == GP_F64_12 && in_prec == SP_F64)
        launch_typed<GP_F64_12, SP_F64>(g, gauge, in, out, self, a, b, q0, nq, s);
}

}  // namespace sfh

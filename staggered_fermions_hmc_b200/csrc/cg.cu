// cg.cu — persistent, batched conjugate-gradient solver for D D^dag x = b.
//
// Restates solve_CG_DDdagger (Fermions.cpp:553-617) for the GPU.  D D^dag =
// m^2 - K^2 and K couples only even and odd sites, so D D^dag is block
// diagonal in parity: M_pp = m^2 - K_{p,1-p} K_{1-p,p}.
//
// One cooperative launch solves every "lane" of a batch: a lane is one
// (system, right-hand side, parity block) CG, or one (system, RHS) CG over
// both parities with shared scalars (the reference's full-lattice CG, used
// for FP64 parity).  Systems may differ in lattice size and mass.  Each CG
// iteration is three grid-wide phases separated by grid.sync():
//
//   P1  t = K p_new,     p_new = r + beta p computed at the neighbours
//   P2  p = p_new, v = m^2 p - K t, partial <p, v>      -> alpha
//   P3  x += alpha p, r -= alpha v, partial <r, r>       -> beta / convergence
//
// Work is split into tiles of 256 sites of one system and one output parity;
// every tile processes all lanes of its system that are active in the phase,
// so a link loaded once serves every right-hand side (RHS blocking).
//
// Reductions are deterministic: each tile writes one FP64 partial per lane;
// the tile that completes a lane's count (atomic ticket) sums the partials in
// a fixed order and updates that lane's FP64 scalars.
//
// Mixed precision (FP32 or FP16+scale vectors with FP32/FP16 12-real links):
// x is accumulated in FP32 between reliable updates.  When |r| has dropped by
// delta since the last update, or the iterated residual meets the target, the
// lane spends one iteration on an FP64 reliable update: x_hi += x_lo and
// r = b - M x_hi recomputed with FP64 links and vectors.  A mixed lane
// converges only on that FP64 true residual.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "sfh_internal.h"

namespace cgrp = cooperative_groups;

namespace sfh {

enum { LM_ACTIVE = 0, LM_RU = 1, LM_DONE = 2, LM_FAILED = 3 };
constexpr int kTile = 256;

struct CgSys {
    Geom g;
    double m2;
    const void* U64;
    const void* Ulo;
    int lane0, nrhs, both, tile0, ntq;
};

struct CgRhs {
    void* b;    // FP64 right-hand side
    void* xhi;  // FP64 solution
    void* thi;  // FP64 temporary (reliable updates)
    void* r;    // residual (solver precision)
    void* p;    // search direction
    void* v;    // M p
    void* t;    // K p on the other parity
    void* xlo;  // low-precision solution increment (FP32; == xhi for FP64)
};

struct CgLane {
    int sys, rhs, parity, poff;
    double bb, target, rr, rr_old, pAp, alpha, beta, rmax;
    int mode[2];
    int iters, nru, status, pad;
    unsigned int ticket, pad2;
};

struct CgArgs {
    int nsys, nlanes, ntiles;
    const CgSys* sys;
    const CgRhs* rhs;
    CgLane* lanes;
    const int* tile_sys;
    double* partial;
    int* n_active;
    double tol2, delta;
    int maxit, maxloop, mixed;
};

namespace {

template <int SP> struct XFmt { static constexpr int v = SP_F32; };
template <> struct XFmt<SP_F64> { static constexpr int v = SP_F64; };

__device__ __forceinline__ int ld_int(const int* p) { return __ldcg(p); }
__device__ __forceinline__ double ld_dbl(const double* p) { return __ldcg(p); }

__device__ __forceinline__ int lane_of(const CgSys& S, int rhs, int q, bool hop1)
{
    if (S.both) return S.lane0 + rhs;
    int lp = hop1 ? 1 - q : q;
    return S.lane0 + rhs * 2 + lp;
}

template <typename R>
__device__ __forceinline__ void vzero(Vec3<R>& a)
{
#pragma unroll
    for (int k = 0; k < 3; ++k) a.c[k] = {R(0), R(0)};
}

template <typename R>
__device__ __forceinline__ void vacc(Vec3<R>& acc, const Vec3<R>& w, bool neg)
{
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (neg) { acc.c[k].re -= w.c[k].re; acc.c[k].im -= w.c[k].im; }
        else     { acc.c[k].re += w.c[k].re; acc.c[k].im += w.c[k].im; }
    }
}

template <typename To, typename From>
__device__ __forceinline__ Vec3<To> vcvt(const Vec3<From>& v)
{
    Vec3<To> o;
#pragma unroll
    for (int k = 0; k < 3; ++k) o.c[k] = {(To)v.c[k].re, (To)v.c[k].im};
    return o;
}

// a + s*b with explicit fused multiply-add (identical rounding in every phase)
__device__ __forceinline__ Vec3<float> vaxpy(const Vec3<float>& a, float s, const Vec3<float>& b)
{
    Vec3<float> o;
#pragma unroll
    for (int k = 0; k < 3; ++k) o.c[k] = {fmaf(s, b.c[k].re, a.c[k].re), fmaf(s, b.c[k].im, a.c[k].im)};
    return o;
}
__device__ __forceinline__ Vec3<double> vaxpy(const Vec3<double>& a, double s, const Vec3<double>& b)
{
    Vec3<double> o;
#pragma unroll
    for (int k = 0; k < 3; ++k) o.c[k] = {fma(s, b.c[k].re, a.c[k].re), fma(s, b.c[k].im, a.c[k].im)};
    return o;
}

template <typename R>
__device__ __forceinline__ double vdot_re(const Vec3<R>& a, const Vec3<R>& b)
{
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) s += (double)a.c[k].re * (double)b.c[k].re + (double)a.c[k].im * (double)b.c[k].im;
    return s;
}

// Block sum of N doubles; result valid in thread 0.  Fixed reduction tree.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double* smem)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < N; ++k) smem[warp * N + k] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            double x = lane < nw ? smem[lane * N + k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
    __syncthreads();
}

// Sum of n partial slots by one warp in a fixed order (all lanes get it).
__device__ __forceinline__ double warp_sum_slots(const double* slots, int n)
{
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    for (int k = lane; k < n; k += 32) s += __ldcg(slots + k);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

__device__ __forceinline__ void set_mode_final(CgLane* L, int mode, int status, int* n_active)
{
    L->mode[0] = mode;
    L->mode[1] = mode;
    L->status = status;
    atomicSub(n_active, 1);
}

struct TileInfo {
    int q, slot, i;
    bool valid;
};

__device__ __forceinline__ TileInfo decode_tile(const CgSys& S, int t)
{
    TileInfo ti;
    int local = t - S.tile0;
    ti.q = local >= S.ntq ? 1 : 0;
    int j = local - ti.q * S.ntq;
    ti.slot = local;
    ti.i = j * kTile + (int)threadIdx.x;
    ti.valid = ti.i < S.g.Vh;
    return ti;
}

__device__ __forceinline__ int lane_slot0(const CgSys& S, int parity)
{
    return S.both ? 0 : parity * S.ntq;
}

__device__ __forceinline__ int lane_nslots(const CgSys& S) { return S.both ? 2 * S.ntq : S.ntq; }

// pointer fields of the per-RHS vector table (read-only during the kernel)
enum RhsField { F_B = 0, F_XHI, F_THI, F_R, F_P, F_V, F_T, F_XLO };
__device__ __forceinline__ void* rhs_ptr(const CgArgs& a, int rid, int f)
{
    const unsigned long long* base = reinterpret_cast<const unsigned long long*>(a.rhs + rid);
    return reinterpret_cast<void*>(__ldg(base + f));
}

// Publish this tile's partials and take the lanes' tickets; returns the mask
// of lanes (within the pass) whose count this block completed.
template <int NB>
__device__ __forceinline__ unsigned arrive(const CgArgs& a, const CgSys& S, const int (&lanes)[NB],
                                           const bool (&part)[NB], const double (&sums)[NB], int slot,
                                           unsigned* s_mask)
{
    if (threadIdx.x == 0) {
        unsigned mask = 0;
#pragma unroll
        for (int l = 0; l < NB; ++l)
            if (part[l]) __stcg(a.partial + a.lanes[lanes[l]].poff + slot, sums[l]);
        __threadfence();
        const unsigned expected = S.both ? 2u * S.ntq : (unsigned)S.ntq;
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            if (!part[l]) continue;
            CgLane* L = a.lanes + lanes[l];
            unsigned old = atomicAdd(&L->ticket, 1u);
            if (old == expected - 1) {
                L->ticket = 0;
                mask |= 1u << l;
            }
        }
        if (mask) __threadfence();
        *s_mask = mask;
    }
    __syncthreads();
    return *s_mask;
}

// ---------------------------------------------------------------------------
// lane scalar updates, run by warp 0 of the block that completed a ticket
// ---------------------------------------------------------------------------
__device__ __noinline__ void finish_init(const CgArgs& a, const CgSys& S, int lane)
{
    CgLane* L = a.lanes + lane;
    double bb = warp_sum_slots(a.partial + L->poff + lane_slot0(S, L->parity), lane_nslots(S));
    if (threadIdx.x == 0) {
        L->bb = bb;
        L->target = a.tol2 * bb;
        L->rr = bb;
        L->rr_old = bb;
        L->rmax = sqrt(bb);
        L->beta = 0.0;
        L->alpha = 0.0;
        L->iters = 0;
        L->nru = 0;
        if (bb < 1e-28) {  // Fermions.cpp:562-564: X = 0
            set_mode_final(L, LM_DONE, SFH_OK, a.n_active);
        } else {
            L->mode[0] = LM_ACTIVE;
            L->mode[1] = LM_ACTIVE;
        }
    }
}

__device__ __noinline__ void finish_hop2(const CgArgs& a, const CgSys& S, int lane, int mode, int cur)
{
    CgLane* L = a.lanes + lane;
    double s = warp_sum_slots(a.partial + L->poff + lane_slot0(S, L->parity), lane_nslots(S));
    if (threadIdx.x != 0) return;
    const int nxt = cur ^ 1;
    if (mode == LM_ACTIVE) {  // s = <p, M p>; Fermions.cpp:573-586
        L->pAp = s;
        double alpha = L->rr / s;
        if (!isfinite(s) || fabs(s) < 1e-30 || !isfinite(alpha)) {
            set_mode_final(L, LM_FAILED, SFH_ERR_BREAKDOWN, a.n_active);
        } else {
            L->alpha = alpha;
            L->mode[nxt] = LM_ACTIVE;
        }
    } else {  // reliable update finished: s = |b - M x|^2 in FP64
        L->nru += 1;
        if (s < L->target) {
            L->rr = s;
            set_mode_final(L, LM_DONE, SFH_OK, a.n_active);
        } else if (!isfinite(s)) {
            set_mode_final(L, LM_FAILED, SFH_ERR_BREAKDOWN, a.n_active);
        } else if (L->iters >= a.maxit) {
            L->rr = s;
            set_mode_final(L, LM_FAILED, SFH_ERR_NOCONV, a.n_active);
        } else {
            L->beta = s / L->rr_old;
            L->rr = s;
            L->rmax = sqrt(s);
            L->mode[nxt] = LM_ACTIVE;
        }
    }
}

__device__ __noinline__ void finish_update(const CgArgs& a, const CgSys& S, int lane, int cur)
{
    CgLane* L = a.lanes + lane;
    double rn = warp_sum_slots(a.partial + L->poff + lane_slot0(S, L->parity), lane_nslots(S));
    if (threadIdx.x != 0) return;
    const int nxt = cur ^ 1;
    L->iters += 1;
    if (!isfinite(rn)) {
        set_mode_final(L, LM_FAILED, SFH_ERR_BREAKDOWN, a.n_active);
    } else if (!a.mixed) {
        double beta = rn / L->rr;  // Fermions.cpp:594-601
        if (!isfinite(beta)) {
            set_mode_final(L, LM_FAILED, SFH_ERR_BREAKDOWN, a.n_active);
        } else {
            L->beta = beta;
            L->rr = rn;
            if (rn < L->target)  // Fermions.cpp:569
                set_mode_final(L, LM_DONE, SFH_OK, a.n_active);
            else if (L->iters >= a.maxit)  // Fermions.cpp:609-614
                set_mode_final(L, LM_FAILED, SFH_ERR_NOCONV, a.n_active);
            else
                L->mode[nxt] = LM_ACTIVE;
        }
    } else {
        double r = sqrt(rn);
        if (rn < L->target || r < a.delta * L->rmax || L->iters >= a.maxit) {
            L->rr_old = L->rr;
            L->rr = rn;
            L->mode[nxt] = LM_RU;
        } else {
            L->beta = rn / L->rr;
            L->rr = rn;
            L->rmax = fmax(L->rmax, r);
            L->mode[nxt] = LM_ACTIVE;
        }
    }
}

// ---------------------------------------------------------------------------
// reliable-update site kernels (FP64 links and vectors), rare
// ---------------------------------------------------------------------------
template <int XP>
__device__ __noinline__ void ru_hop1_site(const CgArgs& a, const CgSys& S, const Coord& c, int q,
                                          int i, int rid)
{
    const int nq = 1 - q, Vh = S.g.Vh;
    const void* xhi = rhs_ptr(a, rid, F_XHI);
    const void* xlo = rhs_ptr(a, rid, F_XLO);
    Vec3<double> acc;
    vzero(acc);
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        const bool eta_neg = eta_sign(c, mu) < 0;
        const int lu = lex_up(S.g, c, mu) >> 1, ld = lex_dn(S.g, c, mu) >> 1;
        const bool wu = (mu == 3) && (c.x[3] == S.g.L[3] - 1);
        const bool wd = (mu == 3) && (c.x[3] == 0);
        Mat3<double> U = GaugeFmt<GP_F64_18>::load(S.U64, q, mu, i, Vh);
        Vec3<double> xu = vaxpy(SpinorFmt<SP_F64>::load_cg(xhi, nq, lu, Vh), 1.0,
                                vcvt<double>(SpinorFmt<XP>::load_cg(xlo, nq, lu, Vh)));
        vacc(acc, mul_mv(U, xu), eta_neg != wu);
        Mat3<double> Ud = GaugeFmt<GP_F64_18>::load(S.U64, nq, mu, ld, Vh);
        Vec3<double> xd = vaxpy(SpinorFmt<SP_F64>::load_cg(xhi, nq, ld, Vh), 1.0,
                                vcvt<double>(SpinorFmt<XP>::load_cg(xlo, nq, ld, Vh)));
        vacc(acc, mul_adj_mv(Ud, xd), !(eta_neg != wd));
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) acc.c[k] = {0.5 * acc.c[k].re, 0.5 * acc.c[k].im};
    SpinorFmt<SP_F64>::store(rhs_ptr(a, rid, F_THI), q, i, Vh, acc);
}

template <int SP, int XP>
__device__ __noinline__ double ru_hop2_site(const CgArgs& a, const CgSys& S, const Coord& c, int q,
                                            int i, int rid)
{
    typedef typename SpinorFmt<SP>::R RS;
    const int nq = 1 - q, Vh = S.g.Vh;
    const void* thi = rhs_ptr(a, rid, F_THI);
    Vec3<double> acc;
    vzero(acc);
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        const bool eta_neg = eta_sign(c, mu) < 0;
        const int lu = lex_up(S.g, c, mu) >> 1, ld = lex_dn(S.g, c, mu) >> 1;
        const bool wu = (mu == 3) && (c.x[3] == S.g.L[3] - 1);
        const bool wd = (mu == 3) && (c.x[3] == 0);
        Mat3<double> U = GaugeFmt<GP_F64_18>::load(S.U64, q, mu, i, Vh);
        vacc(acc, mul_mv(U, SpinorFmt<SP_F64>::load_cg(thi, nq, lu, Vh)), eta_neg != wu);
        Mat3<double> Ud = GaugeFmt<GP_F64_18>::load(S.U64, nq, mu, ld, Vh);
        vacc(acc, mul_adj_mv(Ud, SpinorFmt<SP_F64>::load_cg(thi, nq, ld, Vh)), !(eta_neg != wd));
    }
    void* xhi = rhs_ptr(a, rid, F_XHI);
    void* xlo = rhs_ptr(a, rid, F_XLO);
    Vec3<double> xn = vaxpy(SpinorFmt<SP_F64>::load_cg(xhi, q, i, Vh), 1.0,
                            vcvt<double>(SpinorFmt<XP>::load_cg(xlo, q, i, Vh)));
    SpinorFmt<SP_F64>::store(xhi, q, i, Vh, xn);
    Vec3<typename SpinorFmt<XP>::R> z;
    vzero(z);
    SpinorFmt<XP>::store(xlo, q, i, Vh, z);
    Vec3<double> b = SpinorFmt<SP_F64>::load_cg(rhs_ptr(a, rid, F_B), q, i, Vh);
    Vec3<double> res;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        res.c[k].re = b.c[k].re - (S.m2 * xn.c[k].re - 0.5 * acc.c[k].re);
        res.c[k].im = b.c[k].im - (S.m2 * xn.c[k].im - 0.5 * acc.c[k].im);
    }
    SpinorFmt<SP>::store(rhs_ptr(a, rid, F_R), q, i, Vh, vcvt<RS>(res));
    return vdot_re(res, res);
}

// gather the lanes of one RHS pass
template <int NB>
__device__ __forceinline__ void gather(const CgArgs& a, const CgSys& S, int base, int cnt, int q,
                                       bool hop1, int cur, int (&lanes)[NB], int (&mode)[NB],
                                       int (&rid)[NB])
{
#pragma unroll
    for (int l = 0; l < NB; ++l) {
        lanes[l] = 0;
        mode[l] = LM_DONE;
        rid[l] = 0;
        if (l < cnt) {
            lanes[l] = lane_of(S, base + l, q, hop1);
            const CgLane* L = a.lanes + lanes[l];
            mode[l] = ld_int(&L->mode[cur]);
            rid[l] = __ldg(&L->rhs);
        }
    }
}

// ---------------------------------------------------------------------------
// P0: x = 0, r = b, p = 0; |b|^2
// ---------------------------------------------------------------------------
template <int GP, int SP, int NB>
__device__ void phase_init(const CgArgs& a, const CgSys& S, int t, double* smem, unsigned* s_mask)
{
    typedef typename SpinorFmt<SP>::R R;
    constexpr int XP = XFmt<SP>::v;
    const TileInfo ti = decode_tile(S, t);
    const int Vh = S.g.Vh;
    for (int base = 0; base < S.nrhs; base += NB) {
        const int cnt = min(NB, S.nrhs - base);
        int lanes[NB], rid[NB], mode[NB];
        bool part[NB];
        double sums[NB];
        gather<NB>(a, S, base, cnt, ti.q, false, 0, lanes, mode, rid);
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            sums[l] = 0.0;
            part[l] = l < cnt;
            if (l >= cnt || !ti.valid) continue;
            Vec3<double> b = SpinorFmt<SP_F64>::load_cg(rhs_ptr(a, rid[l], F_B), ti.q, ti.i, Vh);
            Vec3<double> z;
            vzero(z);
            SpinorFmt<SP_F64>::store(rhs_ptr(a, rid[l], F_XHI), ti.q, ti.i, Vh, z);
            if (a.mixed)
                SpinorFmt<XP>::store(rhs_ptr(a, rid[l], F_XLO), ti.q, ti.i, Vh,
                                     vcvt<typename SpinorFmt<XP>::R>(z));
            SpinorFmt<SP>::store(rhs_ptr(a, rid[l], F_R), ti.q, ti.i, Vh, vcvt<R>(b));
            SpinorFmt<SP>::store(rhs_ptr(a, rid[l], F_P), ti.q, ti.i, Vh, vcvt<R>(z));
            sums[l] = vdot_re(b, b);
        }
        block_sum<NB>(sums, smem);
        unsigned mask = arrive<NB>(a, S, lanes, part, sums, ti.slot, s_mask);
        if (mask && threadIdx.x < 32) {
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (mask & (1u << l)) finish_init(a, S, lanes[l]);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// P1: t = K (r + beta p) for normal lanes; thi = K (x_hi + x_lo) for lanes in
// a reliable update.  Output parity q, inputs on parity 1-q.
// ---------------------------------------------------------------------------
template <int GP, int SP, int NB>
__device__ void phase_hop1(const CgArgs& a, const CgSys& S, int t, int cur)
{
    typedef typename GaugeFmt<GP>::R R;
    typedef typename SpinorFmt<SP>::R RS;
    constexpr int XP = XFmt<SP>::v;
    const TileInfo ti = decode_tile(S, t);
    if (!ti.valid) return;
    const Coord c = eo_coords(S.g, ti.q, ti.i);
    const int q = ti.q, nq = 1 - ti.q, Vh = S.g.Vh;
    for (int base = 0; base < S.nrhs; base += NB) {
        const int cnt = min(NB, S.nrhs - base);
        int lanes[NB], rid[NB], mode[NB];
        RS beta[NB];
        gather<NB>(a, S, base, cnt, q, true, cur, lanes, mode, rid);
        bool anyA = false, anyR = false;
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            anyA |= mode[l] == LM_ACTIVE;
            anyR |= mode[l] == LM_RU;
            beta[l] = mode[l] == LM_ACTIVE ? (RS)ld_dbl(&a.lanes[lanes[l]].beta) : RS(0);
        }
        if (anyA) {
            Vec3<R> acc[NB];
#pragma unroll
            for (int l = 0; l < NB; ++l) vzero(acc[l]);
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
                const bool eta_neg = eta_sign(c, mu) < 0;
                const int lu = lex_up(S.g, c, mu) >> 1, ld = lex_dn(S.g, c, mu) >> 1;
                const bool wu = (mu == 3) && (c.x[3] == S.g.L[3] - 1);
                const bool wd = (mu == 3) && (c.x[3] == 0);
                {
                    Mat3<R> U = GaugeFmt<GP>::load(S.Ulo, q, mu, ti.i, Vh);
#pragma unroll
                    for (int l = 0; l < NB; ++l) {
                        if (mode[l] != LM_ACTIVE) continue;
                        Vec3<RS> rr = SpinorFmt<SP>::load_cg(rhs_ptr(a, rid[l], F_R), nq, lu, Vh);
                        Vec3<RS> pp = SpinorFmt<SP>::load_cg(rhs_ptr(a, rid[l], F_P), nq, lu, Vh);
                        Vec3<R> pn = vcvt<R>(SpinorFmt<SP>::quantize(vaxpy(rr, beta[l], pp)));
                        vacc(acc[l], mul_mv(U, pn), eta_neg != wu);
                    }
                }
                {
                    Mat3<R> Ud = GaugeFmt<GP>::load(S.Ulo, nq, mu, ld, Vh);
#pragma unroll
                    for (int l = 0; l < NB; ++l) {
                        if (mode[l] != LM_ACTIVE) continue;
                        Vec3<RS> rr = SpinorFmt<SP>::load_cg(rhs_ptr(a, rid[l], F_R), nq, ld, Vh);
                        Vec3<RS> pp = SpinorFmt<SP>::load_cg(rhs_ptr(a, rid[l], F_P), nq, ld, Vh);
                        Vec3<R> pn = vcvt<R>(SpinorFmt<SP>::quantize(vaxpy(rr, beta[l], pp)));
                        vacc(acc[l], mul_adj_mv(Ud, pn), !(eta_neg != wd));
                    }
                }
            }
#pragma unroll
            for (int l = 0; l < NB; ++l) {
                if (mode[l] != LM_ACTIVE) continue;
                Vec3<R> o;
#pragma unroll
                for (int k = 0; k < 3; ++k) o.c[k] = {R(0.5) * acc[l].c[k].re, R(0.5) * acc[l].c[k].im};
                SpinorFmt<SP>::store(rhs_ptr(a, rid[l], F_T), q, ti.i, Vh, vcvt<RS>(o));
            }
        }
        if (anyR) {
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (mode[l] == LM_RU) ru_hop1_site<XP>(a, S, c, q, ti.i, rid[l]);
        }
    }
}

// ---------------------------------------------------------------------------
// P2: p = r + beta p, v = m^2 p - K t, <p,v> (normal lanes);
//     x_hi += x_lo, x_lo = 0, r = b - (m^2 x_hi - K thi), |r|^2 (reliable update)
// ---------------------------------------------------------------------------
template <int GP, int SP, int NB>
__device__ void phase_hop2(const CgArgs& a, const CgSys& S, int t, int cur, double* smem,
                           unsigned* s_mask)
{
    typedef typename GaugeFmt<GP>::R R;
    typedef typename SpinorFmt<SP>::R RS;
    constexpr int XP = XFmt<SP>::v;
    const TileInfo ti = decode_tile(S, t);
    const int q = ti.q, nq = 1 - ti.q, Vh = S.g.Vh;
    Coord c;
    if (ti.valid) c = eo_coords(S.g, q, ti.i);
    for (int base = 0; base < S.nrhs; base += NB) {
        const int cnt = min(NB, S.nrhs - base);
        int lanes[NB], rid[NB], mode[NB];
        RS beta[NB];
        bool part[NB];
        double sums[NB];
        gather<NB>(a, S, base, cnt, q, false, cur, lanes, mode, rid);
        bool anyA = false, anyR = false;
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            anyA |= mode[l] == LM_ACTIVE;
            anyR |= mode[l] == LM_RU;
            part[l] = mode[l] == LM_ACTIVE || mode[l] == LM_RU;
            sums[l] = 0.0;
            beta[l] = mode[l] == LM_ACTIVE ? (RS)ld_dbl(&a.lanes[lanes[l]].beta) : RS(0);
        }
        if (!anyA && !anyR) continue;  // uniform across the block
        if (anyA && ti.valid) {
            Vec3<R> acc[NB];
#pragma unroll
            for (int l = 0; l < NB; ++l) vzero(acc[l]);
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
                const bool eta_neg = eta_sign(c, mu) < 0;
                const int lu = lex_up(S.g, c, mu) >> 1, ld = lex_dn(S.g, c, mu) >> 1;
                const bool wu = (mu == 3) && (c.x[3] == S.g.L[3] - 1);
                const bool wd = (mu == 3) && (c.x[3] == 0);
                {
                    Mat3<R> U = GaugeFmt<GP>::load(S.Ulo, q, mu, ti.i, Vh);
#pragma unroll
                    for (int l = 0; l < NB; ++l) {
                        if (mode[l] != LM_ACTIVE) continue;
                        Vec3<R> w = vcvt<R>(SpinorFmt<SP>::load_cg(rhs_ptr(a, rid[l], F_T), nq, lu, Vh));
                        vacc(acc[l], mul_mv(U, w), eta_neg != wu);
                    }
                }
                {
                    Mat3<R> Ud = GaugeFmt<GP>::load(S.Ulo, nq, mu, ld, Vh);
#pragma unroll
                    for (int l = 0; l < NB; ++l) {
                        if (mode[l] != LM_ACTIVE) continue;
                        Vec3<R> w = vcvt<R>(SpinorFmt<SP>::load_cg(rhs_ptr(a, rid[l], F_T), nq, ld, Vh));
                        vacc(acc[l], mul_adj_mv(Ud, w), !(eta_neg != wd));
                    }
                }
            }
            const R m2 = (R)S.m2;
#pragma unroll
            for (int l = 0; l < NB; ++l) {
                if (mode[l] != LM_ACTIVE) continue;
                void* pptr = rhs_ptr(a, rid[l], F_P);
                Vec3<RS> rr = SpinorFmt<SP>::load_cg(rhs_ptr(a, rid[l], F_R), q, ti.i, Vh);
                Vec3<RS> pp = SpinorFmt<SP>::load_cg(pptr, q, ti.i, Vh);
                Vec3<RS> pn = SpinorFmt<SP>::quantize(vaxpy(rr, beta[l], pp));
                SpinorFmt<SP>::store(pptr, q, ti.i, Vh, pn);
                Vec3<R> pr = vcvt<R>(pn), v;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    v.c[k].re = m2 * pr.c[k].re - R(0.5) * acc[l].c[k].re;
                    v.c[k].im = m2 * pr.c[k].im - R(0.5) * acc[l].c[k].im;
                }
                Vec3<RS> vq = SpinorFmt<SP>::quantize(vcvt<RS>(v));
                SpinorFmt<SP>::store(rhs_ptr(a, rid[l], F_V), q, ti.i, Vh, vq);
                sums[l] = vdot_re(pn, vq);
            }
        }
        if (anyR && ti.valid) {
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (mode[l] == LM_RU) sums[l] = ru_hop2_site<SP, XP>(a, S, c, q, ti.i, rid[l]);
        }
        block_sum<NB>(sums, smem);
        unsigned mask = arrive<NB>(a, S, lanes, part, sums, ti.slot, s_mask);
        if (mask && threadIdx.x < 32) {
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (mask & (1u << l)) finish_hop2(a, S, lanes[l], mode[l], cur);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// P3: x += alpha p, r -= alpha v, |r|^2 -> beta, convergence, reliable update
// ---------------------------------------------------------------------------
template <int GP, int SP, int NB>
__device__ void phase_update(const CgArgs& a, const CgSys& S, int t, int cur, double* smem,
                             unsigned* s_mask)
{
    typedef typename SpinorFmt<SP>::R RS;
    constexpr int XP = XFmt<SP>::v;
    typedef typename SpinorFmt<XP>::R RX;
    const TileInfo ti = decode_tile(S, t);
    const int q = ti.q, Vh = S.g.Vh;
    for (int base = 0; base < S.nrhs; base += NB) {
        const int cnt = min(NB, S.nrhs - base);
        int lanes[NB], rid[NB], mode[NB];
        bool part[NB];
        double sums[NB];
        gather<NB>(a, S, base, cnt, q, false, cur, lanes, mode, rid);
        bool any = false;
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            part[l] = mode[l] == LM_ACTIVE;
            any |= part[l];
            sums[l] = 0.0;
            if (part[l] && ti.valid) {
                const double alpha = ld_dbl(&a.lanes[lanes[l]].alpha);
                void* xptr = rhs_ptr(a, rid[l], F_XLO);
                void* rptr = rhs_ptr(a, rid[l], F_R);
                Vec3<RS> pp = SpinorFmt<SP>::load_cg(rhs_ptr(a, rid[l], F_P), q, ti.i, Vh);
                Vec3<RS> vv = SpinorFmt<SP>::load_cg(rhs_ptr(a, rid[l], F_V), q, ti.i, Vh);
                Vec3<RS> rr = SpinorFmt<SP>::load_cg(rptr, q, ti.i, Vh);
                Vec3<RX> xx = SpinorFmt<XP>::load_cg(xptr, q, ti.i, Vh);
                SpinorFmt<XP>::store(xptr, q, ti.i, Vh, vaxpy(xx, (RX)alpha, vcvt<RX>(pp)));
                Vec3<RS> rn = SpinorFmt<SP>::quantize(vaxpy(rr, (RS)(-alpha), vv));
                SpinorFmt<SP>::store(rptr, q, ti.i, Vh, rn);
                sums[l] = vdot_re(rn, rn);
            }
        }
        if (!any) continue;
        block_sum<NB>(sums, smem);
        unsigned mask = arrive<NB>(a, S, lanes, part, sums, ti.slot, s_mask);
        if (mask && threadIdx.x < 32) {
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (mask & (1u << l)) finish_update(a, S, lanes[l], cur);
        }
        __syncthreads();
    }
}

// stage the tile's system descriptor in shared memory
__device__ __forceinline__ void load_sys(const CgArgs& a, int t, CgSys* s_sys)
{
    __syncthreads();
    if (threadIdx.x == 0) *s_sys = a.sys[__ldg(a.tile_sys + t)];
    __syncthreads();
}

template <int GP, int SP, int NB>
__global__ void __launch_bounds__(kTile, (SP == SP_F64 ? 1 : 2)) cg_persistent(CgArgs a)
{
    cgrp::grid_group grid = cgrp::this_grid();
    __shared__ double smem[32 * NB];
    __shared__ unsigned s_mask;
    __shared__ CgSys s_sys;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        load_sys(a, t, &s_sys);
        phase_init<GP, SP, NB>(a, s_sys, t, smem, &s_mask);
    }
    grid.sync();
    for (int it = 0; it < a.maxloop; ++it) {
        if (__ldcg(a.n_active) == 0) break;
        const int cur = it & 1;
        for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
            load_sys(a, t, &s_sys);
            phase_hop1<GP, SP, NB>(a, s_sys, t, cur);
        }
        grid.sync();
        for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
            load_sys(a, t, &s_sys);
            phase_hop2<GP, SP, NB>(a, s_sys, t, cur, smem, &s_mask);
        }
        grid.sync();
        for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
            load_sys(a, t, &s_sys);
            phase_update<GP, SP, NB>(a, s_sys, t, cur, smem, &s_mask);
        }
        grid.sync();
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

typedef void (*CgKernel)(CgArgs);

static CgKernel pick_kernel(int prec, int nb)
{
    if (prec == SFH_PREC_F64) {
        if (nb >= 2) return cg_persistent<GP_F64_18, SP_F64, 2>;
        return cg_persistent<GP_F64_18, SP_F64, 1>;
    }
    if (prec == SFH_PREC_F32) {
        if (nb >= 8) return cg_persistent<GP_F32_12, SP_F32, 8>;
        if (nb >= 4) return cg_persistent<GP_F32_12, SP_F32, 4>;
        if (nb >= 2) return cg_persistent<GP_F32_12, SP_F32, 2>;
        return cg_persistent<GP_F32_12, SP_F32, 1>;
    }
    if (nb >= 8) return cg_persistent<GP_F16_12, SP_F16, 8>;
    if (nb >= 4) return cg_persistent<GP_F16_12, SP_F16, 4>;
    if (nb >= 2) return cg_persistent<GP_F16_12, SP_F16, 2>;
    return cg_persistent<GP_F16_12, SP_F16, 1>;
}

static size_t spinor_bytes(int sp, int Vh)
{
    size_t per = sp == SP_F64 ? 48 : (sp == SP_F32 ? 24 : 16);
    return per * 2 * (size_t)Vh;
}

struct SolverSystemHost {
    Geom g;
    double mass;
    int nrhs;
    const void* U64;
    const void* Ulo;
};

// Device workspace for one batch solve.  Owns the per-RHS vectors.
struct CgWorkspace {
    int prec = 0, both = 0, nb = 0;
    int nsys = 0, nlanes = 0, ntiles = 0;
    std::vector<CgSys> sys;
    std::vector<CgRhs> rhs;  // flattened (system, rhs)
    std::vector<int> rhs0;   // first rhs index of each system
    std::vector<CgLane> lanes_h;
    CgSys* d_sys = nullptr;
    CgRhs* d_rhs = nullptr;
    CgLane* d_lanes = nullptr;
    int* d_tile_sys = nullptr;
    double* d_partial = nullptr;
    int* d_active = nullptr;
    std::vector<void*> allocs;
    size_t bytes = 0;

    ~CgWorkspace() { release(); }
    void release()
    {
        for (void* p : allocs) cudaFree(p);
        allocs.clear();
        d_sys = nullptr; d_rhs = nullptr; d_lanes = nullptr;
        d_tile_sys = nullptr; d_partial = nullptr; d_active = nullptr;
    }
    cudaError_t alloc(void** p, size_t n)
    {
        cudaError_t e = cudaMalloc(p, n);
        if (e == cudaSuccess) { allocs.push_back(*p); bytes += n; }
        return e;
    }
};

static cudaError_t workspace_build(CgWorkspace& w, const std::vector<SolverSystemHost>& systems,
                                   int prec, int both)
{
    w.release();
    w.prec = prec;
    w.both = both;
    w.nsys = (int)systems.size();
    w.sys.clear(); w.rhs.clear(); w.rhs0.clear(); w.lanes_h.clear();
    const int sp = prec == SFH_PREC_F64 ? SP_F64 : (prec == SFH_PREC_F32 ? SP_F32 : SP_F16);
    int tile = 0, lane = 0, poff = 0;
    std::vector<int> tile_sys;
    for (int k = 0; k < w.nsys; ++k) {
        const SolverSystemHost& h = systems[k];
        CgSys S;
        S.g = h.g;
        S.m2 = h.mass * h.mass;
        S.U64 = h.U64;
        S.Ulo = prec == SFH_PREC_F64 ? h.U64 : h.Ulo;
        S.lane0 = lane;
        S.nrhs = h.nrhs;
        S.both = both;
        S.tile0 = tile;
        S.ntq = (h.g.Vh + kTile - 1) / kTile;
        for (int q = 0; q < 2; ++q)
            for (int j = 0; j < S.ntq; ++j) tile_sys.push_back(k);
        tile += 2 * S.ntq;
        w.rhs0.push_back((int)w.rhs.size());
        for (int j = 0; j < h.nrhs; ++j) {
            CgRhs R;
            void* ptrs[8] = {};
            size_t sz64 = spinor_bytes(SP_F64, h.g.Vh), szlo = spinor_bytes(sp, h.g.Vh);
            size_t szx = spinor_bytes(prec == SFH_PREC_F64 ? SP_F64 : SP_F32, h.g.Vh);
            cudaError_t e;
            if ((e = w.alloc(&ptrs[0], sz64)) != cudaSuccess) return e;  // b
            if ((e = w.alloc(&ptrs[1], sz64)) != cudaSuccess) return e;  // xhi
            if (prec != SFH_PREC_F64) {
                if ((e = w.alloc(&ptrs[2], sz64)) != cudaSuccess) return e;  // thi
            }
            for (int z = 3; z < 7; ++z)
                if ((e = w.alloc(&ptrs[z], szlo)) != cudaSuccess) return e;  // r p v t
            if (prec != SFH_PREC_F64) {
                if ((e = w.alloc(&ptrs[7], szx)) != cudaSuccess) return e;  // xlo
            } else {
                ptrs[7] = ptrs[1];
            }
            R.b = ptrs[0]; R.xhi = ptrs[1]; R.thi = ptrs[2]; R.r = ptrs[3];
            R.p = ptrs[4]; R.v = ptrs[5]; R.t = ptrs[6]; R.xlo = ptrs[7];
            int rid = (int)w.rhs.size();
            w.rhs.push_back(R);
            int nlp = both ? 1 : 2;
            for (int lp = 0; lp < nlp; ++lp) {
                CgLane L;
                std::memset(&L, 0, sizeof(L));
                L.sys = k;
                L.rhs = rid;
                L.parity = both ? 2 : lp;
                L.poff = poff;  // slots indexed by the tile's local index (both parities)
                poff += 2 * S.ntq;
                L.mode[0] = L.mode[1] = LM_ACTIVE;
                w.lanes_h.push_back(L);
                ++lane;
            }
        }
        w.sys.push_back(S);
    }
    w.nlanes = lane;
    w.ntiles = tile;
    cudaError_t e;
    if ((e = w.alloc((void**)&w.d_sys, sizeof(CgSys) * w.nsys)) != cudaSuccess) return e;
    if ((e = w.alloc((void**)&w.d_rhs, sizeof(CgRhs) * std::max<size_t>(1, w.rhs.size()))) != cudaSuccess) return e;
    if ((e = w.alloc((void**)&w.d_lanes, sizeof(CgLane) * std::max(1, w.nlanes))) != cudaSuccess) return e;
    if ((e = w.alloc((void**)&w.d_tile_sys, sizeof(int) * std::max(1, w.ntiles))) != cudaSuccess) return e;
    if ((e = w.alloc((void**)&w.d_partial, sizeof(double) * std::max(1, poff))) != cudaSuccess) return e;
    if ((e = w.alloc((void**)&w.d_active, sizeof(int))) != cudaSuccess) return e;
    if ((e = cudaMemcpy(w.d_sys, w.sys.data(), sizeof(CgSys) * w.nsys, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if (!w.rhs.empty())
        if ((e = cudaMemcpy(w.d_rhs, w.rhs.data(), sizeof(CgRhs) * w.rhs.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if ((e = cudaMemcpy(w.d_tile_sys, tile_sys.data(), sizeof(int) * tile_sys.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    return cudaSuccess;
}

static int default_nb(int prec, int max_nrhs)
{
    int cap = prec == SFH_PREC_F64 ? 2 : 8;
    int nb = 1;
    while (nb < max_nrhs && nb < cap) nb *= 2;
    return nb;
}

// Launch the persistent solver on a built workspace.  Returns a cudaError.
static cudaError_t workspace_solve(CgWorkspace& w, double tol, int maxit, double delta, int nb,
                                   cudaStream_t stream, int num_sms)
{
    int max_nrhs = 1;
    for (const CgSys& S : w.sys) max_nrhs = std::max(max_nrhs, S.nrhs);
    if (nb <= 0) nb = default_nb(w.prec, max_nrhs);
    w.nb = nb;
    for (CgLane& L : w.lanes_h) {
        L.mode[0] = L.mode[1] = LM_ACTIVE;
        L.ticket = 0;
        L.iters = 0;
        L.nru = 0;
        L.status = SFH_OK;
    }
    cudaError_t e;
    if ((e = cudaMemcpyAsync(w.d_lanes, w.lanes_h.data(), sizeof(CgLane) * w.nlanes,
                             cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return e;
    int nact = w.nlanes;
    if ((e = cudaMemcpyAsync(w.d_active, &nact, sizeof(int), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return e;
    CgArgs a;
    a.nsys = w.nsys;
    a.nlanes = w.nlanes;
    a.ntiles = w.ntiles;
    a.sys = w.d_sys;
    a.rhs = w.d_rhs;
    a.lanes = w.d_lanes;
    a.tile_sys = w.d_tile_sys;
    a.partial = w.d_partial;
    a.n_active = w.d_active;
    a.tol2 = tol * tol;
    a.delta = delta;
    a.maxit = maxit;
    a.mixed = w.prec != SFH_PREC_F64;
    a.maxloop = a.mixed ? 2 * maxit + 64 : maxit + 1;
    CgKernel k = pick_kernel(w.prec, nb);
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kTile, 0)) != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorLaunchOutOfResources;
    int grid = std::min(per_sm * num_sms, w.ntiles);
    void* args[] = {&a};
    e = cudaLaunchCooperativeKernel((const void*)k, dim3(grid), dim3(kTile), args, 0, stream);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(w.lanes_h.data(), w.d_lanes, sizeof(CgLane) * w.nlanes, cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    for (CgLane& L : w.lanes_h)
        if (L.mode[0] == LM_ACTIVE || L.mode[0] == LM_RU) {
            L.status = SFH_ERR_NOCONV;
            L.mode[0] = L.mode[1] = LM_FAILED;
        }
    return cudaSuccess;
}

}  // namespace sfh

// ===========================================================================
// batch object (C ABI)
// ===========================================================================
struct sfh_batch {
    int device = 0, num_sms = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int prec = 0, flags = 0, nb = 0;
    std::vector<sfh_system_desc> desc;
    std::vector<sfh::Geom> geoms;
    std::vector<void*> U64, U32, U16;
    std::vector<bool> lowp_valid;
    void* stage = nullptr;   // device staging (largest 72V doubles)
    size_t stage_bytes = 0;
    void* scratch = nullptr; // FP64 spinor scratch for residual checks (3 fields)
    int* derr = nullptr;     // device error flags
    sfh::CgWorkspace ws;
    bool ws_ready = false;
    std::string last_error;
};

namespace sfh {
Geom make_geom(const int dims[4]);
bool dims_ok(const int dims[4]);
}

static int batch_err(sfh_batch* b, int code, const std::string& m)
{
    if (b) b->last_error = m;
    return code;
}

static int batch_cuda(sfh_batch* b, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return SFH_OK;
    return batch_err(b, e == cudaErrorMemoryAllocation ? SFH_ERR_NOMEM : SFH_ERR_CUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
}

extern "C" int sfh_batch_create(int device, int nsys, const sfh_system_desc* systems, int precision,
                                int flags, sfh_batch** out)
{
    if (!out || nsys <= 0 || !systems) return SFH_ERR_INVALID;
    if (precision < SFH_PREC_F64 || precision > SFH_PREC_F16) return SFH_ERR_INVALID;
    if ((flags & SFH_BATCH_FULL_LATTICE) && precision != SFH_PREC_F64) return SFH_ERR_INVALID;
    for (int k = 0; k < nsys; ++k)
        if (!sfh::dims_ok(systems[k].dims) || systems[k].nrhs <= 0 || systems[k].nrhs > 64)
            return SFH_ERR_INVALID;
    *out = nullptr;
    sfh_batch* b = new sfh_batch();
    b->device = device;
    b->prec = precision;
    b->flags = flags;
    b->desc.assign(systems, systems + nsys);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete b; return SFH_ERR_CUDA; }
    b->own_stream = true;
    size_t maxV = 0;
    for (int k = 0; k < nsys; ++k) {
        sfh::Geom g = sfh::make_geom(systems[k].dims);
        b->geoms.push_back(g);
        maxV = std::max(maxV, (size_t)g.V);
        void *u64 = nullptr, *u32 = nullptr, *u16 = nullptr;
        size_t n64 = (size_t)g.V * 4 * 9 * 16;
        e = cudaMalloc(&u64, n64);
        if (e == cudaSuccess && precision == SFH_PREC_F32) e = cudaMalloc(&u32, (size_t)g.V * 4 * 3 * 16);
        if (e == cudaSuccess && precision == SFH_PREC_F16) e = cudaMalloc(&u16, (size_t)g.V * 4 * 3 * 8);
        b->U64.push_back(u64);
        b->U32.push_back(u32);
        b->U16.push_back(u16);
        b->lowp_valid.push_back(false);
        if (e != cudaSuccess) { sfh_batch_destroy(b); return SFH_ERR_NOMEM; }
    }
    b->stage_bytes = maxV * 72 * sizeof(double);
    e = cudaMalloc(&b->stage, b->stage_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&b->scratch, maxV * 6 * sizeof(double) * 3);
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->derr, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->derr, 0, sizeof(int));
    if (e != cudaSuccess) { sfh_batch_destroy(b); return SFH_ERR_NOMEM; }
    std::vector<sfh::SolverSystemHost> hs;
    for (int k = 0; k < nsys; ++k) {
        sfh::SolverSystemHost h;
        h.g = b->geoms[k];
        h.mass = systems[k].mass;
        h.nrhs = systems[k].nrhs;
        h.U64 = b->U64[k];
        h.Ulo = precision == SFH_PREC_F32 ? b->U32[k] : (precision == SFH_PREC_F16 ? b->U16[k] : b->U64[k]);
        hs.push_back(h);
    }
    e = sfh::workspace_build(b->ws, hs, precision, (flags & SFH_BATCH_FULL_LATTICE) ? 1 : 0);
    if (e != cudaSuccess) { sfh_batch_destroy(b); return SFH_ERR_NOMEM; }
    b->ws_ready = true;
    *out = b;
    return SFH_OK;
}

extern "C" int sfh_batch_destroy(sfh_batch* b)
{
    if (!b) return SFH_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    b->ws.release();
    for (void* p : b->U64) if (p) cudaFree(p);
    for (void* p : b->U32) if (p) cudaFree(p);
    for (void* p : b->U16) if (p) cudaFree(p);
    if (b->stage) cudaFree(b->stage);
    if (b->scratch) cudaFree(b->scratch);
    if (b->derr) cudaFree(b->derr);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return SFH_OK;
}

extern "C" const char* sfh_batch_last_error(const sfh_batch* b)
{
    return b ? b->last_error.c_str() : "null batch";
}

extern "C" int sfh_batch_set_stream(sfh_batch* b, void* s)
{
    if (!b) return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    if (b->own_stream && b->stream) {
        cudaStreamSynchronize(b->stream);
        cudaStreamDestroy(b->stream);
    }
    b->stream = (cudaStream_t)s;
    b->own_stream = false;
    return SFH_OK;
}

extern "C" void* sfh_batch_get_stream(sfh_batch* b) { return b ? (void*)b->stream : nullptr; }

extern "C" int sfh_batch_set_rhs_block(sfh_batch* b, int width)
{
    if (!b || width < 0 || width > 8) return SFH_ERR_INVALID;
    b->nb = width;
    return SFH_OK;
}

extern "C" int sfh_batch_set_gauge(sfh_batch* b, int k, const double* links)
{
    if (!b || !links || k < 0 || k >= (int)b->desc.size()) return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    const sfh::Geom& g = b->geoms[k];
    size_t n = (size_t)g.V * 72 * sizeof(double);
    int st = batch_cuda(b, cudaMemcpyAsync(b->stage, links, n, cudaMemcpyHostToDevice, b->stream), "gauge upload");
    if (st) return st;
    sfh::launch_links_aos_to_eo(g, (const double*)b->stage, b->U64[k], b->stream);
    if (b->prec != SFH_PREC_F64)
        sfh::launch_make_lowp_gauge(g, b->U64[k], b->U32[k], b->U16[k], b->stream);
    return batch_cuda(b, cudaStreamSynchronize(b->stream), "gauge convert");
}

extern "C" int sfh_batch_set_rhs(sfh_batch* b, int k, int j, const double* phi)
{
    if (!b || !phi || k < 0 || k >= (int)b->desc.size() || j < 0 || j >= b->desc[k].nrhs)
        return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    const sfh::Geom& g = b->geoms[k];
    size_t n = (size_t)g.V * 6 * sizeof(double);
    int st = batch_cuda(b, cudaMemcpyAsync(b->stage, phi, n, cudaMemcpyHostToDevice, b->stream), "rhs upload");
    if (st) return st;
    sfh::launch_spinor_aos_to_eo(g, (const double*)b->stage, b->ws.rhs[b->ws.rhs0[k] + j].b, b->stream);
    return batch_cuda(b, cudaStreamSynchronize(b->stream), "rhs convert");
}

extern "C" int sfh_batch_solve(sfh_batch* b, double tol, int maxit)
{
    if (!b || !(tol > 0.0) || maxit <= 0) return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    int st = batch_cuda(b, sfh::workspace_solve(b->ws, tol, maxit, 0.1, b->nb, b->stream, b->num_sms),
                        "batched CG");
    if (st) return st;
    for (const sfh::CgLane& L : b->ws.lanes_h)
        if (L.status != SFH_OK) return L.status;
    return SFH_OK;
}

extern "C" int sfh_batch_get_solution(sfh_batch* b, int k, int j, double* X)
{
    if (!b || !X || k < 0 || k >= (int)b->desc.size() || j < 0 || j >= b->desc[k].nrhs)
        return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    const sfh::Geom& g = b->geoms[k];
    sfh::launch_spinor_eo_to_aos(g, b->ws.rhs[b->ws.rhs0[k] + j].xhi, (double*)b->stage, b->stream);
    int st = batch_cuda(b, cudaMemcpyAsync(X, b->stage, (size_t)g.V * 6 * sizeof(double),
                                           cudaMemcpyDeviceToHost, b->stream), "solution download");
    if (st) return st;
    return batch_cuda(b, cudaStreamSynchronize(b->stream), "solution download");
}

extern "C" int sfh_batch_get_info(sfh_batch* b, int k, int j, sfh_cg_info* info)
{
    if (!b || !info || k < 0 || k >= (int)b->desc.size() || j < 0 || j >= b->desc[k].nrhs)
        return SFH_ERR_INVALID;
    int rid = b->ws.rhs0[k] + j;
    std::memset(info, 0, sizeof(*info));
    double rr = 0.0, bb = 0.0;
    for (const sfh::CgLane& L : b->ws.lanes_h) {
        if (L.rhs != rid) continue;
        if (L.status != SFH_OK && info->status == SFH_OK) info->status = L.status;
        info->iters = std::max(info->iters, L.iters);
        if (L.parity < 2) info->iters_parity[L.parity] = L.iters;
        else info->iters_parity[0] = info->iters_parity[1] = L.iters;
        info->reliable_updates += L.nru;
        rr += L.rr;
        bb += L.bb;
    }
    info->rsq_rel = bb > 0 ? rr / bb : 0.0;
    info->true_resid = -1.0;
    return SFH_OK;
}

extern "C" int sfh_batch_true_residual(sfh_batch* b, int k, int j, double* rel)
{
    if (!b || !rel || k < 0 || k >= (int)b->desc.size() || j < 0 || j >= b->desc[k].nrhs)
        return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    const sfh::Geom& g = b->geoms[k];
    const sfh::CgRhs& R = b->ws.rhs[b->ws.rhs0[k] + j];
    double m = b->desc[k].mass;
    char* s = (char*)b->scratch;
    size_t fs = (size_t)g.V * 6 * sizeof(double);
    void *t = s, *mx = s + fs;
    // t = K x ; mx = m^2 x - K t  (both parities)
    sfh::launch_hop(g, sfh::GP_F64_18, b->U64[k], sfh::SP_F64, R.xhi, sfh::SP_F64, t, nullptr, 0.0, 1.0, 0, 2, b->stream);
    sfh::launch_hop(g, sfh::GP_F64_18, b->U64[k], sfh::SP_F64, t, sfh::SP_F64, mx, R.xhi, m * m, -1.0, 0, 2, b->stream);
    std::vector<double> hb((size_t)g.V * 6), hm((size_t)g.V * 6);
    int st = batch_cuda(b, cudaMemcpyAsync(hb.data(), R.b, fs, cudaMemcpyDeviceToHost, b->stream), "residual");
    if (!st) st = batch_cuda(b, cudaMemcpyAsync(hm.data(), mx, fs, cudaMemcpyDeviceToHost, b->stream), "residual");
    if (!st) st = batch_cuda(b, cudaStreamSynchronize(b->stream), "residual");
    if (st) return st;
    double num = 0, den = 0;
    for (size_t i = 0; i < hb.size(); ++i) {
        double d = hb[i] - hm[i];
        num += d * d;
        den += hb[i] * hb[i];
    }
    *rel = den > 0 ? std::sqrt(num / den) : 0.0;
    return SFH_OK;
}

// ===========================================================================
// single-context solve: a batch of one over the context's own gauge field
// ===========================================================================
namespace sfh {
int ctx_cg_solve(sfh_ctx* c, const double* phi, double* X, double tol, int maxit, int prec,
                 sfh_cg_info* info);
}

int sfh::ctx_cg_solve(sfh_ctx* c, const double* phi, double* X, double tol, int maxit, int prec,
                      sfh_cg_info* info)
{
    if (prec != SFH_PREC_F64 && !c->lowp_valid) {
        launch_make_lowp_gauge(c->g, c->U64, c->U32, c->U16, c->stream);
        c->lowp_valid = true;
    }
    CgWorkspace w;
    SolverSystemHost h;
    h.g = c->g;
    h.mass = c->mass;
    h.nrhs = 1;
    h.U64 = c->U64;
    h.Ulo = prec == SFH_PREC_F32 ? c->U32 : (prec == SFH_PREC_F16 ? c->U16 : c->U64);
    std::vector<SolverSystemHost> hs(1, h);
    cudaError_t e = workspace_build(w, hs, prec, prec == SFH_PREC_F64 ? 1 : 0);
    if (e != cudaSuccess) return cuda_check(c, e, "cg workspace");
    size_t fs = (size_t)c->g.V * 6 * sizeof(double);
    e = cudaMemcpyAsync(c->stage, phi, fs, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "cg upload");
    launch_spinor_aos_to_eo(c->g, (const double*)c->stage, w.rhs[0].b, c->stream);
    e = workspace_solve(w, tol, maxit, 0.1, 0, c->stream, c->num_sms);
    if (e != cudaSuccess) return cuda_check(c, e, "cg solve");
    launch_spinor_eo_to_aos(c->g, w.rhs[0].xhi, (double*)c->stage, c->stream);
    e = cudaMemcpyAsync(X, c->stage, fs, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "cg download");
    int status = SFH_OK;
    sfh_cg_info inf;
    std::memset(&inf, 0, sizeof(inf));
    double rr = 0, bb = 0;
    for (const CgLane& L : w.lanes_h) {
        if (L.status != SFH_OK && status == SFH_OK) status = L.status;
        inf.iters = std::max(inf.iters, L.iters);
        if (L.parity < 2) inf.iters_parity[L.parity] = L.iters;
        else inf.iters_parity[0] = inf.iters_parity[1] = L.iters;
        inf.reliable_updates += L.nru;
        rr += L.rr;
        bb += L.bb;
    }
    inf.status = status;
    inf.rsq_rel = bb > 0 ? rr / bb : 0.0;
    inf.true_resid = -1.0;
    if (info) *info = inf;
    if (status != SFH_OK)
        return set_error(c, status, status == SFH_ERR_NOCONV ? "CG Solver failed to converge"
                                                             : "CG breakdown");
    return SFH_OK;
}

extern "C" int sfh_batch_random_gauge(sfh_batch* b, int k, double eps, unsigned long long seed)
{
    if (!b || k < 0 || k >= (int)b->desc.size()) return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    const sfh::Geom& g = b->geoms[k];
    int st = batch_cuda(b, sfh::launch_random_gauge(g, eps, seed, b->U64[k], b->derr, b->stream), "random gauge");
    if (st) return st;
    if (b->prec != SFH_PREC_F64) sfh::launch_make_lowp_gauge(g, b->U64[k], b->U32[k], b->U16[k], b->stream);
    int h = 0;
    st = batch_cuda(b, cudaMemcpyAsync(&h, b->derr, sizeof(int), cudaMemcpyDeviceToHost, b->stream), "random gauge");
    if (!st) st = batch_cuda(b, cudaStreamSynchronize(b->stream), "random gauge");
    if (st) return st;
    if (h) return batch_err(b, SFH_ERR_DOMAIN, "random gauge: exp(iQ) domain error");
    return SFH_OK;
}

extern "C" int sfh_batch_random_rhs(sfh_batch* b, int k, int j, unsigned long long seed, double sigma)
{
    if (!b || k < 0 || k >= (int)b->desc.size() || j < 0 || j >= b->desc[k].nrhs) return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    int st = batch_cuda(b, sfh::launch_random_spinor(b->geoms[k], sigma, seed, b->ws.rhs[b->ws.rhs0[k] + j].b,
                                                     b->stream), "random rhs");
    if (st) return st;
    return batch_cuda(b, cudaStreamSynchronize(b->stream), "random rhs");
}

extern "C" int sfh_batch_get_gauge(sfh_batch* b, int k, double* links)
{
    if (!b || !links || k < 0 || k >= (int)b->desc.size()) return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    const sfh::Geom& g = b->geoms[k];
    sfh::launch_links_eo_to_aos(g, b->U64[k], (double*)b->stage, b->stream);
    int st = batch_cuda(b, cudaMemcpyAsync(links, b->stage, (size_t)g.V * 72 * sizeof(double),
                                           cudaMemcpyDeviceToHost, b->stream), "gauge download");
    if (st) return st;
    return batch_cuda(b, cudaStreamSynchronize(b->stream), "gauge download");
}

extern "C" int sfh_batch_get_rhs(sfh_batch* b, int k, int j, double* phi)
{
    if (!b || !phi || k < 0 || k >= (int)b->desc.size() || j < 0 || j >= b->desc[k].nrhs)
        return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    const sfh::Geom& g = b->geoms[k];
    sfh::launch_spinor_eo_to_aos(g, b->ws.rhs[b->ws.rhs0[k] + j].b, (double*)b->stage, b->stream);
    int st = batch_cuda(b, cudaMemcpyAsync(phi, b->stage, (size_t)g.V * 6 * sizeof(double),
                                           cudaMemcpyDeviceToHost, b->stream), "rhs download");
    if (st) return st;
    return batch_cuda(b, cudaStreamSynchronize(b->stream), "rhs download");
}

// ===========================================================================
// Allocation-free CG entry point.
//
// For callers that cannot call cudaMalloc: code that runs while a stream is
// being captured into a CUDA graph, host runtimes that own all device memory
// through their own pool and forbid outside allocations, and trajectory loops
// that must not allocate after start-up.  The solver's work vectors and
// control data live in the file-scope array below instead of device
// allocations; the caller passes device inputs and outputs.
// ===========================================================================
namespace sfh {
namespace {

constexpr int kNoAllocMaxSites = SFH_NOALLOC_MAX_SITES;
constexpr int kNoAllocMaxTiles = kNoAllocMaxSites / kTile;  // 2 * tiles per parity
constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kOffSys = 0;
constexpr size_t kOffRhs = align_up(kOffSys + sizeof(CgSys));
constexpr size_t kOffLane = align_up(kOffRhs + sizeof(CgRhs));
constexpr size_t kOffActive = align_up(kOffLane + sizeof(CgLane));
constexpr size_t kOffTiles = align_up(kOffActive + sizeof(int));
constexpr size_t kOffPartial = align_up(kOffTiles + sizeof(int) * kNoAllocMaxTiles);
constexpr size_t kOffVec = align_up(kOffPartial + sizeof(double) * kNoAllocMaxTiles);
constexpr size_t kVecBytes = (size_t)kNoAllocMaxSites * 6 * sizeof(double);
constexpr size_t kNoAllocBytes = kOffVec + 4 * kVecBytes;  // r, p, v, t

// 12.6 MB per device; held by every GPU that loads the library, until exit.
static __device__ __align__(256) unsigned char sfh_noalloc_scratch[kNoAllocBytes];

// Writes the solver's control data into the scratch array (zeroes the
// tickets and partials left by the previous call).
__global__ void noalloc_setup(CgSys S, CgRhs R, unsigned char* base)
{
    CgSys* sys = reinterpret_cast<CgSys*>(base + kOffSys);
    CgRhs* rhs = reinterpret_cast<CgRhs*>(base + kOffRhs);
    CgLane* lane = reinterpret_cast<CgLane*>(base + kOffLane);
    int* active = reinterpret_cast<int*>(base + kOffActive);
    int* tiles = reinterpret_cast<int*>(base + kOffTiles);
    double* partial = reinterpret_cast<double*>(base + kOffPartial);
    for (int k = threadIdx.x; k < 2 * S.ntq; k += blockDim.x) {
        tiles[k] = 0;
        partial[k] = 0.0;
    }
    if (threadIdx.x == 0) {
        *sys = S;
        *rhs = R;
        CgLane L;
        memset(&L, 0, sizeof(L));
        L.sys = 0;
        L.rhs = 0;
        L.parity = 2;
        L.poff = 0;
        L.mode[0] = L.mode[1] = LM_ACTIVE;
        *lane = L;
        *active = 1;
    }
}

struct NoAllocDevice {
    bool ready = false;
    unsigned char* addr = nullptr;
};
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[64];

// Device address of the scratch array on the current device.  The first call
// on a device looks it up with cudaGetSymbolAddress (this can load the
// library's device code on that device).
int noalloc_scratch(unsigned char** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SFH_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (!d.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, sfh_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) return SFH_ERR_CUDA;
        d.addr = static_cast<unsigned char*>(p);
        d.ready = true;
    }
    *out = d.addr;
    return SFH_OK;
}

}  // namespace

extern "C" int sfh_cg_solve_noalloc(const int dims[4], double mass, const void* links_eo,
                                    const void* phi_eo, void* x_eo, double tol, int maxit,
                                    void* cuda_stream, sfh_cg_info* info)
{
    if (!dims || !links_eo || !phi_eo || !x_eo || !(tol > 0.0) || maxit <= 0) return SFH_ERR_INVALID;
    if (!sfh::dims_ok(dims)) return SFH_ERR_INVALID;
    const long V = (long)dims[0] * dims[1] * dims[2] * dims[3];
    if (V > kNoAllocMaxSites) return SFH_ERR_INVALID;  // lattice larger than the scratch array
    unsigned char* base = nullptr;
    int st = noalloc_scratch(&base);
    if (st) return st;
    cudaStream_t stream = (cudaStream_t)cuda_stream;
    int dev = 0, num_sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return SFH_ERR_CUDA;
    if (cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return SFH_ERR_CUDA;

    CgSys S;
    S.g = make_geom(dims);
    S.m2 = mass * mass;
    S.U64 = links_eo;
    S.Ulo = links_eo;
    S.lane0 = 0;
    S.nrhs = 1;
    S.both = 1;
    S.tile0 = 0;
    S.ntq = (S.g.Vh + kTile - 1) / kTile;
    CgRhs R;
    R.b = const_cast<void*>(phi_eo);
    R.xhi = x_eo;
    R.thi = nullptr;
    R.r = base + kOffVec;
    R.p = base + kOffVec + kVecBytes;
    R.v = base + kOffVec + 2 * kVecBytes;
    R.t = base + kOffVec + 3 * kVecBytes;
    R.xlo = x_eo;
    noalloc_setup<<<1, 256, 0, stream>>>(S, R, base);
    if (cudaGetLastError() != cudaSuccess) return SFH_ERR_CUDA;

    CgArgs a;
    a.nsys = 1;
    a.nlanes = 1;
    a.ntiles = 2 * S.ntq;
    a.sys = reinterpret_cast<const CgSys*>(base + kOffSys);
    a.rhs = reinterpret_cast<const CgRhs*>(base + kOffRhs);
    a.lanes = reinterpret_cast<CgLane*>(base + kOffLane);
    a.tile_sys = reinterpret_cast<const int*>(base + kOffTiles);
    a.partial = reinterpret_cast<double*>(base + kOffPartial);
    a.n_active = reinterpret_cast<int*>(base + kOffActive);
    a.tol2 = tol * tol;
    a.delta = 0.1;
    a.maxit = maxit;
    a.mixed = 0;
    a.maxloop = maxit + 1;
    CgKernel k = cg_persistent<GP_F64_18, SP_F64, 1>;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kTile, 0) != cudaSuccess || per_sm < 1)
        return SFH_ERR_CUDA;
    int grid = std::min(per_sm * num_sms, a.ntiles);
    void* args[] = {&a};
    if (cudaLaunchCooperativeKernel((const void*)k, dim3(grid), dim3(kTile), args, 0, stream) != cudaSuccess)
        return SFH_ERR_CUDA;
    CgLane L;
    if (cudaMemcpyAsync(&L, a.lanes, sizeof(CgLane), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        return SFH_ERR_CUDA;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return SFH_ERR_CUDA;
    int status = L.status;
    if (L.mode[0] == LM_ACTIVE || L.mode[0] == LM_RU) status = SFH_ERR_NOCONV;
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->status = status;
        info->iters = L.iters;
        info->iters_parity[0] = info->iters_parity[1] = L.iters;
        info->rsq_rel = L.bb > 0 ? L.rr / L.bb : 0.0;
        info->true_resid = -1.0;
    }
    return status;
}

}  // namespace sfh

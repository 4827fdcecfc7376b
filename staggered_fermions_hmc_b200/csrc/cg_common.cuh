// cg_common.cuh — data structures and device helpers shared by the CG solvers
// (the per-phase batched solver in cg.cu and the single-launch solver in
// cg_noalloc.cu).
#pragma once

#include <cooperative_groups.h>

#include "hop.cuh"
#include "sfh_internal.h"

namespace sfh {

// lane modes; LM_LAST: the update kernel of this iteration still runs for the
// lane, then retires it (DONE)
// LM_RESTART: an active iteration that first restarts the search direction
// (p = r), used after the FP64 residual update of restarting lanes
enum { LM_ACTIVE = 0, LM_RU = 1, LM_DONE = 2, LM_FAILED = 3, LM_LAST = 4, LM_RESTART = 5 };
constexpr int kTile = 256;

struct CgSys {
    Geom g;
    double m2;
    const void* U64;
    const void* Ulo;
    int lane0, nrhs, both, tile0, ntq;
    int rhs0;  // the system's first entry in the RHS table (its RHS are consecutive)
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
    double m2;  // the lane's mass squared (the system's, or its own for RHS at several masses)
    double bb, target, rr, rr_old, pAp, alpha, beta, rmax, rr_next;
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
    int restart;  // restart the Krylov space after every residual update
    int tpi;      // tiles per work item of the iteration kernels
    // lanes due for a reliable update, per iteration parity: [2][1 + nlanes],
    // a count then lane ids (null: the hop kernels do the reliable updates)
    int* ru_list;
    // neighbour staging (schedule 6): shared-memory words of one RHS's staged
    // range per buffer (kTile + the batch's largest Lt), and the device error
    // word a staging wait that gives up sets DEV_ERR_TIMEOUT in (null: unused)
    int nst_words;
    int* err;
    // work-item counters of the hop kernels with a resident grid (schedule
    // 7): [iteration parity][hop1, hop2], zeroed by the update kernel of the
    // same iteration; the item counts of the two hops (null / 0: unused)
    int* qctr;
    int nitems1, nitems2;
};

namespace {

// storage of the low-precision solution x_lo, which sums alpha p between two
// reliable updates and is then added to the FP64 x_hi and cleared: FP32 for
// every mixed precision.  FP16 with a per-site scale for the 16-bit storages
// cut the update kernel's time by 8 % on the uneven batch but its rounding
// cost 6 % more iterations (mean 360 against 341): 401 against 417 solves/s.
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

// Sums of NF arrays of n partial slots (array f at slots + f * stride) by one
// warp in a fixed order (all lanes get them): lane j adds slots j, j + 32,
// j + 64, ... in turn, then the lanes combine by a fixed butterfly.  The
// loads of four rounds are issued before their adds, so that a sum over n
// slots waits about n / 128 memory latencies rather than n / 32 (the slots
// were just written by other blocks and are read from L2); the order of the
// adds is the same either way.
template <int NF>
__device__ __forceinline__ void warp_sum_slots_n(const double* slots, int stride, int n, double (&s)[NF])
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int f = 0; f < NF; ++f) s[f] = 0.0;
    int k = lane;
    for (; k + 96 < n; k += 128) {
        double v[NF][4];
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int u = 0; u < 4; ++u) v[f][u] = __ldcg(slots + (size_t)f * stride + k + 32 * u);
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int u = 0; u < 4; ++u) s[f] += v[f][u];
    }
    for (; k < n; k += 32)
#pragma unroll
        for (int f = 0; f < NF; ++f) s[f] += __ldcg(slots + (size_t)f * stride + k);
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s[f] += __shfl_xor_sync(0xffffffffu, s[f], o);
}

__device__ __forceinline__ double warp_sum_slots(const double* slots, int n)
{
    double s[1];
    warp_sum_slots_n<1>(slots, 0, n, s);
    return s[0];
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
__device__ __forceinline__ void* rhs_ptr(const CgRhs* rhs, int rid, int f)
{
    const unsigned long long* base = reinterpret_cast<const unsigned long long*>(rhs + rid);
    return reinterpret_cast<void*>(__ldg(base + f));
}

__device__ __forceinline__ void* rhs_ptr(const CgArgs& a, int rid, int f) { return rhs_ptr(a.rhs, rid, f); }

}  // namespace
}  // namespace sfh

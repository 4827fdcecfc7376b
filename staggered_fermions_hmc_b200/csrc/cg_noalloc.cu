// cg_noalloc.cu — single-launch CG solver (one cooperative kernel per solve,
// phases separated by grid.sync) and the allocation-free entry point built on
// it.  The kernel runs the reference's FP64 CG (solve_CG_DDdagger,
// Fermions.cpp:553-617) with the three-phase iteration
//   P1  t = K p_new,     p_new = r + beta p computed at the neighbours
//   P2  p = p_new, v = m^2 p - K t, partial <p, v>      -> alpha
//   P3  x += alpha p, r -= alpha v, partial <r, r>       -> beta / convergence
// and deterministic reductions (fixed-order sums of per-tile partials by the
// tile that completes a lane's atomic ticket).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "cg_common.cuh"

namespace cgrp = cooperative_groups;

namespace sfh {
namespace {

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

__device__ __noinline__ void finish_hop2(const CgArgs& a, const CgSys& S, int lane, int cur)
{
    CgLane* L = a.lanes + lane;
    double s = warp_sum_slots(a.partial + L->poff + lane_slot0(S, L->parity), lane_nslots(S));
    if (threadIdx.x != 0) return;
    // s = <p, M p>; Fermions.cpp:573-586
    L->pAp = s;
    double alpha = L->rr / s;
    if (!isfinite(s) || fabs(s) < 1e-30 || !isfinite(alpha)) {
        set_mode_final(L, LM_FAILED, SFH_ERR_BREAKDOWN, a.n_active);
    } else {
        L->alpha = alpha;
        L->mode[cur ^ 1] = LM_ACTIVE;
    }
}

__device__ __noinline__ void finish_update(const CgArgs& a, const CgSys& S, int lane, int cur)
{
    CgLane* L = a.lanes + lane;
    double rn = warp_sum_slots(a.partial + L->poff + lane_slot0(S, L->parity), lane_nslots(S));
    if (threadIdx.x != 0) return;
    const int nxt = cur ^ 1;
    L->iters += 1;
    const double beta = rn / L->rr;  // Fermions.cpp:594-601
    if (!isfinite(rn) || !isfinite(beta)) {
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
// P1: t = K (r + beta p).  Output parity q, inputs on parity 1-q.
// ---------------------------------------------------------------------------
template <int GP, int SP, int NB>
__device__ void phase_hop1(const CgArgs& a, const CgSys& S, int t, int cur)
{
    typedef typename GaugeFmt<GP>::R R;
    typedef typename SpinorFmt<SP>::R RS;
    const TileInfo ti = decode_tile(S, t);
    if (!ti.valid) return;
    const Coord c = eo_coords(S.g, ti.q, ti.i);
    const int q = ti.q, nq = 1 - ti.q, Vh = S.g.Vh;
    for (int base = 0; base < S.nrhs; base += NB) {
        const int cnt = min(NB, S.nrhs - base);
        int lanes[NB], rid[NB], mode[NB];
        RS beta[NB];
        gather<NB>(a, S, base, cnt, q, true, cur, lanes, mode, rid);
        bool anyA = false;
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            anyA |= mode[l] == LM_ACTIVE;
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
    }
}

// ---------------------------------------------------------------------------
// P2: p = r + beta p, v = m^2 p - K t, <p,v>
// ---------------------------------------------------------------------------
template <int GP, int SP, int NB>
__device__ void phase_hop2(const CgArgs& a, const CgSys& S, int t, int cur, double* smem,
                           unsigned* s_mask)
{
    typedef typename GaugeFmt<GP>::R R;
    typedef typename SpinorFmt<SP>::R RS;
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
        bool anyA = false;
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            anyA |= mode[l] == LM_ACTIVE;
            part[l] = mode[l] == LM_ACTIVE;
            sums[l] = 0.0;
            beta[l] = mode[l] == LM_ACTIVE ? (RS)ld_dbl(&a.lanes[lanes[l]].beta) : RS(0);
        }
        if (!anyA) continue;  // uniform across the block
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
        block_sum<NB>(sums, smem);
        unsigned mask = arrive<NB>(a, S, lanes, part, sums, ti.slot, s_mask);
        if (mask && threadIdx.x < 32) {
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (mask & (1u << l)) finish_hop2(a, S, lanes[l], cur);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// P3: x += alpha p, r -= alpha v, |r|^2 -> beta, convergence
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
__global__ void __launch_bounds__(kTile, 1) cg_persistent(CgArgs a)
{
    static_assert(GP == GP_F64_18 && SP == SP_F64, "the single-launch solver runs the FP64 CG only");
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

typedef void (*PersistentKernel)(CgArgs);

}  // namespace
}  // namespace sfh

// ===========================================================================
// Allocation-free CG entry point.
//
// For callers that cannot call cudaMalloc: host runtimes that own all device
// memory through their own pool and forbid outside allocations, and
// trajectory loops that must not allocate after start-up.  FP64 CG only; the
// call copies the lane's status back to the host and waits for the stream,
// and reports no true residual (true_resid = -1: no array is spare for it).
// The solver's work vectors and control data live in the file-scope array
// below instead of device allocations; the caller passes device inputs and
// outputs.
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
    S.rhs0 = 0;
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
    a.ru_list = nullptr;
    a.tol2 = tol * tol;
    a.delta = 0.1;
    a.maxit = maxit;
    a.mixed = 0;
    a.restart = 0;
    a.maxloop = maxit + 1;
    PersistentKernel k = cg_persistent<GP_F64_18, SP_F64, 1>;
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
    if (L.mode[0] == LM_ACTIVE) status = SFH_ERR_NOCONV;
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

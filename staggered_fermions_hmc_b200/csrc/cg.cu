// cg.cu — batched conjugate-gradient solver for D D^dag x = b (three to five
// kernels per iteration, replayed as CUDA-graph chunks, or one persistent
// launch per solve).
//
// Restates solve_CG_DDdagger (Fermions.cpp:553-617) for the GPU.  D D^dag =
// m^2 - K^2 and K couples only even and odd sites, so D D^dag is block
// diagonal in parity: M_pp = m^2 - K_{p,1-p} K_{1-p,p}.
//
// A batch holds "lanes": one lane is the CG of one (system, right-hand side,
// parity block), or of one (system, RHS) over both parities with shared
// scalars (the reference's full-lattice CG).  Systems may differ in lattice
// size and mass.  Iteration k of every lane is three grid-wide kernels:
//
//   hop1    t = K p                                    (other parity)
//   hop2    v = m^2 p - K t, sums <p,v>, <r,v>, |v|^2, |r|^2
//   update  x += alpha p, r -= alpha v, p = r + beta p
//
// The tile that completes a lane's count of hop2 partial sums (atomic ticket)
// adds them in a fixed order and advances the lane in FP64:
// alpha = |r|^2 / <p, M p>, |r - alpha v|^2 = |r|^2 - 2 alpha <r,v> +
// alpha^2 |v|^2 (anchored each iteration on the exact |r|^2, so the
// recurrence does not drift), beta = |r_new|^2 / |r|^2, and the reference's
// convergence test (Fermions.cpp:569).  One reduction point per iteration.
//
// Work is split into tiles of 256 sites of one system and one output parity.
// A work item is a range of tiles and a group of the system's RHS, so a link
// loaded once serves every RHS of the group (RHS blocking).  Schedules (the
// autotuner times them; results never depend on the choice): links read
// directly or staged per work item; the FP64 reliable-update hops inside the
// hop kernels or in two kernels walking a device list of the lanes due for
// one; system-blocked kernels (one tile per block, every RHS of the system,
// the tile's links staged once); the system-blocked work in one
// cooperative launch with a bounded grid barrier; and (FP16) each tile's time
// and z neighbours staged in shared memory by bulk asynchronous copies,
// double-buffered across the item's tiles (tstage.cuh).
//
// Mixed precision (FP32 or FP16+scale vectors with FP32 / FP16 12-real links):
// x is accumulated in FP32 between reliable updates.  When |r| has dropped by
// delta since the last update, or the recurrence meets the target, the lane
// spends its next iteration on an FP64 reliable update: x_hi += x_lo and
// r = b - M x_hi with FP64 links and vectors, keeping p (rebuilt on the
// true residual: p += r_true - r_iter).  Mixed lanes converge only on that
// FP64 true residual.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cg_common.cuh"
#include "tstage.cuh"

namespace sfh {

namespace {

constexpr int kSums = 4;  // <p,v>, <r,v>, |v|^2, |r|^2

// resident 256-thread blocks per SM the hop kernels are compiled for (at most
// 85 registers a thread for three, 64 for four): up to two lanes a block fit
// three blocks, four with FP16 links and vectors (their packed-half products
// hold a link in nine registers; measured 6 % faster on the uneven batch than
// three, despite a few spilled words); wider RHS groups and FP64 take 128
// registers and two
template <int GP, int SP, int NB, bool SUMS, bool RUI = true> struct HopOcc {
    // without the inline FP64 reliable-update hop the kernels need fewer
    // registers: FP16 fits in 48 (five blocks), the FP32-arithmetic ones with
    // 12-real links in 64 (four); 18-real FP32 links keep three.  FP16 in
    // groups of four RHS: the first hop fits in 64 registers (four blocks,
    // no spills), the second, with its sums, in 80 (three)
    static constexpr int v = (NB == 4 && GP == GP_F16_12 && SP == SP_F16 && !RUI) ? (SUMS ? 3 : 4)
                             : (SP == SP_F64 || NB > 2) ? 2
                             : ((GP == GP_F16_12 && SP == SP_F16) ? (RUI ? 4 : 5)
                                                                   : ((RUI || GP == GP_F32_18) ? 3 : 4));
};

// one RHS pass of a tile: the lanes and their scalars
template <int NB>
struct LanePass {
    int lane[NB], mode[NB], rid[NB];
    double alpha[NB], beta[NB], m2[NB];
    bool anyA, anyR;
};

template <int NB>
__device__ __forceinline__ void gather_pass(const CgArgs& a, const CgSys& S, int base, int q, bool hop1,
                                            int cur, bool scalars, LanePass<NB>& P)
{
    const int cnt = min(NB, S.nrhs - base);
    P.anyA = P.anyR = false;
#pragma unroll
    for (int l = 0; l < NB; ++l) {
        P.lane[l] = 0;
        P.mode[l] = LM_DONE;
        P.rid[l] = 0;
        P.alpha[l] = 0.0;
        P.beta[l] = 0.0;
        P.m2[l] = 0.0;
        if (l < cnt) {
            P.lane[l] = lane_of(S, base + l, q, hop1);
            const CgLane* L = a.lanes + P.lane[l];
            P.mode[l] = ld_int(&L->mode[cur]);
            P.rid[l] = S.rhs0 + base + l;  // == L->rhs, without waiting for the lane
            P.m2[l] = __ldg(&L->m2);  // fixed for the solve
            if (scalars && P.mode[l] == LM_ACTIVE) {
                P.alpha[l] = ld_dbl(&L->alpha);
                P.beta[l] = ld_dbl(&L->beta);
            }
            P.anyA |= P.mode[l] == LM_ACTIVE || P.mode[l] == LM_RESTART;
            P.anyR |= P.mode[l] == LM_RU;
        }
    }
}

// stage the tile's system descriptor in shared memory (one tile per block)
__device__ __forceinline__ void stage_sys(const CgArgs& a, int tile, CgSys* s_sys)
{
    if (threadIdx.x == 0) *s_sys = a.sys[__ldg(a.tile_sys + tile)];
    __syncthreads();
}

// A work item of the per-phase kernels: x its first tile, y its first RHS
// (below 64) and its system index above bit kItemSysShift, so that a block
// reaches its system descriptor in one dependent load rather than through
// the tile table, and its vectors' addresses without waiting for its lanes
constexpr int kItemSysShift = 8;
__device__ __forceinline__ int item_rhs(int2 it) { return it.y & ((1 << kItemSysShift) - 1); }

__device__ __forceinline__ void stage_item_sys(const CgArgs& a, int2 it, CgSys* s_sys)
{
    if (threadIdx.x == 0) *s_sys = a.sys[it.y >> kItemSysShift];
    __syncthreads();
}

// the tiles of one work item: tpi consecutive tiles of one parity of a system
struct ItemRange {
    int first, end;  // tile indices [first, end)
    int q;           // output parity
    int slot;        // the item's partial-sum slot of its lanes
};

// work items per parity of a system's lane (their partial-sum slots)
__device__ __forceinline__ int item_groups(const CgArgs& a, const CgSys& S) { return (S.ntq + a.tpi - 1) / a.tpi; }

__device__ __forceinline__ ItemRange item_range(const CgArgs& a, const CgSys& S, int first)
{
    ItemRange r;
    const int local = first - S.tile0;
    r.q = local >= S.ntq ? 1 : 0;
    const int j = local - r.q * S.ntq;
    r.first = first;
    r.end = min(first + a.tpi, S.tile0 + (r.q + 1) * S.ntq);
    r.slot = r.q * item_groups(a, S) + j / a.tpi;
    return r;
}

// neighbour checkerboard indices and hop signs of one output site, computed
// once and shared by every lane of the block
struct Nbr {
    int up[4], dn[4];
    unsigned eta;  // bit mu: eta_mu(x) = -1
    bool wu, wd;   // the forward / backward time hop wraps (anti-periodic sign)
};

__device__ __forceinline__ Nbr neighbours(const Geom& g, const Coord& c)
{
    Nbr n;
    n.eta = 0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        n.up[mu] = lex_up(g, c, mu) >> 1;
        n.dn[mu] = lex_dn(g, c, mu) >> 1;
        if (eta_sign(c, mu) < 0) n.eta |= 1u << mu;
    }
    n.wu = c.x[3] == g.L[3] - 1;
    n.wd = c.x[3] == 0;
    return n;
}

// Link staging: every thread copies the 8 links of its site (4 forward at
// the site, 4 backward at its neighbours) into its own columns of shared
// memory with asynchronous copies, [direction][element][thread], so that all
// of them are in flight at once without holding registers.  FP64 links
// (36 KB per 256 sites and direction pair) are not staged.
template <int GP> struct StageBytes {
    static constexpr size_t v = (GP == GP_F64_18) ? 0 : 8 * GaugeFmt<GP>::K * kTile * sizeof(typename GaugeFmt<GP>::E);
};

template <int N>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(gmem), "n"(N) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

template <int GP>
__device__ __forceinline__ void stage_links(typename GaugeFmt<GP>::E* s, const void* Ulo, const Nbr& n, int q, int i,
                                            int Vh)
{
    typedef GaugeFmt<GP> F;
    typedef typename F::E E;
    const E* U = (const E*)Ulo;
    const int nq = 1 - q, t = threadIdx.x;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu)
#pragma unroll
        for (int k = 0; k < F::K; ++k) {
            cp_async<sizeof(E)>(s + ((2 * mu) * F::K + k) * kTile + t, U + ((size_t)(q * 4 + mu) * F::K + k) * Vh + i);
            cp_async<sizeof(E)>(s + ((2 * mu + 1) * F::K + k) * kTile + t,
                                U + ((size_t)(nq * 4 + mu) * F::K + k) * Vh + n.dn[mu]);
        }
}

template <int GP, bool STG>
__device__ __forceinline__ Mat3<typename GaugeFmt<GP>::R> hop_link(const typename GaugeFmt<GP>::E* s, const void* Ulo,
                                                                   int d, int p, int mu, int i, int Vh)
{
    typedef GaugeFmt<GP> F;
    if constexpr (STG) {
        typename F::E w[F::K];
#pragma unroll
        for (int k = 0; k < F::K; ++k) w[k] = s[(d * F::K + k) * kTile + threadIdx.x];
        return F::unpack(w);
    } else {
        return F::load(Ulo, p, mu, i, Vh);
    }
}

// acc[l] += 1/2 sum_mu eta_mu(x) [bc U_mu(x) in_l(x+mu) - bc U_mu(x-mu)^dag in_l(x-mu)]
// (the hopping term K, Fermions.cpp:218-247) for the lanes with on[l]; each
// link is loaded once for all lanes of the block.  The time-wrap signs apply
// to the input vectors of mu = 3, eta / 2 to the sum of both hops.
// NST (FP16 only): the neighbour vectors of lane l from its staged range at
// sn + l * W where it holds them (tstage.cuh), else from global memory.
template <int GP, int SP, int NB, bool STG, bool COH = false, bool NST = false>
__device__ __forceinline__ void hop_lanes(const void* Ulo, const typename GaugeFmt<GP>::E* sl, const Nbr& n, int q,
                                          int i, int Vh, const void* const (&in)[NB], const bool (&on)[NB],
                                          Vec3<typename GaugeFmt<GP>::R> (&acc)[NB], const uint4* sn = nullptr,
                                          int W = 0, TRange sr = {0, 0}, bool sok = false)
{
    static_assert(!NST || (GP == GP_F16_12 && SP == SP_F16 && !COH), "neighbour staging: FP16 graph kernels");
    typedef typename GaugeFmt<GP>::R R;
    const int nq = 1 - q;
    // FP16 links and vectors: products in packed half2, accumulated in FP32
    // with the scalar factor (hop_half).  Otherwise both hops of a direction
    // accumulate into acc directly, the scalar factor (eta/2, the
    // anti-periodic time sign, the BF16 site scale) going onto the input
    // vector; FP32-12 sums the two hops of a direction first and applies
    // eta/2 once (measured faster there)
    constexpr bool direct = GaugeFmt<GP>::K == 9 || SpinorFmt<SP>::scaled;
    if constexpr (GP == GP_F16_12 && SP == SP_F16) {
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            const float s = ((n.eta >> mu) & 1u) ? -0.5f : 0.5f;
            __half2 U[9];
            hlink_load<STG>(sl, kTile, Ulo, 2 * mu, q, mu, i, Vh, U);
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (on[l]) {
                    const float f = (n.wu && mu == 3) ? -s : s;
                    if constexpr (NST)
                        hop_half_word<false>(
                            acc[l], U, nbr_word(sn + l * W, sr, sok, (const uint4*)in[l] + (size_t)nq * Vh, n.up[mu]),
                            f);
                    else
                        hop_half<false, COH>(acc[l], U, in[l], nq, n.up[mu], Vh, f);
                }
            hlink_load<STG>(sl, kTile, Ulo, 2 * mu + 1, nq, mu, n.dn[mu], Vh, U);
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (on[l]) {
                    const float f = (n.wd && mu == 3) ? s : -s;
                    if constexpr (NST)
                        hop_half_word<true>(
                            acc[l], U, nbr_word(sn + l * W, sr, sok, (const uint4*)in[l] + (size_t)nq * Vh, n.dn[mu]),
                            f);
                    else
                        hop_half<true, COH>(acc[l], U, in[l], nq, n.dn[mu], Vh, f);
                }
        }
        return;
    }
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        const R s = ((n.eta >> mu) & 1u) ? R(-0.5) : R(0.5);
        Vec3<R> w[direct ? 1 : NB];
        {
            const Mat3<R> U = hop_link<GP, STG>(sl, Ulo, 2 * mu, q, mu, i, Vh);
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (on[l]) {
                    if constexpr (direct) {
                        mv_add<false>(acc[l], U, hop_input<SP, R, COH>(in[l], nq, n.up[mu], Vh, n.wu && mu == 3, s));
                    } else {
                        Vec3<R> v = vcvt<R>(SpinorFmt<SP>::template load<COH>(in[l], nq, n.up[mu], Vh));
                        if (mu == 3) v = vneg_if(v, n.wu);
                        mv_add<true>(w[l], U, v);
                    }
                }
        }
        {
            const Mat3<R> U = hop_link<GP, STG>(sl, Ulo, 2 * mu + 1, nq, mu, n.dn[mu], Vh);
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (on[l]) {
                    if constexpr (direct) {
                        mdv_sub(acc[l], U, hop_input<SP, R, COH>(in[l], nq, n.dn[mu], Vh, n.wd && mu == 3, s));
                    } else {
                        Vec3<R> v = vcvt<R>(SpinorFmt<SP>::template load<COH>(in[l], nq, n.dn[mu], Vh));
                        if (mu == 3) v = vneg_if(v, n.wd);
                        mdv_sub(w[l], U, v);
                    }
                }
        }
        if constexpr (!direct) {
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (on[l]) vfma(acc[l], s, w[l]);
        }
    }
}

// ---------------------------------------------------------------------------
// publish the tile's partial sums and take the lanes' tickets
// ---------------------------------------------------------------------------
template <int NB>
__device__ __forceinline__ unsigned arrive_sums(const CgArgs& a, const CgSys& S, const LanePass<NB>& P,
                                                const bool (&part)[NB], const double (&sums)[NB * kSums],
                                                int slot, unsigned expected, unsigned* s_mask)
{
    if (threadIdx.x == 0) {
        unsigned mask = 0;
        const int nslot = 2 * S.ntq;
#pragma unroll
        for (int l = 0; l < NB; ++l)
            if (part[l]) {
                double* dst = a.partial + a.lanes[P.lane[l]].poff + slot;
#pragma unroll
                for (int f = 0; f < kSums; ++f) __stcg(dst + f * nslot, sums[l * kSums + f]);
            }
        __threadfence();
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            if (!part[l]) continue;
            CgLane* L = a.lanes + P.lane[l];
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

// Stop a lane.  mode_now is what the rest of this iteration sees (LM_LAST if
// the update kernel must still run), mode_next what later iterations see.
__device__ __forceinline__ void lane_stop(const CgArgs& a, CgLane* L, int cur, int mode_now, int mode_next,
                                          int status)
{
    L->mode[cur] = mode_now;
    L->mode[cur ^ 1] = mode_next;
    L->status = status;
    atomicSub(a.n_active, 1);
}

// Advance one lane's FP64 scalars from the summed partials of hop2 (warp 0).
// The update of this iteration (x += alpha p, r -= alpha v, p = r + beta p)
// still runs for an ACTIVE lane; the decision applies from the next one.
__device__ __forceinline__ void finish_lane(const CgArgs& a, const CgSys& S, int lane, int mode, int cur)
{
    CgLane* L = a.lanes + lane;
    const int nslot = 2 * S.ntq;
    const int nsq = item_groups(a, S);
    const double* base = a.partial + L->poff + (S.both ? 0 : L->parity * nsq);
    const int n = S.both ? 2 * nsq : nsq;
    double s[kSums];
    warp_sum_slots_n<kSums>(base, nslot, n, s);
    if (threadIdx.x != 0) return;
    const int nxt = cur ^ 1;
    if (mode == LM_ACTIVE || mode == LM_RESTART) {
        const double rr = s[3], pAp = s[0];
        const double alpha = rr / pAp;  // Fermions.cpp:573-586
        if (!isfinite(pAp) || fabs(pAp) < 1e-30 || !isfinite(alpha)) {
            lane_stop(a, L, cur, LM_FAILED, LM_FAILED, SFH_ERR_BREAKDOWN);  // no update
            return;
        }
        const double rr_next = rr - 2.0 * alpha * s[1] + alpha * alpha * s[2];
        const double beta = rr_next / rr;  // Fermions.cpp:594-601
        if (!isfinite(beta)) {
            lane_stop(a, L, cur, LM_FAILED, LM_FAILED, SFH_ERR_BREAKDOWN);
            return;
        }
        L->rr = rr;
        L->pAp = pAp;
        L->alpha = alpha;
        L->beta = beta;
        L->rr_next = rr_next;
        L->iters += 1;
        if (!a.mixed) {
            if (rr_next < L->target)  // Fermions.cpp:569: this iteration's update, then stop
                lane_stop(a, L, cur, LM_LAST, LM_DONE, SFH_OK);
            else if (L->iters >= a.maxit)  // Fermions.cpp:609-614
                lane_stop(a, L, cur, LM_LAST, LM_DONE, SFH_ERR_NOCONV);
            else
                L->mode[nxt] = LM_ACTIVE;
        } else {
            const double r = sqrt(fmax(rr_next, 0.0));
            // update on a drop by delta, at the target, at maxit, or when the
            // iterated residual has grown well past the last true residual
            if (rr_next < L->target || r < a.delta * L->rmax || L->iters >= a.maxit ||
                rr_next > 4.0 * L->rr_old) {
                L->mode[nxt] = LM_RU;
                if (a.ru_list) {  // the next iteration's reliable-update kernels walk this list
                    int* lst = a.ru_list + nxt * (a.nlanes + 1);
                    lst[1 + atomicAdd(lst, 1)] = lane;
                }
            } else {
                L->rmax = fmax(L->rmax, r);
                L->mode[nxt] = LM_ACTIVE;
            }
        }
    } else {  // reliable update: s[3] = |b - M x|^2 in FP64
        const double rt = s[3];
        const double r_iter = L->rr_next;  // the recurrence's |r|^2 that triggered the update
        L->nru += 1;
        L->rr_next = rt;
        if (rt < L->target) {
            lane_stop(a, L, cur, LM_DONE, LM_DONE, SFH_OK);
        } else if (!isfinite(rt)) {
            lane_stop(a, L, cur, LM_FAILED, LM_FAILED, SFH_ERR_BREAKDOWN);
        } else if (L->iters >= a.maxit) {
            lane_stop(a, L, cur, LM_DONE, LM_DONE, SFH_ERR_NOCONV);
        } else {
            // keep the search direction, or restart it (p = r) when the lane
            // restarts after every update, the last stretch made little
            // progress, or the recurrence drifted from the true residual
            // (|r_true|^2 > 1.5 |r_iterated|^2: the search directions lost accuracy)
            const bool restart = a.restart || rt > 0.5 * L->rr_old || rt > 1.5 * r_iter;
            L->rr_old = rt;
            L->rmax = sqrt(rt);
            L->mode[nxt] = restart ? LM_RESTART : LM_ACTIVE;
        }
    }
}

__device__ __noinline__ void finish_init_lane(const CgArgs& a, const CgSys& S, int lane)
{
    CgLane* L = a.lanes + lane;
    const int nslot = 2 * S.ntq;
    const double* base = a.partial + L->poff + 3 * nslot + (S.both ? 0 : L->parity * S.ntq);
    double bb = warp_sum_slots(base, S.both ? 2 * S.ntq : S.ntq);
    if (threadIdx.x != 0) return;
    L->bb = bb;
    L->target = a.tol2 * bb;
    L->rr = bb;
    L->rr_next = bb;
    L->rr_old = bb;
    L->rmax = sqrt(bb);
    L->alpha = 0.0;
    L->beta = 0.0;
    L->iters = 0;
    L->nru = 0;
    L->status = SFH_OK;
    if (bb < 1e-28) {  // Fermions.cpp:562-564: X = 0
        L->mode[0] = L->mode[1] = LM_DONE;
        atomicSub(a.n_active, 1);
    } else {
        L->mode[0] = L->mode[1] = LM_ACTIVE;
    }
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// x = 0, r = p = b (solver precision), |b|^2
template <int SP, int NB>
__global__ void __launch_bounds__(kTile) cg_init(CgArgs a)
{
    typedef typename SpinorFmt<SP>::R RS;
    constexpr int XP = XFmt<SP>::v;
    __shared__ CgSys s_sys;
    __shared__ double smem[32 * NB * kSums];
    __shared__ unsigned s_mask;
    stage_sys(a, blockIdx.x, &s_sys);
    const CgSys& S = s_sys;
    const TileInfo ti = decode_tile(S, blockIdx.x);
    const int Vh = S.g.Vh;
    for (int base = 0; base < S.nrhs; base += NB) {
        LanePass<NB> P;
        const int cnt = min(NB, S.nrhs - base);
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            P.lane[l] = l < cnt ? lane_of(S, base + l, ti.q, false) : 0;
            P.rid[l] = l < cnt ? __ldg(&a.lanes[P.lane[l]].rhs) : 0;
        }
        bool part[NB];
        double sums[NB * kSums];
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            part[l] = l < cnt;
#pragma unroll
            for (int f = 0; f < kSums; ++f) sums[l * kSums + f] = 0.0;
            if (l >= cnt || !ti.valid) continue;
            Vec3<double> b = SpinorFmt<SP_F64>::load(rhs_ptr(a, P.rid[l], F_B), ti.q, ti.i, Vh);
            Vec3<double> z;
            vzero(z);
            SpinorFmt<SP_F64>::store(rhs_ptr(a, P.rid[l], F_XHI), ti.q, ti.i, Vh, z);
            if (a.mixed)
                SpinorFmt<XP>::store(rhs_ptr(a, P.rid[l], F_XLO), ti.q, ti.i, Vh, vcvt<typename SpinorFmt<XP>::R>(z));
            const Vec3<RS> bq = SpinorFmt<SP>::store_q(rhs_ptr(a, P.rid[l], F_R), ti.q, ti.i, Vh, vcvt<RS>(b));
            SpinorFmt<SP>::store(rhs_ptr(a, P.rid[l], F_P), ti.q, ti.i, Vh, bq);
            sums[l * kSums + 3] = vdot_re(b, b);
        }
        block_sum<NB * kSums>(sums, smem);
        unsigned mask = arrive_sums<NB>(a, S, P, part, sums, ti.slot, S.both ? 2u * S.ntq : (unsigned)S.ntq,
                                        &s_mask);
        if (mask && threadIdx.x < 32) {
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (mask & (1u << l)) finish_init_lane(a, S, P.lane[l]);
        }
        __syncthreads();
    }
}

// FP64 hop of x_hi + x_lo for a lane in a reliable update: thi = K x
template <int XP, bool COH = false>
__device__ __forceinline__ void ru_hop1(const CgArgs& a, const CgSys& S, const Coord& c, int q, int i, int rid)
{
    const int nq = 1 - q, Vh = S.g.Vh;
    const void* xhi = rhs_ptr(a, rid, F_XHI);
    const void* xlo = rhs_ptr(a, rid, F_XLO);
    Vec3<double> acc;
    vzero(acc);
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu) {
        const bool eta_neg = eta_sign(c, mu) < 0;
        const int lu = lex_up(S.g, c, mu) >> 1, ld = lex_dn(S.g, c, mu) >> 1;
        const bool wu = (mu == 3) && (c.x[3] == S.g.L[3] - 1);
        const bool wd = (mu == 3) && (c.x[3] == 0);
        {
            Mat3<double> U = GaugeFmt<GP_F64_18>::load(S.U64, q, mu, i, Vh);
            Vec3<double> x = vaxpy(SpinorFmt<SP_F64>::template load<COH>(xhi, nq, lu, Vh), 1.0,
                                   vcvt<double>(SpinorFmt<XP>::template load<COH>(xlo, nq, lu, Vh)));
            vacc(acc, mul_mv(U, x), eta_neg != wu);
        }
        {
            Mat3<double> U = GaugeFmt<GP_F64_18>::load(S.U64, nq, mu, ld, Vh);
            Vec3<double> x = vaxpy(SpinorFmt<SP_F64>::template load<COH>(xhi, nq, ld, Vh), 1.0,
                                   vcvt<double>(SpinorFmt<XP>::template load<COH>(xlo, nq, ld, Vh)));
            vacc(acc, mul_adj_mv(U, x), !(eta_neg != wd));
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) acc.c[k] = {0.5 * acc.c[k].re, 0.5 * acc.c[k].im};
    SpinorFmt<SP_F64>::store(rhs_ptr(a, rid, F_THI), q, i, Vh, acc);
}

// Neighbour staging of one work item's tiles (schedule 6, FP16): buffer
// k & 1 of [2][NB][W] uint4 words holds tile k's range [i0 - Lt/2,
// i0 + kTile + Lt/2) of each active lane's input (tstage.cuh), filled by
// one thread's bulk copies completing on mbarrier k & 1; tile k + 1's copies
// are issued before tile k is computed, and a __syncthreads guards each
// buffer's reuse, so every thread walks every tile of the item.  The
// arithmetic is the unstaged kernels', operand for operand.
struct NstItem {
    uint4* buf;                 // [2][NB][W]
    unsigned long long* bar;    // [2]
    int W, tile0, nt;           // words per lane and buffer; the item's first tile in its parity; tiles
};

// thread 0: tile k's ranges of the active lanes into buffer k & 1
template <int NB>
__device__ __forceinline__ void nst_issue(const NstItem& st, const CgSys& S, int q, const void* const (&in)[NB],
                                          const bool (&on)[NB], int k)
{
    const TRange r = trange(S.g, (st.tile0 + k) * kTile, kTile);
    unsigned bytes = 0;
#pragma unroll
    for (int l = 0; l < NB; ++l)
        if (on[l]) bytes += (unsigned)r.cnt * 16u;
    unsigned long long* bar = st.bar + (k & 1);
    mbar_arrive_expect_tx(bar, bytes);
#pragma unroll
    for (int l = 0; l < NB; ++l)
        if (on[l])
            bulk_copy_g2s(st.buf + ((k & 1) * NB + l) * st.W, (const uint4*)in[l] + (size_t)(1 - q) * S.g.Vh + r.lo,
                          (unsigned)r.cnt * 16u, bar);
}

// set up the item's staging and issue its first tile (every thread calls it)
template <int NB>
__device__ __forceinline__ NstItem nst_begin(const CgArgs& a, const CgSys& S, const ItemRange& ir, int q,
                                             const void* const (&in)[NB], const bool (&on)[NB], void* dyn,
                                             unsigned long long* bar)
{
    NstItem st;
    st.buf = reinterpret_cast<uint4*>(dyn);
    st.bar = bar;
    st.W = a.nst_words;
    st.tile0 = ir.first - S.tile0 - q * S.ntq;
    st.nt = ir.end - ir.first;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) nst_issue<NB>(st, S, q, in, on, 0);
    return st;
}

// before tile k: issue tile k + 1 once every thread is done with tile k - 1,
// then wait (bounded) for tile k's copies; false: read tile k from global
// memory (DEV_ERR_TIMEOUT raised)
template <int NB>
__device__ __forceinline__ bool nst_next(const CgArgs& a, const NstItem& st, const CgSys& S, int q,
                                         const void* const (&in)[NB], const bool (&on)[NB], int k)
{
    if (k + 1 < st.nt) {
        __syncthreads();
        if (threadIdx.x == 0) nst_issue<NB>(st, S, q, in, on, k + 1);
    }
    const unsigned parity = (unsigned)(k >> 1) & 1u;
    if (mbar_wait_bounded(st.bar + (k & 1), parity)) return true;
    if (a.err) atomicOr(a.err, DEV_ERR_TIMEOUT);
    mbar_wait_bounded(st.bar + (k & 1), parity);  // the copy in flight lands before the buffer is reused
    return false;
}

// t = K p for the active lanes of one work item (tpi tiles of output parity
// q, one RHS group); thi for lanes in a reliable update
template <int GP, int SP, int NB, bool STG, bool RUI, bool NST>
__device__ __forceinline__ void hop1_item(const CgArgs& a, const int2 it, int cur)
{
    extern __shared__ __align__(16) unsigned char s_dyn[];
    typename GaugeFmt<GP>::E* sl = reinterpret_cast<typename GaugeFmt<GP>::E*>(s_dyn);
    typedef typename GaugeFmt<GP>::R R;
    typedef typename SpinorFmt<SP>::R RS;
    constexpr int XP = XFmt<SP>::v;
    __shared__ CgSys s_sys;
    stage_item_sys(a, it, &s_sys);
    const CgSys& S = s_sys;
    const ItemRange ir = item_range(a, S, it.x);
    const int q = ir.q, Vh = S.g.Vh;
    LanePass<NB> P;
    // the FP64 hop of lanes in a reliable update (mixed precisions only: FP64
    // vectors belong to the plain FP64 CG, which has no reliable updates;
    // RUI false: the lane-list kernels do it)
    constexpr bool ru_here = RUI && SP != SP_F64;
    const int base = item_rhs(it), cnt = min(NB, S.nrhs - base);
    // the vectors' addresses, loaded alongside the lanes' modes
    const void* pr[NB];
    const void* pp[NB];
    const void* tout[NB];
#pragma unroll
    for (int l = 0; l < NB; ++l) {
        pr[l] = l < cnt ? rhs_ptr(a, S.rhs0 + base + l, F_R) : nullptr;
        pp[l] = l < cnt ? rhs_ptr(a, S.rhs0 + base + l, F_P) : nullptr;
        tout[l] = l < cnt ? rhs_ptr(a, S.rhs0 + base + l, F_T) : nullptr;
    }
    gather_pass<NB>(a, S, base, q, true, cur, false, P);
    if (!(P.anyA || (ru_here && P.anyR))) return;
    const void* pin[NB];
    bool on[NB];
#pragma unroll
    for (int l = 0; l < NB; ++l) {
        on[l] = P.mode[l] == LM_ACTIVE || P.mode[l] == LM_RESTART;
        pin[l] = on[l] ? (P.mode[l] == LM_RESTART ? pr[l] : pp[l]) : nullptr;
    }
    if constexpr (NST) {
        if (P.anyA) {  // uniform across the block
            __shared__ __align__(8) unsigned long long s_bar[2];
            const NstItem st = nst_begin<NB>(a, S, ir, q, pin, on, s_dyn, s_bar);
            for (int k = 0; k < st.nt; ++k) {
                const bool ok = nst_next<NB>(a, st, S, q, pin, on, k);
                const TileInfo ti = decode_tile(S, ir.first + k);
                if (!ti.valid) continue;  // only the parity's last tile is partial
                const Nbr n = neighbours(S.g, eo_coords(S.g, q, ti.i));
                Vec3<R> acc[NB];
#pragma unroll
                for (int l = 0; l < NB; ++l) vzero(acc[l]);
                hop_lanes<GP, SP, NB, false, false, true>(S.Ulo, nullptr, n, q, ti.i, Vh, pin, on, acc,
                                                          st.buf + (k & 1) * NB * st.W, st.W,
                                                          trange(S.g, (st.tile0 + k) * kTile, kTile), ok);
#pragma unroll
                for (int l = 0; l < NB; ++l) {
                    if (!on[l]) continue;
                    SpinorFmt<SP>::store(const_cast<void*>(tout[l]), q, ti.i, Vh, vcvt<RS>(acc[l]));
                }
            }
        }
    } else if (P.anyA) {
        for (int t = ir.first; t < ir.end; ++t) {
            const TileInfo ti = decode_tile(S, t);
            if (!ti.valid) break;  // only the parity's last tile is partial
            const Nbr n = neighbours(S.g, eo_coords(S.g, q, ti.i));
            if constexpr (STG) {
                stage_links<GP>(sl, S.Ulo, n, q, ti.i, Vh);
                cp_async_wait_all();
            }
            Vec3<R> acc[NB];
#pragma unroll
            for (int l = 0; l < NB; ++l) vzero(acc[l]);
            hop_lanes<GP, SP, NB, STG>(S.Ulo, sl, n, q, ti.i, Vh, pin, on, acc);
#pragma unroll
            for (int l = 0; l < NB; ++l) {
                if (!on[l]) continue;
                SpinorFmt<SP>::store(const_cast<void*>(tout[l]), q, ti.i, Vh, vcvt<RS>(acc[l]));
            }
        }
    }
    if constexpr (ru_here) {
        // in a loop of its own: no call inside the hop loop
        if (P.anyR) {
            for (int t = ir.first; t < ir.end; ++t) {
                const TileInfo ti = decode_tile(S, t);
                if (!ti.valid) break;
                const Coord c = eo_coords(S.g, q, ti.i);
#pragma unroll 1
                for (int l = 0; l < NB; ++l)
                    if (P.mode[l] == LM_RU) ru_hop1<XP>(a, S, c, q, ti.i, P.rid[l]);
            }
        }
    }
}

// DYN: a grid of resident blocks takes the work items in turn from a
// device counter (a.qctr, zeroed by the iteration's update kernel), so no
// partial last wave idles the SMs and uneven items balance; otherwise one
// block per item
template <int GP, int SP, int NB, bool STG, bool RUI, bool NST = false, bool DYN = false>
__global__ void __launch_bounds__(kTile, (HopOcc<GP, SP, NB, false, RUI>::v))
    cg_hop1(CgArgs a, const int2* __restrict__ items, int cur)
{
    if constexpr (DYN) {
        __shared__ int s_next;
        for (;;) {
            if (threadIdx.x == 0) s_next = atomicAdd(a.qctr + 2 * cur + 0, 1);
            __syncthreads();
            const int idx = s_next;
            if (idx >= a.nitems1) break;  // uniform across the block
            hop1_item<GP, SP, NB, STG, RUI, NST>(a, items[idx], cur);
            __syncthreads();  // the item's shared memory and s_next are free again
        }
    } else {
        hop1_item<GP, SP, NB, STG, RUI, NST>(a, items[blockIdx.x], cur);
    }
}

// reliable update at the lane's own site: x_hi += x_lo, x_lo = 0,
// r = b - M x_hi; returns the |r|^2 contribution (FP64)
template <int SP, int XP, bool COH = false>
__device__ __forceinline__ double ru_hop2(const CgRhs* a, const CgSys& S, const Coord& c, int q, int i, int rid,
                                          double m2)
{
    typedef typename SpinorFmt<SP>::R RS;
    const int nq = 1 - q, Vh = S.g.Vh;
    const void* thi = rhs_ptr(a, rid, F_THI);
    Vec3<double> acc;
    vzero(acc);
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu) {
        const bool eta_neg = eta_sign(c, mu) < 0;
        const int lu = lex_up(S.g, c, mu) >> 1, ld = lex_dn(S.g, c, mu) >> 1;
        const bool wu = (mu == 3) && (c.x[3] == S.g.L[3] - 1);
        const bool wd = (mu == 3) && (c.x[3] == 0);
        Mat3<double> U = GaugeFmt<GP_F64_18>::load(S.U64, q, mu, i, Vh);
        vacc(acc, mul_mv(U, SpinorFmt<SP_F64>::template load<COH>(thi, nq, lu, Vh)), eta_neg != wu);
        Mat3<double> Ud = GaugeFmt<GP_F64_18>::load(S.U64, nq, mu, ld, Vh);
        vacc(acc, mul_adj_mv(Ud, SpinorFmt<SP_F64>::template load<COH>(thi, nq, ld, Vh)), !(eta_neg != wd));
    }
    void* xhi = rhs_ptr(a, rid, F_XHI);
    void* xlo = rhs_ptr(a, rid, F_XLO);
    Vec3<double> xn = vaxpy(SpinorFmt<SP_F64>::load_cg(xhi, q, i, Vh), 1.0,
                            vcvt<double>(SpinorFmt<XP>::load_cg(xlo, q, i, Vh)));
    SpinorFmt<SP_F64>::store(xhi, q, i, Vh, xn);
    Vec3<typename SpinorFmt<XP>::R> z;
    vzero(z);
    SpinorFmt<XP>::store(xlo, q, i, Vh, z);
    Vec3<double> b = SpinorFmt<SP_F64>::load(rhs_ptr(a, rid, F_B), q, i, Vh);
    Vec3<double> res;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        res.c[k].re = b.c[k].re - (m2 * xn.c[k].re - 0.5 * acc.c[k].re);
        res.c[k].im = b.c[k].im - (m2 * xn.c[k].im - 0.5 * acc.c[k].im);
    }
    // The search direction of the previous update, p = r_iter + beta p_old,
    // was built from the iterated residual; give it the true one instead,
    // p = r_true + beta p_old, by adding the correction r_true - r_iter.
    // Without it the low-precision lanes of ill-conditioned systems lose
    // their Krylov progress at every update (FP16 storage, eps = 1 links,
    // m = 0.02 on 16^4: 7648 iterations against FP64's 1564; 1750 with it).
    void* rp = rhs_ptr(a, rid, F_R);
    void* pp = rhs_ptr(a, rid, F_P);
    const Vec3<RS> r_iter = SpinorFmt<SP>::load_cg(rp, q, i, Vh);
    Vec3<RS> p = SpinorFmt<SP>::load_cg(pp, q, i, Vh);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        p.c[k].re += (RS)res.c[k].re - r_iter.c[k].re;
        p.c[k].im += (RS)res.c[k].im - r_iter.c[k].im;
    }
    SpinorFmt<SP>::store(pp, q, i, Vh, p);
    SpinorFmt<SP>::store(rp, q, i, Vh, vcvt<RS>(res));
    return vdot_re(res, res);
}

// one site's Re <a, b>: in FP32 for FP32 vectors (exactly the same value in
// every schedule, added to the FP64 partials), in FP64 for FP64 vectors
template <typename R>
__device__ __forceinline__ double site_dot(const Vec3<R>& a, const Vec3<R>& b)
{
    if constexpr (sizeof(R) == 4) {
        float s = a.c[0].re * b.c[0].re;
        s = fmaf(a.c[0].im, b.c[0].im, s);
#pragma unroll
        for (int k = 1; k < 3; ++k) {
            s = fmaf(a.c[k].re, b.c[k].re, s);
            s = fmaf(a.c[k].im, b.c[k].im, s);
        }
        return (double)s;
    } else {
        return vdot_re(a, b);
    }
}

// own sites of one work item (tpi tiles, one RHS group): v = m^2 p - K t and
// the four sums; reliable-update residuals
template <int GP, int SP, int NB, bool STG, bool RUI, bool NST>
__device__ __forceinline__ void hop2_item(const CgArgs& a, const int2 it, int cur)
{
    extern __shared__ __align__(16) unsigned char s_dyn[];
    typename GaugeFmt<GP>::E* sl = reinterpret_cast<typename GaugeFmt<GP>::E*>(s_dyn);
    typedef typename GaugeFmt<GP>::R R;
    typedef typename SpinorFmt<SP>::R RS;
    constexpr int XP = XFmt<SP>::v;
    __shared__ CgSys s_sys;
    __shared__ double smem[32 * NB * kSums];
    __shared__ unsigned s_mask;
    stage_item_sys(a, it, &s_sys);
    const CgSys& S = s_sys;
    const ItemRange ir = item_range(a, S, it.x);
    const int q = ir.q, Vh = S.g.Vh;
    LanePass<NB> P;
    // the reliable-update residuals are computed here too: measured faster
    // than a kernel of their own, and the compiler keeps the FP64 hop's
    // registers better with them here
    gather_pass<NB>(a, S, item_rhs(it), q, false, cur, false, P);
    if (!(P.anyA || (RUI && P.anyR))) return;  // uniform across the block
    bool part[NB], on[NB];
    double sums[NB * kSums];
    // this thread's partial sums across the item's tiles, in shared memory
    // rather than registers (fewer spills in the hop loop; measured 3 %
    // faster for FP32 storage, the same for FP16)
    __shared__ double s_part[NB * kSums][kTile];
    const void* tin[NB];
#pragma unroll
    for (int l = 0; l < NB; ++l) {
        on[l] = P.mode[l] == LM_ACTIVE || P.mode[l] == LM_RESTART;
        part[l] = on[l] || (RUI && P.mode[l] == LM_RU);
        tin[l] = on[l] ? rhs_ptr(a, P.rid[l], F_T) : nullptr;
#pragma unroll
        for (int f = 0; f < kSums; ++f) s_part[l * kSums + f][threadIdx.x] = 0.0;
    }
    // v = m^2 p - K t at the tile's sites and the lanes' partial sums
    auto own_sites = [&](const TileInfo& ti, Vec3<R>(&acc)[NB]) {
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            if (!on[l]) continue;
            const R m2 = (R)P.m2[l];
            Vec3<RS> r = SpinorFmt<SP>::load(rhs_ptr(a, P.rid[l], F_R), q, ti.i, Vh);
            Vec3<RS> p = r;
            if (P.mode[l] == LM_RESTART)  // restart: the search direction becomes r
                SpinorFmt<SP>::store(rhs_ptr(a, P.rid[l], F_P), q, ti.i, Vh, r);
            else
                p = SpinorFmt<SP>::load(rhs_ptr(a, P.rid[l], F_P), q, ti.i, Vh);
            Vec3<R> pr = vcvt<R>(p), w;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                w.c[k].re = fma(m2, pr.c[k].re, -acc[l].c[k].re);
                w.c[k].im = fma(m2, pr.c[k].im, -acc[l].c[k].im);
            }
            const Vec3<RS> vn = SpinorFmt<SP>::store_q(rhs_ptr(a, P.rid[l], F_V), q, ti.i, Vh, vcvt<RS>(w));
            s_part[l * kSums + 0][threadIdx.x] += site_dot(p, vn);
            s_part[l * kSums + 1][threadIdx.x] += site_dot(r, vn);
            s_part[l * kSums + 2][threadIdx.x] += site_dot(vn, vn);
            s_part[l * kSums + 3][threadIdx.x] += site_dot(r, r);
        }
    };
    if constexpr (NST) {
        if (P.anyA) {  // uniform across the block
            __shared__ __align__(8) unsigned long long s_bar[2];
            const NstItem st = nst_begin<NB>(a, S, ir, q, tin, on, s_dyn, s_bar);
            for (int k = 0; k < st.nt; ++k) {
                const bool ok = nst_next<NB>(a, st, S, q, tin, on, k);
                const TileInfo ti = decode_tile(S, ir.first + k);
                if (!ti.valid) continue;  // only the parity's last tile is partial
                const Nbr n = neighbours(S.g, eo_coords(S.g, q, ti.i));
                Vec3<R> acc[NB];
#pragma unroll
                for (int l = 0; l < NB; ++l) vzero(acc[l]);
                hop_lanes<GP, SP, NB, false, false, true>(S.Ulo, nullptr, n, q, ti.i, Vh, tin, on, acc,
                                                          st.buf + (k & 1) * NB * st.W, st.W,
                                                          trange(S.g, (st.tile0 + k) * kTile, kTile), ok);
                own_sites(ti, acc);
            }
        }
    } else if (P.anyA) {
        for (int t = ir.first; t < ir.end; ++t) {
            const TileInfo ti = decode_tile(S, t);
            if (!ti.valid) break;  // no barrier inside the loop
            const Nbr n = neighbours(S.g, eo_coords(S.g, q, ti.i));
            if constexpr (STG) {
                stage_links<GP>(sl, S.Ulo, n, q, ti.i, Vh);
                cp_async_wait_all();
            }
            Vec3<R> acc[NB];
#pragma unroll
            for (int l = 0; l < NB; ++l) vzero(acc[l]);
            hop_lanes<GP, SP, NB, STG>(S.Ulo, sl, n, q, ti.i, Vh, tin, on, acc);
            own_sites(ti, acc);
        }
    }
#pragma unroll
    for (int f = 0; f < NB * kSums; ++f) sums[f] = s_part[f][threadIdx.x];
    if (RUI && P.anyR) {
        for (int t = ir.first; t < ir.end; ++t) {
            const TileInfo ti = decode_tile(S, t);
            if (!ti.valid) break;
            const Coord c = eo_coords(S.g, q, ti.i);
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (P.mode[l] == LM_RU)
                    sums[l * kSums + 3] += ru_hop2<SP, XP>(a.rhs, S, c, q, ti.i, P.rid[l], P.m2[l]);
        }
    }
    block_sum<NB * kSums>(sums, smem);
    const unsigned nsq = (unsigned)item_groups(a, S);
    unsigned mask = arrive_sums<NB>(a, S, P, part, sums, ir.slot, S.both ? 2u * nsq : nsq, &s_mask);
    if (mask && threadIdx.x < 32) {
#pragma unroll
        for (int l = 0; l < NB; ++l)
            if (mask & (1u << l)) finish_lane(a, S, P.lane[l], P.mode[l], cur);
    }
}

// DYN: a grid of resident blocks takes the work items in turn from a
// device counter (a.qctr, zeroed by the iteration's update kernel), so no
// partial last wave idles the SMs and uneven items balance; otherwise one
// block per item
template <int GP, int SP, int NB, bool STG, bool RUI, bool NST = false, bool DYN = false>
__global__ void __launch_bounds__(kTile, (HopOcc<GP, SP, NB, true, RUI>::v))
    cg_hop2(CgArgs a, const int2* __restrict__ items, int cur)
{
    if constexpr (DYN) {
        __shared__ int s_next;
        for (;;) {
            if (threadIdx.x == 0) s_next = atomicAdd(a.qctr + 2 * cur + 1, 1);
            __syncthreads();
            const int idx = s_next;
            if (idx >= a.nitems2) break;  // uniform across the block
            hop2_item<GP, SP, NB, STG, RUI, NST>(a, items[idx], cur);
            __syncthreads();  // the item's shared memory and s_next are free again
        }
    } else {
        hop2_item<GP, SP, NB, STG, RUI, NST>(a, items[blockIdx.x], cur);
    }
}

// own sites of one lane (work item: tpi tiles, one RHS) if ACTIVE:
// x += alpha p, r -= alpha v, p = r + beta p
template <int SP, bool COH>
__device__ __forceinline__ void update_body(const CgArgs& a, int2 it, int cur, CgSys* s_sys)
{
    typedef typename SpinorFmt<SP>::R RS;
    constexpr int XP = XFmt<SP>::v;
    typedef typename SpinorFmt<XP>::R RX;
    // this iteration's reliable-update list was read by the kernels before
    // this one: empty it for the iteration after next
    if (a.ru_list && blockIdx.x == 0 && threadIdx.x == 0) a.ru_list[cur * (a.nlanes + 1)] = 0;
    // this iteration's hop kernels have taken their work items: their
    // counters start from zero again two iterations on
    if (a.qctr && blockIdx.x == 0 && threadIdx.x == 0) {
        a.qctr[2 * cur] = 0;
        a.qctr[2 * cur + 1] = 0;
    }
    stage_item_sys(a, it, s_sys);
    const CgSys& S = *s_sys;
    const ItemRange ir = item_range(a, S, it.x);
    const int q = ir.q, Vh = S.g.Vh;
    const int rid = S.rhs0 + item_rhs(it);
    void* pp = rhs_ptr(a, rid, F_P);
    void* rp = rhs_ptr(a, rid, F_R);
    void* xp = rhs_ptr(a, rid, F_XLO);
    const void* vp = rhs_ptr(a, rid, F_V);
    CgLane* L = a.lanes + lane_of(S, item_rhs(it), q, false);
    const int mode = ld_int(&L->mode[cur]);
    if (mode != LM_ACTIVE && mode != LM_RESTART && mode != LM_LAST) return;
    if (mode == LM_LAST && threadIdx.x == 0) {  // the last item retires the lane
        const unsigned nsq = (unsigned)item_groups(a, S);
        const unsigned expected = S.both ? 2u * nsq : nsq;
        if (atomicAdd(&L->ticket, 1u) == expected - 1) {
            L->ticket = 0;
            L->mode[cur] = LM_DONE;
        }
    }
    const double alpha = ld_dbl(&L->alpha), beta = ld_dbl(&L->beta);
    for (int t = ir.first; t < ir.end; ++t) {
        const TileInfo ti = decode_tile(S, t);
        if (!ti.valid) break;
        Vec3<RS> p = SpinorFmt<SP>::template load<COH>(pp, q, ti.i, Vh);
        Vec3<RS> r = SpinorFmt<SP>::template load<COH>(rp, q, ti.i, Vh);
        Vec3<RS> v = SpinorFmt<SP>::template load<COH>(vp, q, ti.i, Vh);
        Vec3<RX> x = SpinorFmt<XP>::template load<COH>(xp, q, ti.i, Vh);
        SpinorFmt<XP>::store(xp, q, ti.i, Vh, vaxpy(x, (RX)alpha, vcvt<RX>(p)));
        const Vec3<RS> rn = SpinorFmt<SP>::store_q(rp, q, ti.i, Vh, vaxpy(r, (RS)(-alpha), v));
        SpinorFmt<SP>::store(pp, q, ti.i, Vh, vaxpy(rn, (RS)beta, p));
    }
}

template <int SP>
__global__ void __launch_bounds__(kTile) cg_update(CgArgs a, const int2* __restrict__ items, int cur)
{
    __shared__ CgSys s_sys;
    update_body<SP, false>(a, items[blockIdx.x], cur, &s_sys);
}

// ---------------------------------------------------------------------------
// System-blocked hop kernels: one block per 256-site tile of one parity of
// one system, serving every right-hand side of the system.  The tile's links
// are read from HBM once and kept in shared memory for all RHS groups: FP16
// links unpacked (row 2 rebuilt) to nine half2 each, so the groups only read
// them; the other reduced precisions staged as stored and unpacked per
// group.  Within the block the RHS are taken NB at a time (register-blocked
// accumulators), the neighbour indices and hop signs computed once per site.
// The CG sums of cg_hop2_sys are reduced per group through shared memory in
// a fixed order (each site's dot products in FP32, summed in FP64).  The
// FP64 reliable-update hops run in kernels of their own (cg_ru1_list,
// cg_ru2_list, over the lanes due for one), so that their registers do not
// weigh on the hop kernels.
// ---------------------------------------------------------------------------
// unpacked FP16 links of a tile: [direction slot 8][half2 word 9][kTile]
constexpr size_t kHStageBytes = (size_t)8 * 9 * kTile * sizeof(uint32_t);

template <int GP, int SP> struct SysStage {
    static constexpr bool unpacked = (GP == GP_F16_12 && SP == SP_F16);
    static constexpr size_t bytes = unpacked ? kHStageBytes : StageBytes<GP>::v;
};

// resident blocks per SM of the system-blocked kernels: hop1 three (FP16
// unpacked links 72 KB, BF16 staged 48 KB), two for FP32-12 (96 KB staged);
// hop2 two (its per-group reduction rows on top of the links)
template <int GP, bool HOP2> struct SysOcc {
    static constexpr int v = (HOP2 || GP == GP_F32_12) ? 2 : 3;
};

// FP16 links of this thread's site (4 forward at the site, 4 backward at its
// neighbours), unpacked into its own column of the staging area
__device__ __forceinline__ void stage_hlinks(uint32_t* s, const void* Ulo, const Nbr& n, int q, int i, int Vh)
{
    const int nq = 1 - q, t = threadIdx.x;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        const uint2* f = (const uint2*)Ulo + ((size_t)(q * 4 + mu) * 3) * Vh + i;
        const uint2* b = (const uint2*)Ulo + ((size_t)(nq * 4 + mu) * 3) * Vh + n.dn[mu];
        uint2 w[2][3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            w[0][k] = __ldg(f + (size_t)k * Vh);
            w[1][k] = __ldg(b + (size_t)k * Vh);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            __half2 e[9];
            hlink_unpack(w[h], e);
#pragma unroll
            for (int k = 0; k < 9; ++k)
                s[((2 * mu + h) * 9 + k) * kTile + t] = *reinterpret_cast<const uint32_t*>(&e[k]);
        }
    }
}

__device__ __forceinline__ void hlink_smem(const uint32_t* s, int d, __half2 (&e)[9])
{
#pragma unroll
    for (int k = 0; k < 9; ++k) e[k] = h2_bits(s[(d * 9 + k) * kTile + threadIdx.x]);
}

// acc[l] += K in_l at the site for the lanes with on[l], links from the
// tile's staging area (unpacked FP16, or as stored for the other formats)
template <int GP, int SP, int NB, bool COH>
__device__ __forceinline__ void hop_lanes_sys(const void* Ulo, const void* stage, const Nbr& n, int q, int i,
                                              int Vh, const void* const (&in)[NB], const bool (&on)[NB],
                                              Vec3<typename GaugeFmt<GP>::R> (&acc)[NB])
{
    if constexpr (SysStage<GP, SP>::unpacked) {
        const uint32_t* sl = (const uint32_t*)stage;
        const int nq = 1 - q;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            const float s = ((n.eta >> mu) & 1u) ? -0.5f : 0.5f;
            __half2 U[9];
            hlink_smem(sl, 2 * mu, U);
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (on[l]) hop_half<false, COH>(acc[l], U, in[l], nq, n.up[mu], Vh, (n.wu && mu == 3) ? -s : s);
            hlink_smem(sl, 2 * mu + 1, U);
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (on[l]) hop_half<true, COH>(acc[l], U, in[l], nq, n.dn[mu], Vh, (n.wd && mu == 3) ? s : -s);
        }
    } else {
        hop_lanes<GP, SP, NB, true, COH>(Ulo, (const typename GaugeFmt<GP>::E*)stage, n, q, i, Vh, in, on, acc);
    }
}

template <int GP, int SP>
__device__ __forceinline__ void stage_tile_links(void* stage, const void* Ulo, const Nbr& n, int q, int i, int Vh)
{
    if constexpr (SysStage<GP, SP>::unpacked) {
        stage_hlinks((uint32_t*)stage, Ulo, n, q, i, Vh);
    } else {
        stage_links<GP>((typename GaugeFmt<GP>::E*)stage, Ulo, n, q, i, Vh);
        cp_async_wait_all();
    }
}

// which of the system's lanes take part in this phase (uniform in the block)
__device__ __forceinline__ void scan_lanes(const CgArgs& a, const CgSys& S, int q, bool hop1, int cur, bool* anyA,
                                           bool* anyR)
{
    bool A = false, R = false;
    for (int r = 0; r < S.nrhs; ++r) {
        const int m = ld_int(&a.lanes[lane_of(S, r, q, hop1)].mode[cur]);
        A |= m == LM_ACTIVE || m == LM_RESTART;
        R |= m == LM_RU;
    }
    *anyA = A;
    *anyR = R;
}

// hop1, system-blocked: t = K p for every active lane of the system on one
// tile (the lanes in a reliable update are ru1's)
template <int GP, int SP, int NB, bool COH>
__device__ __forceinline__ void hop1_sys_body(const CgArgs& a, int tile, int cur, CgSys* s_sys, void* stage)
{
    typedef typename GaugeFmt<GP>::R R;
    typedef typename SpinorFmt<SP>::R RS;
    stage_sys(a, tile, s_sys);
    const CgSys& S = *s_sys;
    const TileInfo ti = decode_tile(S, tile);
    const int q = ti.q, Vh = S.g.Vh;
    bool anyA, anyR;
    scan_lanes(a, S, q, true, cur, &anyA, &anyR);
    if (!anyA || !ti.valid) return;  // no barrier below
    const Nbr n = neighbours(S.g, eo_coords(S.g, q, ti.i));
    stage_tile_links<GP, SP>(stage, S.Ulo, n, q, ti.i, Vh);
    for (int base = 0; base < S.nrhs; base += NB) {
        LanePass<NB> P;
        gather_pass<NB>(a, S, base, q, true, cur, false, P);
        if (!P.anyA) continue;
        const void* pin[NB];
        bool on[NB];
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            on[l] = P.mode[l] == LM_ACTIVE || P.mode[l] == LM_RESTART;
            pin[l] = on[l] ? rhs_ptr(a, P.rid[l], P.mode[l] == LM_RESTART ? F_R : F_P) : nullptr;
        }
        Vec3<R> acc[NB];
#pragma unroll
        for (int l = 0; l < NB; ++l) vzero(acc[l]);
        hop_lanes_sys<GP, SP, NB, COH>(S.Ulo, stage, n, q, ti.i, Vh, pin, on, acc);
#pragma unroll
        for (int l = 0; l < NB; ++l)
            if (on[l]) SpinorFmt<SP>::store(rhs_ptr(a, P.rid[l], F_T), q, ti.i, Vh, vcvt<RS>(acc[l]));
    }
}

// Fixed-order block sum of F float rows (one value per thread each) in FP64:
// lane j of warp w adds the row's elements j, j + 32, ... in order, then the
// warp's lanes by the xor tree; results in tot[F] (all threads).
template <int F>
__device__ __forceinline__ void rows_sum(const float (&v)[F], float (*red)[kTile], double* tot)
{
#pragma unroll
    for (int f = 0; f < F; ++f) red[f][threadIdx.x] = v[f];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int f = warp; f < F; f += kTile / 32) {
        double x = 0.0;
#pragma unroll
        for (int k = 0; k < kTile / 32; ++k) x += (double)red[f][lane + 32 * k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) tot[f] = x;
    }
    __syncthreads();
}

// hop2, system-blocked: v = m^2 p - K t and the four CG sums for every active
// lane of the system on one tile (the lanes in a reliable update are ru2's)
template <int GP, int SP, int NB, bool COH>
__device__ __forceinline__ void hop2_sys_body(const CgArgs& a, int tile, int cur, CgSys* s_sys, void* stage,
                                              float (*s_red)[kTile], double* s_tot, unsigned* s_mask)
{
    typedef typename GaugeFmt<GP>::R R;
    typedef typename SpinorFmt<SP>::R RS;
    static_assert(sizeof(RS) == 4, "system-blocked kernels serve the reduced precisions");
    stage_sys(a, tile, s_sys);
    const CgSys& S = *s_sys;
    const TileInfo ti = decode_tile(S, tile);
    const int q = ti.q, Vh = S.g.Vh;
    const ItemRange ir = item_range(a, S, tile);
    const unsigned nsq = (unsigned)item_groups(a, S);
    bool anyA, anyR;
    scan_lanes(a, S, q, false, cur, &anyA, &anyR);
    if (!anyA) return;  // uniform in the block
    Nbr n;
    if (ti.valid) {
        n = neighbours(S.g, eo_coords(S.g, q, ti.i));
        stage_tile_links<GP, SP>(stage, S.Ulo, n, q, ti.i, Vh);
    }
    for (int base = 0; base < S.nrhs; base += NB) {
        LanePass<NB> P;
        gather_pass<NB>(a, S, base, q, false, cur, false, P);
        if (!P.anyA) continue;  // uniform in the block
        bool on[NB];
        const void* tin[NB];
        float v[NB * kSums];
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            on[l] = P.mode[l] == LM_ACTIVE || P.mode[l] == LM_RESTART;
            tin[l] = on[l] ? rhs_ptr(a, P.rid[l], F_T) : nullptr;
#pragma unroll
            for (int f = 0; f < kSums; ++f) v[l * kSums + f] = 0.f;
        }
        if (ti.valid) {
            Vec3<R> acc[NB];
#pragma unroll
            for (int l = 0; l < NB; ++l) vzero(acc[l]);
            hop_lanes_sys<GP, SP, NB, COH>(S.Ulo, stage, n, q, ti.i, Vh, tin, on, acc);
#pragma unroll
            for (int l = 0; l < NB; ++l) {
                if (!on[l]) continue;
                const R m2 = (R)P.m2[l];
                Vec3<RS> r = SpinorFmt<SP>::template load<COH>(rhs_ptr(a, P.rid[l], F_R), q, ti.i, Vh);
                Vec3<RS> p = r;
                if (P.mode[l] == LM_RESTART)  // restart: the search direction becomes r
                    SpinorFmt<SP>::store(rhs_ptr(a, P.rid[l], F_P), q, ti.i, Vh, r);
                else
                    p = SpinorFmt<SP>::template load<COH>(rhs_ptr(a, P.rid[l], F_P), q, ti.i, Vh);
                Vec3<R> pr = vcvt<R>(p), w;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    w.c[k].re = fma(m2, pr.c[k].re, -acc[l].c[k].re);
                    w.c[k].im = fma(m2, pr.c[k].im, -acc[l].c[k].im);
                }
                const Vec3<RS> vn = SpinorFmt<SP>::store_q(rhs_ptr(a, P.rid[l], F_V), q, ti.i, Vh, vcvt<RS>(w));
                v[l * kSums + 0] = (float)site_dot(p, vn);
                v[l * kSums + 1] = (float)site_dot(r, vn);
                v[l * kSums + 2] = (float)site_dot(vn, vn);
                v[l * kSums + 3] = (float)site_dot(r, r);
            }
        }
        rows_sum<NB * kSums>(v, s_red, s_tot);
        double sums[NB * kSums];
#pragma unroll
        for (int f = 0; f < NB * kSums; ++f) sums[f] = s_tot[f];
        const unsigned mask = arrive_sums<NB>(a, S, P, on, sums, ir.slot, nsq, s_mask);
        if (mask && threadIdx.x < 32) {
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (mask & (1u << l)) finish_lane(a, S, P.lane[l], P.mode[l], cur);
        }
        __syncthreads();
    }
}

// blocks of the lane-list kernels per SM (their grid, and their launch bounds)
constexpr int kListBlocksPerSm = 3;

// The FP64 reliable updates of the lanes on this iteration's list (the
// lanes whose recurrence asked for one in the last iteration), walked by a
// small fixed grid of nblk blocks.
// ru1: thi = K (x_hi + x_lo) on the tiles of the other parity; ru2: x_hi +=
// x_lo, r = b - M x_hi and |r|^2 on the lane's own tiles, in work items of
// tpi tiles whose sums complete the lane's partial-sum slots and ticket (the
// same order of additions as the hop kernels' own reliable-update loops).
// The listed lanes' work items (tpi tiles of a lane's tiles) are numbered in
// list order and dealt to the blocks round robin: pair k goes to block
// k mod nblk.  Every block walks the list (block-uniform) and takes its pairs.
template <int SP, bool COH>
__device__ __forceinline__ void ru1_list_body(const CgArgs& a, int cur, int blk, int nblk, CgSys* s_sys)
{
    constexpr int XP = XFmt<SP>::v;
    const int* lst = a.ru_list + cur * (a.nlanes + 1);
    const int n = ld_int(lst);
    int off = 0;  // pairs of the lanes before this one
    for (int u = 0; u < n; ++u) {
        const int lane = ld_int(lst + 1 + u);
        const CgLane* L = a.lanes + lane;  // sys, rhs and parity are fixed for the solve
        const int ntq = a.sys[L->sys].ntq;
        const int nsq = (ntq + a.tpi - 1) / a.tpi;
        int g = ((blk - off) % nblk + nblk) % nblk;  // this block's first item of the lane
        off += nsq;
        if (g >= nsq) continue;  // uniform in the block
        __syncthreads();
        if (threadIdx.x == 0) *s_sys = a.sys[L->sys];
        __syncthreads();
        const CgSys& S = *s_sys;
        const int q = 1 - L->parity, rid = L->rhs;
        for (; g < nsq; g += nblk) {
            const int j1 = min((g + 1) * a.tpi, S.ntq);
            for (int j = g * a.tpi; j < j1; ++j) {
                const int i = j * kTile + (int)threadIdx.x;
                if (i < S.g.Vh) ru_hop1<XP, COH>(a, S, eo_coords(S.g, q, i), q, i, rid);
            }
        }
    }
}

template <int SP, bool COH>
__device__ __forceinline__ void ru2_list_body(const CgArgs& a, int cur, int blk, int nblk, CgSys* s_sys,
                                              double* s_bs, unsigned* s_mask)
{
    constexpr int XP = XFmt<SP>::v;
    const int* lst = a.ru_list + cur * (a.nlanes + 1);
    const int n = ld_int(lst);
    int off = 0;
    for (int u = 0; u < n; ++u) {
        const int lane = ld_int(lst + 1 + u);
        const CgLane* L = a.lanes + lane;
        const int ntq = a.sys[L->sys].ntq;
        const int nsq = (ntq + a.tpi - 1) / a.tpi;
        int g = ((blk - off) % nblk + nblk) % nblk;
        off += nsq;
        if (g >= nsq) continue;  // uniform in the block
        __syncthreads();
        if (threadIdx.x == 0) *s_sys = a.sys[L->sys];
        __syncthreads();
        const CgSys& S = *s_sys;
        const int p = L->parity, rid = L->rhs;
        LanePass<1> P;
        P.lane[0] = lane;
        P.mode[0] = LM_RU;
        P.rid[0] = rid;
        P.alpha[0] = P.beta[0] = 0.0;
        P.m2[0] = L->m2;
        P.anyA = false;
        P.anyR = true;
        for (; g < nsq; g += nblk) {
            double sums[kSums] = {0.0, 0.0, 0.0, 0.0};
            const int j1 = min((g + 1) * a.tpi, S.ntq);
            for (int j = g * a.tpi; j < j1; ++j) {
                const int i = j * kTile + (int)threadIdx.x;
                if (i < S.g.Vh) sums[3] += ru_hop2<SP, XP, COH>(a.rhs, S, eo_coords(S.g, p, i), p, i, rid, P.m2[0]);
            }
            block_sum<kSums>(sums, s_bs);
            const bool part[1] = {true};
            const unsigned mask = arrive_sums<1>(a, S, P, part, sums, p * nsq + g, (unsigned)nsq, s_mask);
            if (mask && threadIdx.x < 32) finish_lane(a, S, lane, LM_RU, cur);
            __syncthreads();
        }
    }
}

template <int SP>
__global__ void __launch_bounds__(kTile, kListBlocksPerSm) cg_ru1_list(CgArgs a, const int2* __restrict__, int cur)
{
    __shared__ CgSys s_sys;
    ru1_list_body<SP, false>(a, cur, blockIdx.x, gridDim.x, &s_sys);
}

template <int SP>
__global__ void __launch_bounds__(kTile, kListBlocksPerSm) cg_ru2_list(CgArgs a, const int2* __restrict__, int cur)
{
    __shared__ CgSys s_sys;
    __shared__ double s_bs[32];
    __shared__ unsigned s_mask;
    ru2_list_body<SP, false>(a, cur, blockIdx.x, gridDim.x, &s_sys, s_bs, &s_mask);
}

template <int GP, int SP, int NB>
__global__ void __launch_bounds__(kTile, (SysOcc<GP, false>::v)) cg_hop1_sys(CgArgs a, const int2* __restrict__ items,
                                                                              int cur)
{
    extern __shared__ __align__(16) unsigned char s_dyn[];
    __shared__ CgSys s_sys;
    hop1_sys_body<GP, SP, NB, false>(a, items[blockIdx.x].x, cur, &s_sys, s_dyn);
}

template <int GP, int SP, int NB>
__global__ void __launch_bounds__(kTile, (SysOcc<GP, true>::v)) cg_hop2_sys(CgArgs a, const int2* __restrict__ items,
                                                                             int cur)
{
    extern __shared__ __align__(16) unsigned char s_dyn[];
    __shared__ CgSys s_sys;
    __shared__ float s_red[NB * kSums][kTile];
    __shared__ double s_tot[NB * kSums];
    __shared__ unsigned s_mask;
    hop2_sys_body<GP, SP, NB, false>(a, items[blockIdx.x].x, cur, &s_sys, s_dyn, s_red, s_tot, &s_mask);
}

// ---------------------------------------------------------------------------
// Persistent batched CG: the whole solve in one cooperative launch.  Every
// block walks the work items of each phase (grid-stride), the phases of an
// iteration separated by a grid barrier: {hop1, ru1}, {hop2, ru2}, update
// (hop1 and ru1 touch different lanes, as do hop2 and ru2, so each pair
// shares a phase; the reliable updates walk the lane list).  The per-tile bodies are those of the system-blocked
// kernels, with every load of data written during the solve taken through
// L2 (coherent across the blocks), so the solutions equal the graph path's
// bit for bit.  The grid barrier waits a bounded number of polls; a block
// that gives up sets the error word and returns, and the others follow at
// their next wait.
// ---------------------------------------------------------------------------
struct GridBar {
    unsigned count, gen;
    int err;  // set when a wait gave up
    unsigned pad;
    long long polls;  // bound on each wait
};

constexpr long long kBarrierPolls = 1ll << 25;  // about 4 s at the 128 ns back-off (the default bound)

__device__ __forceinline__ bool grid_barrier(GridBar* b, unsigned nblocks, int* s_ok)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &b->gen;
        volatile int* verr = &b->err;
        int ok = *verr == 0;
        const unsigned g = *vgen;
        __threadfence();
        if (ok) {
            if (atomicAdd(&b->count, 1u) == nblocks - 1) {
                atomicExch(&b->count, 0u);
                __threadfence();
                atomicAdd(&b->gen, 1u);
            } else {
                long long polls = 0;
                const long long limit = b->polls;
                while (*vgen == g) {
                    if (*verr != 0 || ++polls > limit) {
                        atomicOr(&b->err, 1);
                        ok = 0;
                        break;
                    }
                    __nanosleep(128);
                }
            }
        }
        __threadfence();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

template <int GP, int SP, int NB>
__global__ void __launch_bounds__(kTile, 2) cg_persistent_sys(CgArgs a, const int2* __restrict__ hop_items, int nhop,
                                                              const int2* __restrict__ upd_items, int nupd,
                                                              GridBar* bar)
{
    extern __shared__ __align__(16) unsigned char s_dyn[];
    __shared__ CgSys s_sys;
    __shared__ float s_red[NB * kSums][kTile];
    __shared__ double s_tot[NB * kSums];
    __shared__ double s_bs[32];
    __shared__ unsigned s_mask;
    __shared__ int s_ok;
    const unsigned nblk = gridDim.x;
    for (int it = 0; it < a.maxloop; ++it) {
        if (ld_int(a.n_active) <= 0) break;  // read after the last barrier: the same in every block
        const int cur = it & 1;
        for (int k = blockIdx.x; k < nhop; k += gridDim.x) {
            __syncthreads();
            hop1_sys_body<GP, SP, NB, true>(a, hop_items[k].x, cur, &s_sys, s_dyn);
        }
        ru1_list_body<SP, true>(a, cur, blockIdx.x, gridDim.x, &s_sys);
        if (!grid_barrier(bar, nblk, &s_ok)) return;
        for (int k = blockIdx.x; k < nhop; k += gridDim.x) {
            __syncthreads();
            hop2_sys_body<GP, SP, NB, true>(a, hop_items[k].x, cur, &s_sys, s_dyn, s_red, s_tot, &s_mask);
        }
        ru2_list_body<SP, true>(a, cur, blockIdx.x, gridDim.x, &s_sys, s_bs, &s_mask);
        if (!grid_barrier(bar, nblk, &s_ok)) return;
        for (int k = blockIdx.x; k < nupd; k += gridDim.x) {
            __syncthreads();
            update_body<SP, true>(a, upd_items[k], cur, &s_sys);
        }
        if (!grid_barrier(bar, nblk, &s_ok)) return;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

typedef void (*InitKernel)(CgArgs);
typedef void (*HopKernel)(CgArgs, const int2*, int);

// the kernels of one CG iteration, in launch order, with their work items
// and timing slots
enum { PH_HOP1 = 0, PH_HOP2 = 1, PH_UPDATE = 2, PH_RU1 = 3, PH_RU2 = 4, PH_PERSISTENT = 5, kTimedPhases = 6 };
typedef void (*PersKernel)(CgArgs, const int2*, int, const int2*, int, GridBar*);
constexpr int kMaxPhases = 5;

struct CgKernels {
    InitKernel init;
    HopKernel hop1, hop2, update;
    HopKernel ru1, ru2;  // separate reliable-update kernels (system-blocked schedule only)
    int nb1, nb2;   // RHS widths of the hop kernels' work items
    size_t smem;    // dynamic shared memory of the hop kernels (staged links)
    bool sys;       // system-blocked hop kernels (one tile per block, every RHS)
    PersKernel pers;  // the whole solve in one cooperative launch (or null)
    bool nst = false;  // hop kernels stage their neighbours (schedule 6)
    size_t nst1 = 0, nst2 = 0;  // their staging buffers' bytes (set per workspace)
    bool dyn = false;  // hop kernels take their work items from a counter (schedule 7)
    int grid1 = 0, grid2 = 0;  // their resident grids (set per solve; 0: one block per item)
};

struct Phase {
    HopKernel fn;
    int width;      // RHS width of the work items
    size_t smem;
    int slot;       // timing slot
    bool list;      // walks the reliable-update lane list with a fixed grid
    int grid;       // blocks of a resident grid taking items from a counter (0: one per item)
};

// blocks a phase launches for nitems work items
static int phase_grid(const Phase& p, int nitems) { return p.grid > 0 ? std::min(p.grid, nitems) : nitems; }

static int phases_of(const CgKernels& k, Phase (&ph)[kMaxPhases])
{
    int n = 0;
    ph[n++] = {k.hop1, k.nb1, k.smem + k.nst1, PH_HOP1, false, k.grid1};
    if (k.ru1) ph[n++] = {k.ru1, k.nb1, 0, PH_RU1, true, 0};
    ph[n++] = {k.hop2, k.nb2, k.smem + k.nst2, PH_HOP2, false, k.grid2};
    if (k.ru2) ph[n++] = {k.ru2, k.nb2, 0, PH_RU2, true, 0};
    ph[n++] = {k.update, 1, 0, PH_UPDATE, false, 0};
    return n;
}



// work-item width of the system-blocked kernels: one item per tile, covering
// every RHS of the system
constexpr int kSysItems = 1 << 20;

// the largest neighbour-staging buffers of a hop kernel (schedule 6): two
// buffers of four RHS at Lt up to 1024 fit
constexpr size_t kMaxNstBytes = 160 * 1024;

template <int GP, int SP>
static CgKernels pick_sys(int nb, bool persistent)
{
    CgKernels k;
    // FP32 arithmetic on FP32 links keeps at most four accumulators in
    // registers; the packed-half FP16 products take eight
    if (nb >= 4) { k.hop1 = cg_hop1_sys<GP, SP, 4>; k.hop2 = cg_hop2_sys<GP, SP, 4>; }
    else if (nb >= 2) { k.hop1 = cg_hop1_sys<GP, SP, 2>; k.hop2 = cg_hop2_sys<GP, SP, 2>; }
    else { k.hop1 = cg_hop1_sys<GP, SP, 1>; k.hop2 = cg_hop2_sys<GP, SP, 1>; }
    k.pers = nullptr;
    if (persistent) {
        if (nb >= 4) k.pers = cg_persistent_sys<GP, SP, 4>;
        else if (nb >= 2) k.pers = cg_persistent_sys<GP, SP, 2>;
        else k.pers = cg_persistent_sys<GP, SP, 1>;
    }
    if constexpr (SysStage<GP, SP>::unpacked) {
        if (nb >= 8) {
            k.hop1 = cg_hop1_sys<GP, SP, 8>;
            k.hop2 = cg_hop2_sys<GP, SP, 8>;
            if (persistent) k.pers = cg_persistent_sys<GP, SP, 8>;
        }
    }
    k.init = cg_init<SP, 2>;
    k.update = cg_update<SP>;
    k.ru1 = cg_ru1_list<SP>;
    k.ru2 = cg_ru2_list<SP>;
    k.nb1 = k.nb2 = kSysItems;
    k.smem = SysStage<GP, SP>::bytes;
    k.sys = true;
    return k;
}

template <int GP, int SP, bool STG, bool RUI>
static HopKernel pick_hop1(int nb, int* nb_eff)
{
    if constexpr (SP != SP_F64) {
        if (nb >= 8) { *nb_eff = 8; return cg_hop1<GP, SP, 8, STG, RUI>; }
        if (nb >= 4) { *nb_eff = 4; return cg_hop1<GP, SP, 4, STG, RUI>; }
    }
    if (nb >= 2) { *nb_eff = 2; return cg_hop1<GP, SP, 2, STG, RUI>; }
    *nb_eff = 1;
    return cg_hop1<GP, SP, 1, STG, RUI>;
}

template <int GP, int SP, bool STG, bool RUI>
static void pick_hop2(int nb, HopKernel* hop2, InitKernel* init, int* nb_eff)
{
    if constexpr (SP != SP_F64) {
        if (nb >= 4) { *hop2 = cg_hop2<GP, SP, 4, STG, RUI>; *init = cg_init<SP, 4>; *nb_eff = 4; return; }
    }
    if (nb >= 2) { *hop2 = cg_hop2<GP, SP, 2, STG, RUI>; *init = cg_init<SP, 2>; *nb_eff = 2; return; }
    *hop2 = cg_hop2<GP, SP, 1, STG, RUI>;
    *init = cg_init<SP, 1>;
    *nb_eff = 1;
}

// RUI: the hop kernels do the reliable-update hops of their lanes (inline);
// otherwise the lane-list kernels cg_ru1_list / cg_ru2_list follow them
template <int GP, int SP, bool STG, bool RUI>
static CgKernels pick_typed(int nb1, int nb2)
{
    CgKernels k;
    k.hop1 = pick_hop1<GP, SP, STG, RUI>(nb1, &k.nb1);
    pick_hop2<GP, SP, STG, RUI>(nb2, &k.hop2, &k.init, &k.nb2);
    k.update = cg_update<SP>;
    if constexpr (RUI || SP == SP_F64) {
        k.ru1 = k.ru2 = nullptr;
    } else {
        k.ru1 = cg_ru1_list<SP>;
        k.ru2 = cg_ru2_list<SP>;
    }
    k.smem = STG ? StageBytes<GP>::v : 0;
    k.sys = false;
    k.pers = nullptr;
    return k;
}

// schedule 6 (FP16): schedule 4's kernels with each tile's time and z
// neighbours staged in shared memory; RHS groups of at most four
template <int GP, int SP>
static CgKernels pick_nst(int nb1, int nb2)
{
    CgKernels k = pick_typed<GP, SP, false, false>(nb1, nb2);
    if (nb1 >= 4) { k.hop1 = cg_hop1<GP, SP, 4, false, false, true>; k.nb1 = 4; }
    else if (nb1 >= 2) { k.hop1 = cg_hop1<GP, SP, 2, false, false, true>; k.nb1 = 2; }
    else { k.hop1 = cg_hop1<GP, SP, 1, false, false, true>; k.nb1 = 1; }
    if (nb2 >= 4) { k.hop2 = cg_hop2<GP, SP, 4, false, false, true>; k.nb2 = 4; }
    else if (nb2 >= 2) { k.hop2 = cg_hop2<GP, SP, 2, false, false, true>; k.nb2 = 2; }
    else { k.hop2 = cg_hop2<GP, SP, 1, false, false, true>; k.nb2 = 1; }
    k.nst = true;
    return k;
}

// schedule 7: schedule 4's kernels on resident grids taking their work
// items from a counter
template <int GP, int SP>
static CgKernels pick_dyn(int nb1, int nb2)
{
    CgKernels k = pick_typed<GP, SP, false, false>(nb1, nb2);
    if constexpr (SP != SP_F64) {
        if (nb1 >= 8) { k.hop1 = cg_hop1<GP, SP, 8, false, false, false, true>; k.nb1 = 8; }
        else if (nb1 >= 4) { k.hop1 = cg_hop1<GP, SP, 4, false, false, false, true>; k.nb1 = 4; }
        else if (nb1 >= 2) { k.hop1 = cg_hop1<GP, SP, 2, false, false, false, true>; k.nb1 = 2; }
        else { k.hop1 = cg_hop1<GP, SP, 1, false, false, false, true>; k.nb1 = 1; }
        if (nb2 >= 4) { k.hop2 = cg_hop2<GP, SP, 4, false, false, false, true>; k.nb2 = 4; }
        else if (nb2 >= 2) { k.hop2 = cg_hop2<GP, SP, 2, false, false, false, true>; k.nb2 = 2; }
        else { k.hop2 = cg_hop2<GP, SP, 1, false, false, false, true>; k.nb2 = 1; }
        k.dyn = true;
    }
    return k;
}

template <int GP, int SP>
static CgKernels pick_staged(int nb1, int nb2, bool stage, bool list)
{
    if constexpr (GP == GP_F64_18) {
        return pick_typed<GP, SP, false, true>(nb1, nb2);
    } else {
        if (list) return stage ? pick_typed<GP, SP, true, false>(nb1, nb2) : pick_typed<GP, SP, false, false>(nb1, nb2);
        return stage ? pick_typed<GP, SP, true, true>(nb1, nb2) : pick_typed<GP, SP, false, true>(nb1, nb2);
    }
}

// stage: 0 links read directly, 1 staged per work item, 2 system-blocked
// kernels, 3 the system-blocked bodies in one persistent cooperative launch
// (2 and 3: FP16, BF16 and FP32 12-real storage; FP32-18 takes 1)
// stage 4, 5: 0, 1 with the reliable updates in the lane-list kernels
// stage 6: 4 with the neighbours staged along the time direction (FP16; the
// other precisions run 4); stage 7: 4 with the hop kernels on resident grids
// taking their work items from a counter (FP64 runs 0)
static CgKernels pick_kernels(int prec, int nb1, int nb2, int stage)
{
    CgKernels k;
    if (stage == 6 && prec == SFH_PREC_F16) return pick_nst<GP_F16_12, SP_F16>(nb1, nb2);
    if (stage == 7) {
        if (prec == SFH_PREC_F16) return pick_dyn<GP_F16_12, SP_F16>(nb1, nb2);
        if (prec == SFH_PREC_F32) return pick_dyn<GP_F32_12, SP_F32>(nb1, nb2);
        if (prec == SFH_PREC_BF16) return pick_dyn<GP_BF16_12, SP_BF16>(nb1, nb2);
        if (prec == SFH_PREC_F32_18) return pick_dyn<GP_F32_18, SP_F32>(nb1, nb2);
        stage = 0;  // FP64: schedule 0
    }
    const bool sys = stage == 2 || stage == 3, pers = stage == 3, list = stage >= 4;
    const bool stg = stage == 1 || stage == 5 || (sys && prec == SFH_PREC_F32_18);
    if (prec == SFH_PREC_F64) k = pick_staged<GP_F64_18, SP_F64>(nb1, nb2, false, false);
    else if (sys && prec == SFH_PREC_F16) k = pick_sys<GP_F16_12, SP_F16>(nb1, pers);
    else if (sys && prec == SFH_PREC_BF16) k = pick_sys<GP_BF16_12, SP_BF16>(nb1, pers);
    else if (sys && prec == SFH_PREC_F32) k = pick_sys<GP_F32_12, SP_F32>(nb1, pers);
    else if (prec == SFH_PREC_F32) k = pick_staged<GP_F32_12, SP_F32>(nb1, nb2, stg, list);
    else if (prec == SFH_PREC_F32_18) k = pick_staged<GP_F32_18, SP_F32>(nb1, nb2, stg, list);
    else if (prec == SFH_PREC_BF16) k = pick_staged<GP_BF16_12, SP_BF16>(nb1, nb2, stg, list);
    else k = pick_staged<GP_F16_12, SP_F16>(nb1, nb2, stg, list);
    if (k.smem) {  // opt in to the staged kernels' shared memory (idempotent)
        cudaFuncSetAttribute((const void*)k.hop1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem);
        cudaFuncSetAttribute((const void*)k.hop2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem);
        if (k.pers)
            cudaFuncSetAttribute((const void*)k.pers, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem);
    }
    return k;
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
    GridBar* d_bar = nullptr;  // grid barrier of the persistent solve
    int* d_rulist = nullptr;   // reliable-update lane lists [2][1 + nlanes]
    int* d_qctr = nullptr;     // work-item counters of schedule 7 [2][2]
    bool timed_out = false;    // the last persistent solve gave up at a barrier
    long long barrier_polls = 0;  // bound on each barrier wait (0: the default)
    int num_sms = 0;
    std::vector<void*> allocs;
    size_t bytes = 0;
    // iteration chunks replayed as one graph launch each
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CgKernels gk = {};
    double g_tol = -1.0, g_delta = -1.0;
    int g_maxit = -1, g_tpi = -1;
    int* h_active = nullptr;  // pinned, two slots
    cudaEvent_t ev[2] = {nullptr, nullptr};
    long launches = 0;        // kernels launched by the last solve
    struct Items {
        int nb, tpi;
        int2* ptr;
        int n;
    };
    std::vector<Items> item_cache;  // work-item lists by RHS-group width

    ~CgWorkspace() { release(); }
    void release_graph()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        g_tol = -1.0;
    }
    void release()
    {
        release_graph();
        if (h_active) cudaFreeHost(h_active);
        h_active = nullptr;
        for (int k = 0; k < 2; ++k)
            if (ev[k]) cudaEventDestroy(ev[k]);
        ev[0] = ev[1] = nullptr;
        for (void* p : allocs) cudaFree(p);
        allocs.clear();
        item_cache.clear();
        d_sys = nullptr; d_rhs = nullptr; d_lanes = nullptr;
        d_tile_sys = nullptr; d_partial = nullptr; d_active = nullptr; d_bar = nullptr; d_rulist = nullptr; d_qctr = nullptr;
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
    const int sp = prec == SFH_PREC_F64 ? SP_F64 : (prec == SFH_PREC_F16 ? SP_F16 : (prec == SFH_PREC_BF16 ? SP_BF16 : SP_F32));
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
        S.rhs0 = (int)w.rhs.size();
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
                L.m2 = S.m2;
                L.parity = both ? 2 : lp;
                L.poff = poff;  // slots indexed by the tile's local index (both parities)
                poff += kSums * 2 * S.ntq;
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
    if ((e = w.alloc((void**)&w.d_rulist, sizeof(int) * 2 * (w.nlanes + 1))) != cudaSuccess) return e;
    {
        int dev = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&w.num_sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    }
    if ((e = cudaMemcpy(w.d_sys, w.sys.data(), sizeof(CgSys) * w.nsys, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if (!w.rhs.empty())
        if ((e = cudaMemcpy(w.d_rhs, w.rhs.data(), sizeof(CgRhs) * w.rhs.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if ((e = cudaMemcpy(w.d_tile_sys, tile_sys.data(), sizeof(int) * tile_sys.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if ((e = cudaHostAlloc((void**)&w.h_active, 2 * sizeof(int), cudaHostAllocDefault)) != cudaSuccess) return e;
    for (int k = 0; k < 2; ++k)
        if ((e = cudaEventCreateWithFlags(&w.ev[k], cudaEventDisableTiming)) != cudaSuccess) return e;
    return cudaSuccess;
}

static int default_nb(int max_nrhs, int cap)
{
    int nb = 1;
    while (nb < max_nrhs && nb < cap) nb *= 2;
    return nb;
}

constexpr int kChunk = 16;  // CG iterations per graph launch (even)

// Work items (first tile, first RHS): tpi tiles of one parity of a system and
// one RHS group of width nb; one block each.  The groups of a tile range are
// adjacent, so the blocks sharing its links run side by side and the second
// and later reads of a link hit L2.
static cudaError_t items_for(CgWorkspace& w, int nb, int tpi, const int2** d, int* n)
{
    for (const CgWorkspace::Items& c : w.item_cache)
        if (c.nb == nb && c.tpi == tpi) {
            *d = c.ptr;
            *n = c.n;
            return cudaSuccess;
        }
    std::vector<int2> h;
    for (int k = 0; k < (int)w.sys.size(); ++k) {
        const CgSys& S = w.sys[k];
        for (int q = 0; q < 2; ++q)
            for (int j = 0; j < S.ntq; j += tpi)
                for (int b = 0; b < S.nrhs; b += nb)
                    h.push_back(make_int2(S.tile0 + q * S.ntq + j, b | (k << kItemSysShift)));
    }
    int2* p = nullptr;
    cudaError_t e = w.alloc((void**)&p, sizeof(int2) * std::max<size_t>(1, h.size()));
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(p, h.data(), sizeof(int2) * h.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    w.item_cache.push_back({nb, tpi, p, (int)h.size()});
    *d = p;
    *n = (int)h.size();
    return cudaSuccess;
}

static CgArgs make_args(const CgWorkspace& w, double tol, int maxit, double delta, int tpi)
{
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
    a.restart = 0;  // restart only when an update shows little progress (finish_lane)
    a.maxloop = a.mixed ? 2 * maxit + 64 : maxit + 1;
    a.tpi = tpi;
    a.ru_list = nullptr;
    a.nst_words = 0;
    a.err = nullptr;
    a.qctr = nullptr;
    a.nitems1 = a.nitems2 = 0;
    return a;
}

// (Re)build the graph of kChunk iterations: the iteration's kernels in order
// (hop1, hop2, update; with the system-blocked schedule hop1, ru1, hop2, ru2,
// update), repeated
static bool same_kernels(const CgKernels& a, const CgKernels& b)
{
    return a.hop1 == b.hop1 && a.hop2 == b.hop2 && a.update == b.update && a.ru1 == b.ru1 && a.ru2 == b.ru2;
}

static cudaError_t ensure_graph(CgWorkspace& w, const CgKernels& k, CgArgs a, double tol, int maxit,
                                double delta)
{
    if (w.exec && same_kernels(w.gk, k) && w.g_tol == tol && w.g_tpi == a.tpi && w.g_maxit == maxit &&
        w.g_delta == delta)
        return cudaSuccess;
    w.release_graph();
    Phase ph[kMaxPhases];
    const int nph = phases_of(k, ph);
    const int2* items[kMaxPhases];
    int nitems[kMaxPhases];
    cudaError_t e;
    for (int j = 0; j < nph; ++j) {
        if ((e = items_for(w, ph[j].width, a.tpi, &items[j], &nitems[j])) != cudaSuccess) return e;
        if (ph[j].list) nitems[j] = kListBlocksPerSm * w.num_sms;
    }
    e = cudaGraphCreate(&w.graph, 0);
    if (e != cudaSuccess) return e;
    cudaGraphNode_t prev = nullptr;
    for (int it = 0; it < kChunk; ++it) {
        int cur = it & 1;
        for (int j = 0; j < nph; ++j) {
            cudaKernelNodeParams p;
            std::memset(&p, 0, sizeof(p));
            p.func = (void*)ph[j].fn;
            p.gridDim = dim3(phase_grid(ph[j], nitems[j]));
            p.blockDim = dim3(kTile);
            p.sharedMemBytes = (unsigned)ph[j].smem;
            void* args[] = {&a, (void*)&items[j], &cur};
            p.kernelParams = args;
            cudaGraphNode_t node;
            e = cudaGraphAddKernelNode(&node, w.graph, prev ? &prev : nullptr, prev ? 1 : 0, &p);
            if (e != cudaSuccess) return e;
            prev = node;
        }
    }
    e = cudaGraphInstantiate(&w.exec, w.graph, 0);
    if (e != cudaSuccess) return e;
    w.gk = k;
    w.g_tol = tol;
    w.g_maxit = maxit;
    w.g_delta = delta;
    w.g_tpi = a.tpi;
    return cudaSuccess;
}

// Device time of each iteration kernel over one solve (timed solves launch
// the kernels one by one between CUDA events instead of replaying the graph),
// by timing slot: hop1, hop2, update, ru1, ru2.
struct PhaseTimes {
    double ms[kTimedPhases];
    long n[kTimedPhases];
};

static cudaError_t finish_solve(CgWorkspace& w, cudaStream_t stream);

// The persistent schedule: the whole solve (after cg_init) in one cooperative
// launch of as many blocks as fit on the GPU at once, each walking the work
// items of every phase.  Same per-tile bodies and reductions as the
// system-blocked graph path, so the same solutions.
static cudaError_t persistent_solve(CgWorkspace& w, const CgKernels& k, CgArgs a, cudaStream_t stream,
                                    PhaseTimes* timing)
{
    cudaError_t e;
    if (!w.d_bar && (e = w.alloc((void**)&w.d_bar, sizeof(GridBar))) != cudaSuccess) return e;
    if (!w.num_sms) {
        int dev = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&w.num_sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    }
    const int2* hop_items;
    const int2* upd_items;
    int nhop = 0, nupd = 0;
    if ((e = items_for(w, kSysItems, 1, &hop_items, &nhop)) != cudaSuccess) return e;
    if ((e = items_for(w, 1, 1, &upd_items, &nupd)) != cudaSuccess) return e;
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.pers, kTile, k.smem)) != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    const int grid = std::max(1, std::min(per_sm * w.num_sms, std::max(nhop, nupd)));
    GridBar bar0;
    std::memset(&bar0, 0, sizeof(bar0));
    bar0.polls = w.barrier_polls > 0 ? w.barrier_polls : kBarrierPolls;
    if ((e = cudaMemcpyAsync(w.d_bar, &bar0, sizeof(GridBar), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return e;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    if (timing) {
        for (int r = 0; r < kTimedPhases; ++r) {
            timing->ms[r] = 0.0;
            timing->n[r] = 0;
        }
        for (cudaEvent_t& x : ev)
            if ((e = cudaEventCreate(&x)) != cudaSuccess) return e;
        cudaEventRecord(ev[0], stream);
    }
    void* args[] = {&a, (void*)&hop_items, &nhop, (void*)&upd_items, &nupd, (void*)&w.d_bar};
    e = cudaLaunchCooperativeKernel((const void*)k.pers, dim3(grid), dim3(kTile), args, k.smem, stream);
    w.launches += 1;
    if (timing) {
        if (e == cudaSuccess) e = cudaEventRecord(ev[1], stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
        timing->ms[PH_PERSISTENT] = ms;
        timing->n[PH_PERSISTENT] = 1;
        for (cudaEvent_t x : ev)
            if (x) cudaEventDestroy(x);
    }
    if (e != cudaSuccess) return e;
    int err = 0;
    if ((e = cudaMemcpyAsync(&err, &w.d_bar->err, sizeof(int), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
        return e;
    if ((e = finish_solve(w, stream)) != cudaSuccess) return e;
    w.timed_out = err != 0;
    return cudaSuccess;
}

// Reliable-update threshold (|r| drop between FP64 updates) of the mixed
// precisions: FP16 storage needs the tighter 0.1 (at 0.02 its recurrence
// drifts too far to converge); FP32 keeps its recurrence to 0.01, half the
// updates of 0.1 at the same iteration count.
static double default_reliable_delta(int prec)
{
    return (prec == SFH_PREC_F16 || prec == SFH_PREC_BF16) ? 0.1 : 0.01;
}

// Tiles per work item when the caller leaves it open: two, or one where two
// would give the first hop fewer than four work items per SM.  A single
// 16^4 solve has 128 two-tile items for 148 SMs; with one tile per item it
// ran 15 % (FP64) to 20 % (FP16) faster.  The choice never changes results.
static int default_tpi(const CgWorkspace& w, int nb1)
{
    long items = 0;  // first-hop work items at two tiles each
    for (const CgSys& S : w.sys) items += 2L * ((S.ntq + 1) / 2) * ((S.nrhs + nb1 - 1) / std::max(1, nb1));
    return items < 4L * std::max(1, w.num_sms) ? 1 : 2;
}

// Solve every lane of a built workspace.  nb1 / nb2: RHS-block widths of the
// two hop kernels (0 = from the largest RHS count); tpi: tiles per block of
// the iteration kernels (0 = default_tpi); stage: hop kernels stage their
// links in shared memory (reduced precisions only).  Returns a cudaError.
static cudaError_t workspace_solve(CgWorkspace& w, double tol, int maxit, double delta, int nb1, int nb2,
                                   int tpi, int stage, cudaStream_t stream, PhaseTimes* timing = nullptr)
{
    int max_nrhs = 1;
    for (const CgSys& S : w.sys) max_nrhs = std::max(max_nrhs, S.nrhs);
    const bool f64 = w.prec == SFH_PREC_F64;
    if (nb1 <= 0) nb1 = default_nb(max_nrhs, f64 ? 2 : 8);
    if (nb2 <= 0) nb2 = default_nb(max_nrhs, f64 ? 2 : 4);
    w.nb = nb1;
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
    w.h_active[0] = w.h_active[1] = w.nlanes;
    if ((e = cudaMemcpyAsync(w.d_active, &w.h_active[0], sizeof(int), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return e;
    CgKernels k = pick_kernels(w.prec, nb1, nb2, stage);
    int nst_words = 0;
    if (k.nst) {  // staging buffers for the batch's largest Lt; schedule 4 where they do not fit
        int max_lt = 2;
        for (const CgSys& S : w.sys) max_lt = std::max(max_lt, S.g.L[3]);
        nst_words = kTile + max_lt;
        k.nst1 = (size_t)2 * k.nb1 * nst_words * sizeof(uint4);
        k.nst2 = (size_t)2 * k.nb2 * nst_words * sizeof(uint4);
        if (std::max(k.nst1, k.nst2) > kMaxNstBytes) {
            k = pick_kernels(w.prec, nb1, nb2, 4);
            nst_words = 0;
        } else {
            if ((e = cudaFuncSetAttribute((const void*)k.hop1, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)k.nst1)) != cudaSuccess)
                return e;
            if ((e = cudaFuncSetAttribute((const void*)k.hop2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)k.nst2)) != cudaSuccess)
                return e;
            if (!w.d_bar && (e = w.alloc((void**)&w.d_bar, sizeof(GridBar))) != cudaSuccess) return e;
            if ((e = cudaMemsetAsync(&w.d_bar->err, 0, sizeof(int), stream)) != cudaSuccess) return e;
        }
    }
    // the system-blocked kernels serve one tile per block: one partial-sum
    // slot per tile, so every kernel of the iteration takes single tiles
    CgArgs a = make_args(w, tol, maxit, delta, k.sys ? 1 : (tpi > 0 ? tpi : default_tpi(w, k.nb1)));
    if (k.nst) {
        a.nst_words = nst_words;
        a.err = &w.d_bar->err;
    }
    if (k.dyn) {  // resident grids: as many blocks as fit at once, at most one per item
        if (!w.d_qctr && (e = w.alloc((void**)&w.d_qctr, 4 * sizeof(int))) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(w.d_qctr, 0, 4 * sizeof(int), stream)) != cudaSuccess) return e;
        const int2* it;
        if ((e = items_for(w, k.nb1, a.tpi, &it, &a.nitems1)) != cudaSuccess) return e;
        if ((e = items_for(w, k.nb2, a.tpi, &it, &a.nitems2)) != cudaSuccess) return e;
        int b1 = 0, b2 = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k.hop1, kTile, k.smem)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, k.hop2, kTile, k.smem)) != cudaSuccess) return e;
        k.grid1 = std::max(1, b1) * w.num_sms;
        k.grid2 = std::max(1, b2) * w.num_sms;
        a.qctr = w.d_qctr;
    }
    if (k.ru1 || k.pers) {  // reliable updates by lane list: both lists start empty
        a.ru_list = w.d_rulist;
        if ((e = cudaMemsetAsync(w.d_rulist, 0, sizeof(int) * 2 * (w.nlanes + 1), stream)) != cudaSuccess) return e;
    }
    k.init<<<w.ntiles, kTile, 0, stream>>>(a);
    w.launches = 1;
    w.timed_out = false;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (k.pers) return persistent_solve(w, k, a, stream, timing);
    if (!timing && (e = ensure_graph(w, k, a, tol, maxit, delta)) != cudaSuccess) return e;
    // timed solves: the same kernels and work items, launched one by one
    Phase ph[kMaxPhases];
    const int nph = phases_of(k, ph);
    const int2* items[kMaxPhases];
    int nitems[kMaxPhases];
    std::vector<cudaEvent_t> tev;
    const int per_chunk = nph * kChunk;
    if (timing) {
        for (int j = 0; j < nph; ++j) {
            if ((e = items_for(w, ph[j].width, a.tpi, &items[j], &nitems[j])) != cudaSuccess) return e;
            if (ph[j].list) nitems[j] = kListBlocksPerSm * w.num_sms;
        }
        for (int r = 0; r < kTimedPhases; ++r) {
            timing->ms[r] = 0.0;
            timing->n[r] = 0;
        }
        tev.resize(2 * (per_chunk + 1));
        for (cudaEvent_t& ev : tev)
            if ((e = cudaEventCreate(&ev)) != cudaSuccess) return e;
    }
    auto destroy_events = [&]() {
        for (cudaEvent_t ev : tev)
            if (ev) cudaEventDestroy(ev);
        tev.clear();
    };
    auto accumulate = [&](int pool) {  // a finished chunk's per-kernel times
        cudaEvent_t* ev = tev.data() + pool * (per_chunk + 1);
        for (int j = 0; j < per_chunk; ++j) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[j], ev[j + 1]);
            const int r = ph[j % nph].slot;
            timing->ms[r] += ms;
            timing->n[r] += 1;
        }
    };
    const int max_chunks = a.maxloop / kChunk + 2;
    // keep one chunk queued ahead of the convergence check
    for (int c = 0; c < max_chunks; ++c) {
        if (timing) {
            cudaEvent_t* ev = tev.data() + (c & 1) * (per_chunk + 1);
            if ((e = cudaEventRecord(ev[0], stream)) != cudaSuccess) { destroy_events(); return e; }
            for (int it = 0; it < kChunk; ++it)
                for (int j = 0; j < nph; ++j) {
                    ph[j].fn<<<phase_grid(ph[j], nitems[j]), kTile, ph[j].smem, stream>>>(a, items[j], it & 1);
                    if ((e = cudaEventRecord(ev[nph * it + j + 1], stream)) != cudaSuccess) {
                        destroy_events();
                        return e;
                    }
                }
        } else if ((e = cudaGraphLaunch(w.exec, stream)) != cudaSuccess) {
            return e;
        }
        w.launches += per_chunk;
        if ((e = cudaMemcpyAsync(&w.h_active[c & 1], w.d_active, sizeof(int), cudaMemcpyDeviceToHost, stream)) !=
            cudaSuccess)
            return e;
        if ((e = cudaEventRecord(w.ev[c & 1], stream)) != cudaSuccess) return e;
        if (c >= 1) {
            if ((e = cudaEventSynchronize(w.ev[(c - 1) & 1])) != cudaSuccess) { destroy_events(); return e; }
            if (timing) accumulate((c - 1) & 1);
            if (w.h_active[(c - 1) & 1] <= 0) {
                if (timing) {  // the chunk queued ahead ran as well
                    if ((e = cudaEventSynchronize(w.ev[c & 1])) != cudaSuccess) { destroy_events(); return e; }
                    accumulate(c & 1);
                }
                break;
            }
        }
    }
    destroy_events();
    int err = 0;
    if (k.nst &&
        (e = cudaMemcpyAsync(&err, &w.d_bar->err, sizeof(int), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
        return e;
    if ((e = finish_solve(w, stream)) != cudaSuccess) return e;
    w.timed_out = err != 0;  // a staging wait gave up: the solve reports SFH_ERR_TIMEOUT
    return cudaSuccess;
}

// the lanes' final state to the host; a lane that never stopped did not
// converge
static cudaError_t finish_solve(CgWorkspace& w, cudaStream_t stream)
{
    cudaError_t e = cudaMemcpyAsync(w.lanes_h.data(), w.d_lanes, sizeof(CgLane) * w.nlanes, cudaMemcpyDeviceToHost,
                                    stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    // a lane that stopped holds DONE or FAILED in one of its two mode slots
    for (CgLane& L : w.lanes_h) {
        bool stopped = false;
        for (int k = 0; k < 2; ++k) stopped |= L.mode[k] == LM_DONE || L.mode[k] == LM_FAILED;
        if (!stopped) {
            L.status = SFH_ERR_NOCONV;
            L.mode[0] = L.mode[1] = LM_FAILED;
        }
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
    int prec = 0, flags = 0, nb = 0, nb2 = 0, tpi = 0, stage_links = 0;
    double delta = 0.1;  // reliable-update threshold of the mixed precisions (set at creation)
    std::vector<sfh_system_desc> desc;
    std::vector<sfh::Geom> geoms;
    std::vector<void*> U64, U32, U16;  // U16: the FP16 or BF16 links of a 16-bit batch
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

// derived reduced-precision links of system k (U32 holds the 18-real FP32
// field for SFH_PREC_F32_18)
static void batch_make_lowp(sfh_batch* b, int k)
{
    if (b->prec == SFH_PREC_F64) return;
    if (b->prec == SFH_PREC_F32_18)
        sfh::launch_make_lowp_gauge(b->geoms[k], b->U64[k], nullptr, nullptr, b->stream, b->U32[k]);
    else if (b->prec == SFH_PREC_BF16)
        sfh::launch_make_lowp_gauge(b->geoms[k], b->U64[k], nullptr, nullptr, b->stream, nullptr, b->U16[k]);
    else
        sfh::launch_make_lowp_gauge(b->geoms[k], b->U64[k], b->U32[k], b->U16[k], b->stream);
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
    if (!sfh::valid_precision(precision)) return SFH_ERR_INVALID;
    if ((flags & SFH_BATCH_FULL_LATTICE) && precision != SFH_PREC_F64) return SFH_ERR_INVALID;
    for (int k = 0; k < nsys; ++k)
        if (!sfh::dims_ok(systems[k].dims) || systems[k].nrhs <= 0 || systems[k].nrhs > 64)
            return SFH_ERR_INVALID;
    if (nsys >= (1 << (31 - sfh::kItemSysShift))) return SFH_ERR_INVALID;  // the work items' system field
    *out = nullptr;
    sfh_batch* b = new sfh_batch();
    b->device = device;
    b->prec = precision;
    b->flags = flags;
    // FP16 vectors track a drop of about 10x before they lose accuracy; FP32
    // ones a drop of 100x (fewer FP64 updates, same iterations: measured)
    b->delta = sfh::default_reliable_delta(precision);
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
        if (e == cudaSuccess && (precision == SFH_PREC_F16 || precision == SFH_PREC_BF16))
            e = cudaMalloc(&u16, (size_t)g.V * 4 * 3 * 8);
        if (e == cudaSuccess && precision == SFH_PREC_F32_18) e = cudaMalloc(&u32, (size_t)g.V * 4 * 9 * 8);
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
        h.Ulo = (precision == SFH_PREC_F32 || precision == SFH_PREC_F32_18)
                    ? b->U32[k]
                    : ((precision == SFH_PREC_F16 || precision == SFH_PREC_BF16) ? b->U16[k] : b->U64[k]);
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
    b->nb2 = width;
    return SFH_OK;
}

extern "C" int sfh_batch_set_hop_widths(sfh_batch* b, int hop1_width, int hop2_width)
{
    if (!b || hop1_width < 0 || hop1_width > 8 || hop2_width < 0 || hop2_width > 8) return SFH_ERR_INVALID;
    b->nb = hop1_width;
    b->nb2 = hop2_width;
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
        batch_make_lowp(b, k);
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
    int st = batch_cuda(b, sfh::workspace_solve(b->ws, tol, maxit, b->delta, b->nb, b->nb2, b->tpi, b->stage_links, b->stream),
                        "batched CG");
    if (st) return st;
    if (b->ws.timed_out)
        return batch_err(b, SFH_ERR_TIMEOUT, "batched CG: a bounded device wait (grid barrier or neighbour staging) gave up");
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
        rr += L.rr_next;
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
    for (const sfh::CgLane& L : b->ws.lanes_h)  // the RHS's own mass, if it has one
        if (L.rhs == b->ws.rhs0[k] + j) m = std::sqrt(L.m2);
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
// device-resident single-context solve with a cached workspace (used by the
// trajectory), and the host-pointer solve built on it
// ===========================================================================
namespace sfh {

void workspace_free(CgWorkspace* w) { delete w; }

static CgWorkspace* ctx_workspace(sfh_ctx* c, int prec, cudaError_t* err)
{
    *err = cudaSuccess;
    if (!valid_precision(prec)) {
        *err = cudaErrorInvalidValue;
        return nullptr;
    }
    if (c->ws[prec]) return c->ws[prec];
    CgWorkspace* w = new CgWorkspace();
    SolverSystemHost h;
    h.g = c->g;
    h.mass = c->mass;
    h.nrhs = 1;
    h.U64 = c->U64;
    const void* const lo[5] = {c->U64, c->U32, c->U16, c->U32_18, c->Ubf16};
    h.Ulo = lo[prec];
    std::vector<SolverSystemHost> hs(1, h);
    *err = workspace_build(*w, hs, prec, prec == SFH_PREC_F64 ? 1 : 0);
    if (*err != cudaSuccess) {
        delete w;
        return nullptr;
    }
    c->ws[prec] = w;
    c->ws_mass[prec] = c->mass;
    return w;
}

int ctx_solve_device(sfh_ctx* c, const void* b_eo, void* x_eo, double tol, int maxit, int prec,
                     sfh_cg_info* info)
{
    if (prec != SFH_PREC_F64 && !c->lowp_valid) {
        launch_make_lowp_gauge(c->g, c->U64, c->U32, c->U16, c->stream, c->U32_18, c->Ubf16);
        c->lowp_valid = true;
    }
    cudaError_t e;
    CgWorkspace* w = ctx_workspace(c, prec, &e);
    if (!w) return cuda_check(c, e, "cg workspace");
    if (c->ws_mass[prec] != c->mass) {  // the mass lives in the device system table
        w->sys[0].m2 = c->mass * c->mass;
        for (CgLane& L : w->lanes_h) L.m2 = w->sys[0].m2;  // uploaded with the lanes at the solve
        e = cudaMemcpyAsync(w->d_sys, w->sys.data(), sizeof(CgSys), cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) return cuda_check(c, e, "cg mass");
        c->ws_mass[prec] = c->mass;
    }
    size_t fs = (size_t)c->g.V * 6 * sizeof(double);
    e = cudaMemcpyAsync(w->rhs[0].b, b_eo, fs, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "cg rhs");
    const bool lowp = prec != SFH_PREC_F64;  // the FP64 CG keeps the reference's schedule
    e = workspace_solve(*w, tol, maxit, default_reliable_delta(prec), lowp ? c->sched_nb : 0, lowp ? c->sched_nb : 0,
                        lowp ? c->sched_tpi : 0, lowp ? c->sched_stage : 0, c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "cg solve");
    if (w->timed_out) return set_error(c, SFH_ERR_TIMEOUT, "CG: a bounded device wait (grid barrier or neighbour staging) gave up");
    e = cudaMemcpyAsync(x_eo, w->rhs[0].xhi, fs, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "cg solution");
    int status = SFH_OK;
    sfh_cg_info inf;
    std::memset(&inf, 0, sizeof(inf));
    double rr = 0, bb = 0;
    for (const CgLane& L : w->lanes_h) {
        if (L.status != SFH_OK && status == SFH_OK) status = L.status;
        inf.iters = std::max(inf.iters, L.iters);
        if (L.parity < 2) inf.iters_parity[L.parity] = L.iters;
        else inf.iters_parity[0] = inf.iters_parity[1] = L.iters;
        inf.reliable_updates += L.nru;
        rr += L.rr_next;
        bb += L.bb;
    }
    inf.status = status;
    inf.rsq_rel = bb > 0 ? rr / bb : 0.0;
    inf.true_resid = -1.0;
    if (info) *info = inf;
    if (status != SFH_OK)
        return set_error(c, status, status == SFH_ERR_NOCONV ? "CG Solver failed to converge" : "CG breakdown");
    return SFH_OK;
}

// Two solves on the context's links at two masses (a Hasenbusch pair) as one
// system with two right-hand sides, each lane carrying its own mass, in one
// sequence of launches; the heavy mass's lanes retire first.  FP64 runs
// full-lattice lanes (the reference's CG), as ctx_solve_device does, with
// both RHS in each work item (a link read once serves both masses).
int ctx_solve_pair_device(sfh_ctx* c, const void* const b_eo[2], void* const x_eo[2], const double mass[2],
                          double tol, int maxit, int prec, sfh_cg_info info[2])
{
    if (!valid_precision(prec)) return set_error(c, SFH_ERR_INVALID, "precision");
    if (prec != SFH_PREC_F64 && !c->lowp_valid) {
        launch_make_lowp_gauge(c->g, c->U64, c->U32, c->U16, c->stream, c->U32_18, c->Ubf16);
        c->lowp_valid = true;
    }
    cudaError_t e = cudaSuccess;
    CgWorkspace* w = c->ws_pair[prec];
    if (!w) {
        w = new CgWorkspace();
        const void* const lo[5] = {c->U64, c->U32, c->U16, c->U32_18, c->Ubf16};
        std::vector<SolverSystemHost> hs(1);
        hs[0].g = c->g;
        hs[0].mass = mass[0];
        hs[0].nrhs = 2;
        hs[0].U64 = c->U64;
        hs[0].Ulo = lo[prec];
        e = workspace_build(*w, hs, prec, prec == SFH_PREC_F64 ? 1 : 0);
        if (e != cudaSuccess) {
            delete w;
            return cuda_check(c, e, "cg pair workspace");
        }
        c->ws_pair[prec] = w;
        c->ws_pair_mass[prec][0] = c->ws_pair_mass[prec][1] = -1.0;  // set below
    }
    if (c->ws_pair_mass[prec][0] != mass[0] || c->ws_pair_mass[prec][1] != mass[1]) {
        for (CgLane& L : w->lanes_h) L.m2 = mass[L.rhs] * mass[L.rhs];  // uploaded with the lanes
        c->ws_pair_mass[prec][0] = mass[0];
        c->ws_pair_mass[prec][1] = mass[1];
    }
    const size_t fs = (size_t)c->g.V * 6 * sizeof(double);
    for (int k = 0; k < 2; ++k) {
        e = cudaMemcpyAsync(w->rhs[k].b, b_eo[k], fs, cudaMemcpyDeviceToDevice, c->stream);
        if (e != cudaSuccess) return cuda_check(c, e, "cg pair rhs");
    }
    // the mixed precisions take one RHS per work item unless the context's
    // schedule says otherwise: the heavy mass retires after a fifth of the
    // light one's iterations, and a two-RHS item with one lane left runs its
    // hops slower than a one-RHS item (24^4, FP32 storage: 62.2 ms for the
    // pair at width 1 against 74.4 ms at width 2 and 64.5 ms for two solves)
    const bool lowp = prec != SFH_PREC_F64;
    const int nb = lowp ? (c->sched_nb > 0 ? c->sched_nb : 1) : 0;
    e = workspace_solve(*w, tol, maxit, default_reliable_delta(prec), nb, nb, lowp ? c->sched_tpi : 0,
                        lowp ? c->sched_stage : 0, c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "cg pair solve");
    if (w->timed_out) return set_error(c, SFH_ERR_TIMEOUT, "CG: a bounded device wait (grid barrier or neighbour staging) gave up");
    for (int k = 0; k < 2; ++k) {
        e = cudaMemcpyAsync(x_eo[k], w->rhs[k].xhi, fs, cudaMemcpyDeviceToDevice, c->stream);
        if (e != cudaSuccess) return cuda_check(c, e, "cg pair solution");
    }
    int status = SFH_OK;
    for (int k = 0; k < 2; ++k) {
        sfh_cg_info inf;
        std::memset(&inf, 0, sizeof(inf));
        double rr = 0, bb = 0;
        for (const CgLane& L : w->lanes_h) {
            if (L.rhs != k) continue;
            if (L.status != SFH_OK && inf.status == SFH_OK) inf.status = L.status;
            inf.iters = std::max(inf.iters, L.iters);
            if (L.parity < 2) inf.iters_parity[L.parity] = L.iters;
            else inf.iters_parity[0] = inf.iters_parity[1] = L.iters;
            inf.reliable_updates += L.nru;
            rr += L.rr_next;
            bb += L.bb;
        }
        inf.rsq_rel = bb > 0 ? rr / bb : 0.0;
        inf.true_resid = -1.0;
        if (inf.status != SFH_OK && status == SFH_OK) status = inf.status;
        if (info) info[k] = inf;
    }
    if (status != SFH_OK)
        return set_error(c, status, status == SFH_ERR_NOCONV ? "CG Solver failed to converge" : "CG breakdown");
    return SFH_OK;
}

}  // namespace sfh

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
    size_t fs = (size_t)c->g.V * 6 * sizeof(double);
    cudaError_t e = cudaMemcpyAsync(c->stage, phi, fs, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "cg upload");
    launch_spinor_aos_to_eo(c->g, (const double*)c->stage, c->spin[3], c->stream);
    int st = ctx_solve_device(c, c->spin[3], c->spin[4], tol, maxit, prec, info);
    if (st != SFH_OK && st != SFH_ERR_NOCONV && st != SFH_ERR_BREAKDOWN) return st;
    launch_spinor_eo_to_aos(c->g, c->spin[4], (double*)c->stage, c->stream);
    e = cudaMemcpyAsync(X, c->stage, fs, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "cg download");
    return st;
}

extern "C" int sfh_batch_random_gauge(sfh_batch* b, int k, double eps, unsigned long long seed)
{
    if (!b || k < 0 || k >= (int)b->desc.size()) return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    const sfh::Geom& g = b->geoms[k];
    int st = batch_cuda(b, sfh::launch_random_gauge(g, eps, seed, b->U64[k], b->derr, b->stream), "random gauge");
    if (st) return st;
    batch_make_lowp(b, k);
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

extern "C" int sfh_batch_solve_timed(sfh_batch* b, double tol, int maxit, double* ms, long* n)
{
    if (!b || !ms || !n || !(tol > 0.0) || maxit <= 0) return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    sfh::PhaseTimes t;
    int st = batch_cuda(b, sfh::workspace_solve(b->ws, tol, maxit, b->delta, b->nb, b->nb2, b->tpi, b->stage_links, b->stream, &t),
                        "timed batched CG");
    if (st) return st;
    if (b->ws.timed_out)
        return batch_err(b, SFH_ERR_TIMEOUT, "batched CG: a bounded device wait (grid barrier or neighbour staging) gave up");
    static_assert(sfh::kTimedPhases == SFH_TIMED_KERNELS, "timing slots of include/sfh.h");
    for (int k = 0; k < sfh::kTimedPhases; ++k) {
        ms[k] = t.ms[k];
        n[k] = t.n[k];
    }
    for (const sfh::CgLane& L : b->ws.lanes_h)
        if (L.status != SFH_OK) return L.status;
    return SFH_OK;
}

extern "C" int sfh_batch_kernel_launches(sfh_batch* b, long* n)
{
    if (!b || !n) return SFH_ERR_INVALID;
    *n = b->ws.launches;
    return SFH_OK;
}

// Autotuner: times a capped solve (probe_iters iterations, no lane converges)
// for every RHS-block width, tiles-per-block count and link staging mode
// (read directly, staged per work item, system-blocked) and keeps the
// fastest.
extern "C" int sfh_batch_autotune(sfh_batch* b, int probe_iters, int* best_width)
{
    if (!b || probe_iters < 1) return SFH_ERR_INVALID;
    cudaSetDevice(b->device);
    const int widths64[] = {1, 2};
    const int widths[] = {1, 2, 4, 8};
    const int tiles[] = {1, 2, 4};
    const bool f64 = b->prec == SFH_PREC_F64;
    const int* cand = f64 ? widths64 : widths;
    const int ncand = f64 ? 2 : 4;
    double best = 1e300;
    int bw = 1, bw2 = 1, bt = 2, bs = 0;
    for (int stage = 0; stage < (f64 ? 1 : 8); ++stage)
        for (int c = 0; c < ncand + 1; ++c)
            for (int tp : tiles) {
                if (stage == 6 && b->prec != SFH_PREC_F16) continue;  // schedule 4 there
                if ((stage == 2 || stage == 3) && (tp != 1 || b->prec == SFH_PREC_F32_18))
                    continue;  // system-blocked: one tile per block; not for FP32 18-real links
                // the last candidate: the first hop in groups of four, the
                // second in groups of two (lane-list stages only)
                const bool split = c == ncand;
                if (split && (f64 || stage < 4)) continue;
                const int w1 = split ? 4 : cand[c], w2 = split ? 2 : cand[c];
                double t = 0.0;
                for (int rep = 0; rep < 2; ++rep) {  // the first run builds the graph
                    auto t0 = std::chrono::steady_clock::now();
                    cudaError_t e = sfh::workspace_solve(b->ws, 1e-30, probe_iters, 0.1, w1, w2, tp, stage, b->stream);
                    if (e != cudaSuccess) return batch_cuda(b, e, "autotune");
                    t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                }
                if (t < best) {
                    best = t;
                    bw = w1;
                    bw2 = w2;
                    bt = tp;
                    bs = stage;
                }
            }
    b->nb = bw;
    b->nb2 = bw2;
    b->tpi = bt;
    b->stage_links = bs;
    if (best_width) *best_width = bw;
    return SFH_OK;
}

extern "C" int sfh_batch_set_schedule(sfh_batch* b, int width, int tiles_per_block, int stage_links)
{
    if (!b || width < 0 || tiles_per_block < 0 || tiles_per_block > 64) return SFH_ERR_INVALID;
    b->nb = b->nb2 = width;
    b->tpi = tiles_per_block;
    if (stage_links < 0 || stage_links > 7) return SFH_ERR_INVALID;
    b->stage_links = stage_links;
    return SFH_OK;
}

extern "C" int sfh_set_schedule(sfh_ctx* c, int width, int tiles_per_block, int stage_links)
{
    if (!c || width < 0 || width > 8 || tiles_per_block < 0 || tiles_per_block > 64 || stage_links < 0 ||
        stage_links > 7)
        return SFH_ERR_INVALID;
    c->sched_nb = width;
    c->sched_tpi = tiles_per_block;
    c->sched_stage = stage_links;
    return SFH_OK;
}

extern "C" int sfh_batch_set_rhs_mass(sfh_batch* b, int k, int j, double mass)
{
    if (!b || k < 0 || k >= (int)b->desc.size() || j < 0 || j >= b->desc[k].nrhs || !(mass >= 0.0))
        return SFH_ERR_INVALID;
    const int rid = b->ws.rhs0[k] + j;
    for (sfh::CgLane& L : b->ws.lanes_h)  // uploaded with the lanes at the next solve
        if (L.rhs == rid) L.m2 = mass * mass;
    return SFH_OK;
}

extern "C" int sfh_batch_set_barrier_polls(sfh_batch* b, long long polls)
{
    if (!b || polls < 0) return SFH_ERR_INVALID;
    b->ws.barrier_polls = polls;
    return SFH_OK;
}

extern "C" int sfh_batch_set_reliable_delta(sfh_batch* b, double delta)
{
    if (!b || !(delta > 0.0) || !(delta < 1.0)) return SFH_ERR_INVALID;
    b->delta = delta;
    return SFH_OK;
}

extern "C" int sfh_batch_get_hop_widths(sfh_batch* b, int* hop1_width, int* hop2_width)
{
    if (!b) return SFH_ERR_INVALID;
    if (hop1_width) *hop1_width = b->nb;
    if (hop2_width) *hop2_width = b->nb2;
    return SFH_OK;
}

extern "C" int sfh_batch_get_schedule(sfh_batch* b, int* width, int* tiles_per_block, int* stage_links)
{
    if (!b) return SFH_ERR_INVALID;
    if (width) *width = b->nb;
    if (tiles_per_block) *tiles_per_block = b->tpi;
    if (stage_links) *stage_links = b->stage_links;
    return SFH_OK;
}

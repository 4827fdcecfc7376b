// gauge.cu — link-field kernels of the HMC: Symanzik gauge force, fermion
// force, momentum kick, link update U <- exp(i eps P) U, and the FP64
// reductions Tr P^2, gauge action, plaquette and Re<phi, X>.
//
// Fields are FP64 in the even-odd SoA layout of sfh_core.cuh.  One thread per
// link (parity p, direction mu, checkerboard site i).  Staples are products of
// links along lattice paths (periodic in every direction for gauge links,
// Lattice.cpp:213-235); the paths are those of compute_staple_sum_at_link
// (Lattice.cpp:249-313) and compute_rectangle_staple_sum_at_link
// (Lattice.cpp:315-499), each written as the walk from x+mu back to x so that
// U_mu(x) * staple is a closed loop.
#include "sfh_internal.h"
#include "su3.cuh"
#include "walk.cuh"

namespace sfh {

namespace {

constexpr int kThreads = 128;

// product of links along a path; step s > 0 walks +(s-1), s < 0 walks -(-s-1)
template <int N>
__device__ __forceinline__ M3 path(const void* U, const Geom& g, Walker w, const int (&steps)[N])
{
    M3 m = m3_id();
#pragma unroll
    for (int k = 0; k < N; ++k) {
        int s = steps[k];
        int mu = (s > 0 ? s : -s) - 1;
        if (s > 0) {
            m = m3_mul(m, link_at(U, g, w, mu));
            walk(g, w, mu, +1);
        } else {
            walk(g, w, mu, -1);
            m = m3_mul_adj(m, link_at(U, g, w, mu));
        }
    }
    return m;
}

// A1 (plaquette staples) and A2 (rectangle staples) of link (x, mu); RECT
// false: A1 alone (the same paths in the same order, A2 left zero)
template <bool RECT = true>
__device__ void staples(const void* U, const Geom& g, const Walker& x, int mu, M3& A1, M3& A2)
{
    Walker xp = x;
    walk(g, xp, mu, +1);
    const int M = mu + 1;
    A1 = m3_zero();
    A2 = m3_zero();
#pragma unroll 1
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        const int N = nu + 1;
        const int top[3] = {+N, -M, -N};
        const int bot[3] = {-N, -M, +N};
        m3_acc(A1, path(U, g, xp, top));
        m3_acc(A1, path(U, g, xp, bot));
        if constexpr (!RECT) continue;
        const int r1[5] = {-N, -N, -M, +N, +N};
        const int r2[5] = {+N, +N, -M, -N, -N};
        const int r3[5] = {+M, -N, -M, -M, +N};
        const int r4[5] = {+N, -M, -M, -N, +M};
        const int r5[5] = {-N, -M, -M, +N, +M};
        const int r6[5] = {+M, +N, -M, -M, -N};
        m3_acc(A2, path(U, g, xp, r1));
        m3_acc(A2, path(U, g, xp, r2));
        m3_acc(A2, path(U, g, xp, r3));
        m3_acc(A2, path(U, g, xp, r4));
        m3_acc(A2, path(U, g, xp, r5));
        m3_acc(A2, path(U, g, xp, r6));
    }
}

// F = -i f (Q - Q^dag), trace removed
__device__ __forceinline__ M3 antiherm_force(const M3& Q, double f)
{
    M3 F;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Cx<double> d = csub(Q.e[i * 3 + j], cconj(Q.e[j * 3 + i]));
            F.e[i * 3 + j] = {f * d.im, -f * d.re};  // -i f d
        }
    m3_traceless(F);
    return F;
}

// Fermions.cpp:372-384: F_g = -i (beta/12) (U V - (U V)^dag), V = c11 A1 + c12 A2
__device__ __forceinline__ M3 gauge_force_link(const void* U, const Geom& g, const Walker& x, int mu, double beta,
                                               double c11, double c12)
{
    M3 A1, A2;
    staples(U, g, x, mu, A1, A2);
    M3 Vs;
#pragma unroll
    for (int k = 0; k < 9; ++k)
        Vs.e[k] = {c11 * A1.e[k].re + c12 * A2.e[k].re, c11 * A1.e[k].im + c12 * A2.e[k].im};
    M3 Q = m3_mul(link_at(U, g, x, mu), Vs);
    return antiherm_force(Q, beta / 12.0);
}

__device__ __forceinline__ Vec3<double> spinor_at(const void* f, const Geom& g, const Walker& w)
{
    int par = (w.x[0] + w.x[1] + w.x[2] + w.x[3]) & 1;
    int i = lex_of(g, w) >> 1;
    const double2* b = (const double2*)f + (size_t)par * 3 * g.Vh + i;
    Vec3<double> v;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double2 t = __ldg(b + (size_t)c * g.Vh);
        v.c[c] = {t.x, t.y};
    }
    return v;
}

// Fermions.cpp:443-515: c = eta bc / 4, A_f = (U Y(x+mu)) X(x)^dag,
// A_b = Y(x) X(x+mu)^dag U^dag, F = -i c [(A_f - A_f^dag) + (A_b - A_b^dag)]
__device__ __forceinline__ M3 fermion_force_link(const void* U, const void* X, const void* Y, const Geom& g,
                                                 const Walker& x, int mu)
{
    Walker xu = x;
    walk(g, xu, mu, +1);
    int eta = 0;
    for (int nu = 0; nu < mu; ++nu) eta += x.x[nu];
    double c = 0.25 * ((eta & 1) ? -1.0 : 1.0) * ((mu == 3 && x.x[3] == g.L[3] - 1) ? -1.0 : 1.0);
    M3 Ux = link_at(U, g, x, mu);
    Vec3<double> Xx = spinor_at(X, g, x), Xu = spinor_at(X, g, xu);
    Vec3<double> Yx = spinor_at(Y, g, x), Yu = spinor_at(Y, g, xu);
    Vec3<double> uy = mul_mv(Ux, Yu);
    M3 Af, T;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Af.e[i * 3 + j] = cmul(uy.c[i], cconj(Xx.c[j]));
            T.e[i * 3 + j] = cmul(Yx.c[i], cconj(Xu.c[j]));
        }
    M3 Ab = m3_mul_adj(T, Ux);
    M3 S;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            S.e[i * 3 + j] = cadd(csub(Af.e[i * 3 + j], cconj(Af.e[j * 3 + i])),
                                  csub(Ab.e[i * 3 + j], cconj(Ab.e[j * 3 + i])));
    M3 F;
#pragma unroll
    for (int k = 0; k < 9; ++k) F.e[k] = {c * S.e[k].im, -c * S.e[k].re};  // -i c S
    m3_traceless(F);
    return F;
}

// what: bit 0 gauge force, bit 1 fermion force.  out = F (kick == 0, out = F)
// or P -= kick * F (mom != nullptr).
__global__ void __launch_bounds__(kThreads) force_kernel(Geom g, const void* U, const void* X, const void* Y,
                                                         double beta, double c11, double c12, int what,
                                                         void* out, void* mom, double kick)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    Walker x = link_coords(g, p, i);
    M3 F = m3_zero();
    if (what & 1) F = gauge_force_link(U, g, x, mu, beta, c11, c12);
    if (what & 2) m3_acc(F, fermion_force_link(U, X, Y, g, x, mu));
    if (mom) {
        M3 P = ld_link(mom, p, mu, i, g.Vh);
        m3_axpy(P, -kick, F);
        st_link(mom, p, mu, i, g.Vh, P);
    } else {
        st_link(out, p, mu, i, g.Vh, F);
    }
}

__global__ void __launch_bounds__(kThreads) staple_kernel(Geom g, const void* U, void* A1out, void* A2out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    Walker x = link_coords(g, p, i);
    M3 A1, A2;
    staples(U, g, x, mu, A1, A2);
    st_link(A1out, p, mu, i, g.Vh, A1);
    st_link(A2out, p, mu, i, g.Vh, A2);
}

// Fermions.cpp:699-723, 984-994: U <- exp(i eps P) U.  check: the production
// path of the reference rejects P_pre with |P-P^dag| > 1e-10 or |tr P| > 1e-10.
__global__ void link_update_kernel(Geom g, void* U, const void* P, double eps, int check, int* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    M3 Q = ld_link(P, p, mu, i, g.Vh);
#pragma unroll
    for (int k = 0; k < 9; ++k) Q.e[k] = cscale(Q.e[k], eps);
    if (check) {
        double n2 = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                Cx<double> d = csub(Q.e[a * 3 + b], cconj(Q.e[b * 3 + a]));
                n2 += d.re * d.re + d.im * d.im;
            }
        Cx<double> t = m3_tr(Q);
        if (sqrt(n2) > 1e-10 || sqrt(t.re * t.re + t.im * t.im) > 1e-10) {
            atomicOr(err, DEV_ERR_NOT_HERMITIAN);
            return;
        }
    }
    M3 E;
    if (!expiq(Q, E)) {
        atomicOr(err, DEV_ERR_DOMAIN);
        return;
    }
    M3 Uo = ld_link(U, p, mu, i, g.Vh);
    st_link(U, p, mu, i, g.Vh, m3_mul(E, Uo));
}

// ---------------------------------------------------------------------------
// deterministic FP64 reductions: fixed grid, per-block partials, one final
// block summing the partials in order
// ---------------------------------------------------------------------------
constexpr int kRedBlocks = 1024;
constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_reduce(double v, double* sm)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;
}

// per link: Re Tr P^2 (Fermions.cpp:662-678); gauge action density
// -(beta/3)(c11 ReTr(U A1)/4 + c12 ReTr(U A2)/6) (Lattice.cpp:759-781);
// ReTr(U A1)/3 (Lattice.cpp:784-804).  RED_DOT: Re<a, b> over spinors.
__global__ void __launch_bounds__(kRedThreads) reduce_kernel(Geom g, int kind, const void* A, const void* B,
                                                             double beta, double c11, double c12, double* partial)
{
    __shared__ double sm[32];
    double acc = 0.0;
    const long nlinks = 4L * g.V;
    if (kind == RED_DOT) {
        const double* a = (const double*)A;
        const double* b = (const double*)B;
        const long n = 6L * g.V;
        for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
            acc += a[k] * b[k];
    } else {
        for (long l = blockIdx.x * (long)blockDim.x + threadIdx.x; l < nlinks; l += (long)gridDim.x * blockDim.x) {
            int pm = (int)(l / g.Vh);
            int i = (int)(l - (long)pm * g.Vh);
            int p = pm >> 2, mu = pm & 3;
            if (kind == RED_TRP2) {
                M3 P = ld_link(A, p, mu, i, g.Vh);
                acc += m3_tr(m3_mul(P, P)).re;
            } else {
                Walker x = link_coords(g, p, i);
                M3 A1, A2;
                if (kind == RED_PLAQ)
                    staples<false>(A, g, x, mu, A1, A2);  // the plaquette staples only
                else
                    staples(A, g, x, mu, A1, A2);
                M3 Ux = link_at(A, g, x, mu);
                double plaq = m3_tr(m3_mul(Ux, A1)).re;
                if (kind == RED_PLAQ) {
                    acc += plaq / 3.0;
                } else {
                    double rect = m3_tr(m3_mul(Ux, A2)).re;
                    acc += -(beta / 3.0) * (c11 * plaq / 4.0 + c12 * rect / 6.0);
                }
            }
        }
    }
    double r = block_reduce(acc, sm);
    if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

__global__ void reduce_final(const double* partial, int n, double* out)
{
    __shared__ double sm[32];
    double acc = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) acc += partial[k];
    double r = block_reduce(acc, sm);
    if (threadIdx.x == 0) *out = r;
}

}  // namespace

cudaError_t launch_force(const Geom& g, const void* U, const void* X, const void* Y, double beta, double c11,
                         double c12, int what, void* out, void* mom, double kick, cudaStream_t s)
{
    force_kernel<<<dim3((g.Vh + kThreads - 1) / kThreads, 8), kThreads, 0, s>>>(g, U, X, Y, beta, c11, c12, what,
                                                                                 out, mom, kick);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Heatbath (single_link_heatbath, Lattice.cpp:722-757, with the SU(2)
// sampler of SU3_Sampling.cpp:17-199).  Per link: A = c11 A1 + c12 A2; for
// the subgroups R (0,1), S (0,2), T (1,2): W = the SU(2) projection of that
// block of U A, a = sqrt(det W); a <= 1e-14: a uniform SU(2) element, else X
// drawn with (a, 2 beta / 3) and R = X (W / a)^dag; U <- R U.  One launch
// updates one direction and one colour (x_mu mod 2) * 4 + (sum_{nu != mu} x_nu
// mod 4): links whose staples do not contain each other.  Uniforms: Philox-
// 4x32-10 keyed by the seed, counter (link, draw, sweep, 0x48420000 + subgroup).
// ---------------------------------------------------------------------------
struct HbRng {
    uint2 key;
    unsigned link, sweep, tag, draw;
    double buf[2];
    int have;
    __device__ double u()  // uniform in [0, 1)
    {
        if (have == 0) {
            uint4 r = Philox::gen(make_uint4(link, draw++, sweep, tag), key);
            unsigned long long a = (((unsigned long long)r.x << 21) ^ (unsigned long long)(r.y >> 11)) & ((1ull << 53) - 1);
            unsigned long long b = (((unsigned long long)r.z << 21) ^ (unsigned long long)(r.w >> 11)) & ((1ull << 53) - 1);
            buf[0] = (double)a * (1.0 / 9007199254740992.0);
            buf[1] = (double)b * (1.0 / 9007199254740992.0);
            have = 2;
        }
        return buf[2 - have--];
    }
};

// generate_x0 (SU3_Sampling.cpp:17-31)
__device__ double hb_x0(HbRng& r, double a, double beta)
{
    for (;;) {
        double r1 = 1.0 - r.u(), r2 = 1.0 - r.u(), r3 = 1.0 - r.u();
        double c = cospi(2.0 * r2);
        double l2 = -1.0 / (2.0 * a * beta) * (log(r1) + c * c * log(r3));
        double x = 1.0 - l2;
        double rr = r.u();
        if (rr * rr <= x && x >= -1.0 && x <= 1.0) return 1.0 - 2.0 * l2;
    }
}

template <int N>
__device__ void hb_unit(HbRng& r, double (&v)[N])
{
    for (;;) {
        double len2 = 0.0;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            v[k] = 2.0 * r.u() - 1.0;
            len2 += v[k] * v[k];
        }
        double len = sqrt(len2);
        if (len <= 1.0 && len > 0.0) {
#pragma unroll
            for (int k = 0; k < N; ++k) v[k] /= len;
            return;
        }
    }
}

// q0 I + i (q1 sx + q2 sy + q3 sz), row-major 2x2
__device__ __forceinline__ void quat_su2(const double (&q)[4], Cx<double> (&m)[4])
{
    m[0] = {q[0], q[3]};
    m[1] = {q[2], q[1]};
    m[2] = {-q[2], q[1]};
    m[3] = {q[0], -q[3]};
}

__device__ void hb_subgroup(HbRng& r, M3& U, const M3& A, int i, int j, double beta)
{
    const M3 UA = m3_mul(U, A);
    const Cx<double> b0 = UA.e[i * 3 + i], b1 = UA.e[i * 3 + j], b2 = UA.e[j * 3 + i], b3 = UA.e[j * 3 + j];
    const double w0 = 0.5 * (b0.re + b3.re), w1 = 0.5 * (b1.im + b2.im);
    const double w2 = 0.5 * (b1.re - b2.re), w3 = 0.5 * (b0.im - b3.im);
    const double a = sqrt(w0 * w0 + w1 * w1 + w2 * w2 + w3 * w3);
    Cx<double> R[4];
    if (a <= 1e-14) {
        double q[4];
        hb_unit<4>(r, q);
        quat_su2(q, R);
    } else {
        const double x0 = hb_x0(r, a, 2.0 * beta / 3.0);
        double v[3];
        hb_unit<3>(r, v);
        const double nx = sqrt(1.0 - x0 * x0);
        const double qx[4] = {x0, nx * v[0], nx * v[1], nx * v[2]};
        const double qw[4] = {w0 / a, -w1 / a, -w2 / a, -w3 / a};
        Cx<double> X[4], Wd[4];
        quat_su2(qx, X);
        quat_su2(qw, Wd);
        R[0] = cadd(cmul(X[0], Wd[0]), cmul(X[1], Wd[2]));
        R[1] = cadd(cmul(X[0], Wd[1]), cmul(X[1], Wd[3]));
        R[2] = cadd(cmul(X[2], Wd[0]), cmul(X[3], Wd[2]));
        R[3] = cadd(cmul(X[2], Wd[1]), cmul(X[3], Wd[3]));
    }
    M3 E = m3_id();
    E.e[i * 3 + i] = R[0];
    E.e[i * 3 + j] = R[1];
    E.e[j * 3 + i] = R[2];
    E.e[j * 3 + j] = R[3];
    U = m3_mul(E, U);
}

__global__ void __launch_bounds__(128) heatbath_kernel(Geom g, void* U, int mu, int colour, double beta, double c11,
                                                       double c12, unsigned long long seed, int sweep)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.V) return;
    Walker x;
    int rest = s;
    x.x[3] = rest % g.L[3];
    rest /= g.L[3];
    x.x[2] = rest % g.L[2];
    rest /= g.L[2];
    x.x[1] = rest % g.L[1];
    x.x[0] = rest / g.L[1];
    int sum = 0;
#pragma unroll
    for (int nu = 0; nu < 4; ++nu)
        if (nu != mu) sum += x.x[nu];
    if ((x.x[mu] & 1) * 4 + (sum & 3) != colour) return;
    M3 A1, A2;
    staples(U, g, x, mu, A1, A2);
    M3 A = m3_zero();
    m3_axpy(A, c11, A1);
    m3_axpy(A, c12, A2);
    const int p = (x.x[0] + x.x[1] + x.x[2] + x.x[3]) & 1, i = s >> 1;
    M3 u = ld_link(U, p, mu, i, g.Vh);
    const int sub[3][2] = {{0, 1}, {0, 2}, {1, 2}};
#pragma unroll 1
    for (int k = 0; k < 3; ++k) {
        HbRng r;
        r.key = make_uint2((unsigned)seed, (unsigned)(seed >> 32));
        r.link = (unsigned)(s * 4 + mu);
        r.sweep = (unsigned)sweep;
        r.tag = 0x48420000u + (unsigned)k;
        r.draw = 0;
        r.have = 0;
        hb_subgroup(r, u, A, sub[k][0], sub[k][1], beta);
    }
    st_link(U, p, mu, i, g.Vh, u);
}

cudaError_t launch_heatbath(const Geom& g, void* U, double beta, double c11, double c12, unsigned long long seed,
                            int sweep0, int nsweeps, cudaStream_t s)
{
    for (int sw = sweep0; sw < sweep0 + nsweeps; ++sw)
        for (int mu = 0; mu < 4; ++mu)
            for (int col = 0; col < 8; ++col)
                heatbath_kernel<<<(g.V + 127) / 128, 128, 0, s>>>(g, U, mu, col, beta, c11, c12, seed, sw);
    return cudaGetLastError();
}

// Y += a X over a link field (FP64 18-real)
__global__ void link_axpy_kernel(Geom g, double2* Y, double a, const double2* X, long n)
{
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double2 x = X[k], y = Y[k];
    Y[k] = make_double2(fma(a, x.x, y.x), fma(a, x.y, y.y));
}

cudaError_t launch_link_axpy(const Geom& g, void* Y, double a, const void* X, cudaStream_t s)
{
    long n = (long)g.V * 4 * 9;
    link_axpy_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, (double2*)Y, a, (const double2*)X, n);
    return cudaGetLastError();
}

cudaError_t launch_staples(const Geom& g, const void* U, void* A1, void* A2, cudaStream_t s)
{
    staple_kernel<<<dim3((g.Vh + kThreads - 1) / kThreads, 8), kThreads, 0, s>>>(g, U, A1, A2);
    return cudaGetLastError();
}

cudaError_t launch_link_update(const Geom& g, void* U, const void* P, double eps, int check, int* err,
                               cudaStream_t s)
{
    link_update_kernel<<<dim3((g.Vh + 127) / 128, 8), 128, 0, s>>>(g, U, P, eps, check, err);
    return cudaGetLastError();
}

// partial must hold kRedBlocks doubles; the result lands in *out (device)
cudaError_t launch_reduce(const Geom& g, int kind, const void* A, const void* B, double beta, double c11,
                          double c12, double* partial, double* out, cudaStream_t s)
{
    reduce_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(g, kind, A, B, beta, c11, c12, partial);
    reduce_final<<<1, 1024, 0, s>>>(partial, kRedBlocks, out);
    return cudaGetLastError();
}

}  // namespace sfh

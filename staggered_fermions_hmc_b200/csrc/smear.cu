// smear.cu — stout and HEX link smearing on the device.
//
// Every level is U'_mu(x) = exp(A) U_mu(x) with A = c * proj(G U_mu(x)^dag),
// proj(M) = (M - M^dag)/2 - tr((M - M^dag)/2)/3 (Smearing.cpp:126-129) and G a
// sum of staples running from x to x+mu.  exp(A) of the traceless
// anti-Hermitian A is evaluated as exp(i Q) with Q = -i A by the Cayley-
// Hamilton exponential (Fermions.cpp:843-902); the reference passes A itself,
// which that function rejects, so its smearing cannot run as shipped.
//
// Stout: one level per call with the plaquette staples, c = rho.
// HEX (Smearing.cpp:76-311, with c = alpha/2 at every level as there):
//   level 1  V1(a; r)   : link a smeared with the single staple through r,
//                         c = alpha3/2  (Gamma^1 of Smearing.cpp:76-123 for the
//                         triples that level 2 uses: all directions distinct)
//   level 2  V2(mu; nu) : staples of V1 links through sigma not in {mu, nu},
//                         c = alpha2/2  (Smearing.cpp:157-234)
//   level 3  U'_mu      : staples of V2 links through nu != mu,
//                         c = alpha1/2  (Smearing.cpp:236-301, Gamma_3 = 0 at start)
// Decorated fields are stored as link fields: field k of V1 holds, for
// direction a, the k-th direction r != a; likewise for V2.
#include "sfh_internal.h"
#include "walk.cuh"

namespace sfh {

namespace {

constexpr int kThreads = 128;

// exp(c proj(G U^dag)) U
__device__ __forceinline__ bool smear_link(const M3& G, const M3& U, double coef, M3& out)
{
    M3 om = m3_mul_adj(G, U);
    M3 A;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Cx<double> d = csub(om.e[i * 3 + j], cconj(om.e[j * 3 + i]));
            A.e[i * 3 + j] = {0.5 * d.re, 0.5 * d.im};
        }
    Cx<double> t = m3_tr(A);
    Cx<double> t3 = {t.re / 3.0, t.im / 3.0};
    A.e[0] = csub(A.e[0], t3);
    A.e[4] = csub(A.e[4], t3);
    A.e[8] = csub(A.e[8], t3);
    M3 Q;  // Q = -i (coef A)
#pragma unroll
    for (int k = 0; k < 9; ++k) Q.e[k] = {coef * A.e[k].im, -coef * A.e[k].re};
    M3 E;
    if (!expiq(Q, E)) return false;
    out = m3_mul(E, U);
    return true;
}

__device__ __forceinline__ int slot_of(int dir, int other) { return other - (other > dir ? 1 : 0); }

__device__ __forceinline__ const void* field(const void* base, int k, const Geom& g)
{
    return (const char*)base + (size_t)k * g.V * 4 * 9 * 16;
}

// staple from x to x+mu through direction nu with side links from S and the
// middle link from M: S_nu(x) M_mu(x+nu) S_nu(x+mu)^dag + S_nu(x-nu)^dag M_mu(x-nu) S_nu(x-nu+mu)
__device__ __forceinline__ M3 staple(const void* Sf, int s_slot, const void* Mf, int m_slot, const Geom& g,
                                     const Walker& x, int mu, int nu)
{
    Walker xn = x, xm = x, xd = x;
    walk(g, xn, nu, +1);
    walk(g, xm, mu, +1);
    walk(g, xd, nu, -1);
    Walker xdm = xd;
    walk(g, xdm, mu, +1);
    M3 up = m3_mul_adj(m3_mul(link_at(field(Sf, s_slot, g), g, x, nu), link_at(field(Mf, m_slot, g), g, xn, mu)),
                       link_at(field(Sf, s_slot, g), g, xm, nu));
    M3 dn = m3_mul(m3_adj_mul(link_at(field(Sf, s_slot, g), g, xd, nu), link_at(field(Mf, m_slot, g), g, xd, mu)),
                   link_at(field(Sf, s_slot, g), g, xdm, nu));
    m3_acc(up, dn);
    return up;
}

__global__ void __launch_bounds__(kThreads) stout_kernel(Geom g, const void* Uin, void* Uout, double rho, int* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    Walker x = link_coords(g, p, i);
    M3 C = m3_zero();
#pragma unroll 1
    for (int nu = 0; nu < 4; ++nu)
        if (nu != mu) m3_acc(C, staple(Uin, 0, Uin, 0, g, x, mu, nu));
    M3 out;
    if (!smear_link(C, ld_link(Uin, p, mu, i, g.Vh), rho, out)) {
        atomicOr(err, DEV_ERR_DOMAIN);
        out = ld_link(Uin, p, mu, i, g.Vh);
    }
    st_link(Uout, p, mu, i, g.Vh, out);
}

// V1(a; r) for the three r != a
__global__ void __launch_bounds__(kThreads) hex1_kernel(Geom g, const void* U, void* V1, double coef, int* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, a = blockIdx.y & 3;
    if (i >= g.Vh) return;
    Walker x = link_coords(g, p, i);
    M3 Ua = ld_link(U, p, a, i, g.Vh);
#pragma unroll 1
    for (int r = 0; r < 4; ++r) {
        if (r == a) continue;
        M3 out;
        if (!smear_link(staple(U, 0, U, 0, g, x, a, r), Ua, coef, out)) {
            atomicOr(err, DEV_ERR_DOMAIN);
            out = Ua;
        }
        st_link((char*)V1 + (size_t)slot_of(a, r) * g.V * 4 * 9 * 16, p, a, i, g.Vh, out);
    }
}

// V2(mu; nu) for the three nu != mu
__global__ void __launch_bounds__(kThreads) hex2_kernel(Geom g, const void* U, const void* V1, void* V2, double coef,
                                                        int* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    Walker x = link_coords(g, p, i);
    M3 Umu = ld_link(U, p, mu, i, g.Vh);
#pragma unroll 1
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        M3 G = m3_zero();
        for (int sg = 0; sg < 4; ++sg) {
            if (sg == mu || sg == nu) continue;
            const int r = 6 - mu - nu - sg;  // the direction left out of {mu, nu, sigma}
            // side links V1(sigma; r), middle link V1(mu; r)
            m3_acc(G, staple(V1, slot_of(sg, r), V1, slot_of(mu, r), g, x, mu, sg));
        }
        M3 out;
        if (!smear_link(G, Umu, coef, out)) {
            atomicOr(err, DEV_ERR_DOMAIN);
            out = Umu;
        }
        st_link((char*)V2 + (size_t)slot_of(mu, nu) * g.V * 4 * 9 * 16, p, mu, i, g.Vh, out);
    }
}

// U'_mu from the V2 staples (in place: level 3 reads U only at its own link)
__global__ void __launch_bounds__(kThreads) hex3_kernel(Geom g, void* U, const void* V2, double coef, int* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    Walker x = link_coords(g, p, i);
    M3 G = m3_zero();
#pragma unroll 1
    for (int nu = 0; nu < 4; ++nu)
        if (nu != mu) m3_acc(G, staple(V2, slot_of(nu, mu), V2, slot_of(mu, nu), g, x, mu, nu));
    M3 Umu = ld_link(U, p, mu, i, g.Vh);
    M3 out;
    if (!smear_link(G, Umu, coef, out)) {
        atomicOr(err, DEV_ERR_DOMAIN);
        out = Umu;
    }
    st_link(U, p, mu, i, g.Vh, out);
}

dim3 link_grid(const Geom& g) { return dim3((g.Vh + kThreads - 1) / kThreads, 8); }

// ---------------------------------------------------------------------------
// Smeared-link force: the chain rule through stout levels (no counterpart in
// the reference).  Method of Morningstar & Peardon, Phys. Rev. D 69 (2004)
// 054501.  Per level, with C the staples of U, Q = -i rho TA(C U^dag),
// V = exp(iQ) U and G = dS/dV (dS = sum Re Tr(G dV)):
//   L = TH(b0 Q^2 + b1 Q + f1 B + f2 (Q B + B Q)), B = U G,
//   b0 = sum_j Tr(B Q^j) df_j/dc0, b1 = sum_j Tr(B Q^j) df_j/dc1,
//   K = -i rho L, W = U^dag K,
//   dS/dU = G exp(iQ) - C^dag K + staple terms of W (sforce_gather_kernel).
// The force convention at both ends is the reference's (dS/deps = 2 Tr(F H)
// under U -> exp(i eps H) U): G = -2i V^dag F on top, F = TH(i U G)/2 below.
// ---------------------------------------------------------------------------
typedef Cx<double> Z;

__device__ __forceinline__ Z zm(Z a, Z b) { return cmul(a, b); }
__device__ __forceinline__ Z zs(Z a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ Z za(Z a, Z b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Z zd(Z a, Z b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Z zi(Z a) { return {-a.im, a.re}; }  // i a
__device__ __forceinline__ Z zdiv(Z a, double s) { return {a.re / s, a.im / s}; }

__device__ __forceinline__ double xi1_stable(double w)
{
    if (fabs(w) < 0.05) {
        double w2 = w * w;
        return -1.0 / 3.0 + w2 / 30.0 - w2 * w2 / 840.0 + w2 * w2 * w2 / 45360.0;
    }
    return (cos(w) - sin(w) / w) / (w * w);
}

// f_j of exp(iQ) = f0 + f1 Q + f2 Q^2 and df_j/dc0, df_j/dc1 (c0 = det Q,
// c1 = Tr Q^2 / 2); h_j as in expiq, dh_j/dw = w g_j, D = 9u^2 - w^2
__device__ bool expiq_coeffs(const M3& Q, const M3& Q2, Z (&f)[3], Z (&d0)[3], Z (&d1)[3])
{
    M3 Q3 = m3_mul(Q2, Q);
    double c0 = m3_tr(Q3).re / 3.0;
    double c1 = 0.5 * m3_tr(Q2).re;
    if (c1 < 0.0) return false;
    if (c1 < 1e-12) {
        f[0] = {1.0, 0.0};
        f[1] = {0.0, 1.0};
        f[2] = {-0.5, 0.0};
        for (int j = 0; j < 3; ++j) d0[j] = d1[j] = {0.0, 0.0};
        return true;
    }
    const bool neg = c0 < 0.0;
    c0 = fabs(c0);
    double c0max = 2.0 * sqrt(c1 * c1 * c1 / 27.0);
    double ratio = c0max > 0.0 ? fmin(c0 / c0max, 1.0) : 1.0;
    double theta = acos(ratio);
    double st3, ct3;
    sincos(theta / 3.0, &st3, &ct3);
    const double w = sqrt(c1) * st3, u = sqrt(c1 / 3.0) * ct3;
    const double u2 = u * u, w2 = w * w;
    const double xi0 = sinc_stable(w), xi1 = xi1_stable(w), cw = cos(w);
    double s2u, c2u, su, cu;
    sincos(2.0 * u, &s2u, &c2u);
    sincos(u, &su, &cu);
    const Z E = {c2u, s2u}, e = {cu, -su};
    const Z P0 = {8.0 * u2 * cw, 2.0 * u * (3.0 * u2 + w2) * xi0};
    const Z P1 = {2.0 * u * cw, -(3.0 * u2 - w2) * xi0};
    const Z P2 = {cw, 3.0 * u * xi0};
    Z h[3], hu[3], g[3];
    h[0] = za(zs(E, u2 - w2), zm(e, P0));
    h[1] = zd(zs(E, 2.0 * u), zm(e, P1));
    h[2] = zd(E, zm(e, P2));
    hu[0] = za(za(zs(E, 2.0 * u), zi(zs(E, 2.0 * (u2 - w2)))),
               zd(zm(e, Z{16.0 * u * cw, 2.0 * (9.0 * u2 + w2) * xi0}), zi(zm(e, P0))));
    hu[1] = za(za(zs(E, 2.0), zi(zs(E, 4.0 * u))), zd(zi(zm(e, P1)), zm(e, Z{2.0 * cw, -6.0 * u * xi0})));
    hu[2] = za(zi(zs(E, 2.0)), zd(zi(zm(e, P2)), zm(e, Z{0.0, 3.0 * xi0})));
    g[0] = za(zs(E, -2.0), zm(e, Z{-8.0 * u2 * xi0, 2.0 * u * (2.0 * xi0 + (3.0 * u2 + w2) * xi1)}));
    g[1] = zm(e, Z{2.0 * u * xi0, -2.0 * xi0 + (3.0 * u2 - w2) * xi1});
    g[2] = zm(e, Z{xi0, -3.0 * u * xi1});
    const double D = 9.0 * u2 - w2, D2 = D * D;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        Z fu = zdiv(zd(zs(hu[j], D), zs(h[j], 18.0 * u)), D2);
        Z k = zdiv(za(zs(g[j], D), zs(h[j], 2.0)), D2);
        f[j] = zdiv(h[j], D);
        d0[j] = zdiv(zd(fu, zs(k, 3.0 * u)), 2.0 * D);
        d1[j] = zdiv(za(zs(fu, u), zs(k, 0.5 * (3.0 * u2 - w2))), D);
    }
    if (neg) {  // f_j(Q) = (-1)^j conj(f_j(-Q)); c0 changes sign
        f[0] = cconj(f[0]);
        f[1] = {-f[1].re, f[1].im};
        f[2] = cconj(f[2]);
        d1[0] = cconj(d1[0]);
        d1[1] = {-d1[1].re, d1[1].im};
        d1[2] = cconj(d1[2]);
        d0[0] = {-d0[0].re, d0[0].im};
        d0[1] = cconj(d0[1]);
        d0[2] = {-d0[2].re, d0[2].im};
    }
    return true;
}

__device__ __forceinline__ M3 m3_th(const M3& a)  // traceless Hermitian part
{
    M3 t;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Z x = a.e[i * 3 + j], y = cconj(a.e[j * 3 + i]);
            t.e[i * 3 + j] = {0.5 * (x.re + y.re), 0.5 * (x.im + y.im)};
        }
    m3_traceless(t);
    return t;
}

__device__ __forceinline__ M3 m3_scale(const M3& a, Z s)
{
    M3 o;
#pragma unroll
    for (int k = 0; k < 9; ++k) o.e[k] = zm(a.e[k], s);
    return o;
}

// G = -2i V^dag F
__global__ void __launch_bounds__(kThreads) sforce_top_kernel(Geom g, const void* V, const void* F, void* G)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    st_link(G, p, mu, i, g.Vh, m3_scale(m3_adj_mul(ld_link(V, p, mu, i, g.Vh), ld_link(F, p, mu, i, g.Vh)), Z{0.0, -2.0}));
}

// per link of level U: W = U^dag K and Gn = G exp(iQ) - C^dag K
__global__ void __launch_bounds__(kThreads) sforce_level_kernel(Geom g, const void* U, const void* G, void* W, void* Gn,
                                                                double rho, int* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    Walker x = link_coords(g, p, i);
    M3 C = m3_zero();
#pragma unroll 1
    for (int nu = 0; nu < 4; ++nu)
        if (nu != mu) m3_acc(C, staple(U, 0, U, 0, g, x, mu, nu));
    const M3 u = ld_link(U, p, mu, i, g.Vh);
    M3 om = m3_mul_adj(C, u), Q;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            Z d = zd(om.e[a * 3 + b], cconj(om.e[b * 3 + a]));  // Q = -i rho TA(om)
            Q.e[a * 3 + b] = {0.5 * rho * d.im, -0.5 * rho * d.re};
        }
    m3_traceless(Q);
    const M3 Q2 = m3_mul(Q, Q);
    Z f[3], d0[3], d1[3];
    if (!expiq_coeffs(Q, Q2, f, d0, d1)) {
        atomicOr(err, DEV_ERR_DOMAIN);
        return;
    }
    M3 eq;
#pragma unroll
    for (int k = 0; k < 9; ++k) eq.e[k] = za(zm(f[1], Q.e[k]), zm(f[2], Q2.e[k]));
    eq.e[0] = za(eq.e[0], f[0]);
    eq.e[4] = za(eq.e[4], f[0]);
    eq.e[8] = za(eq.e[8], f[0]);
    const M3 Gl = ld_link(G, p, mu, i, g.Vh);
    const M3 B = m3_mul(u, Gl);
    const M3 BQ = m3_mul(B, Q), BQ2 = m3_mul(B, Q2), QB = m3_mul(Q, B);
    const Z t0 = m3_tr(B), t1 = m3_tr(BQ), t2 = m3_tr(BQ2);
    const Z b0 = za(za(zm(t0, d0[0]), zm(t1, d0[1])), zm(t2, d0[2]));
    const Z b1 = za(za(zm(t0, d1[0]), zm(t1, d1[1])), zm(t2, d1[2]));
    M3 Lh;
#pragma unroll
    for (int k = 0; k < 9; ++k)
        Lh.e[k] = za(za(zm(b0, Q2.e[k]), zm(b1, Q.e[k])), za(zm(f[1], B.e[k]), zm(f[2], za(QB.e[k], BQ.e[k]))));
    const M3 K = m3_scale(m3_th(Lh), Z{0.0, -rho});
    st_link(W, p, mu, i, g.Vh, m3_adj_mul(u, K));
    M3 out = m3_mul(Gl, eq);
    const M3 cK = m3_adj_mul(C, K);
    m3_axpy(out, -1.0, cK);
    st_link(Gn, p, mu, i, g.Vh, out);
}

// dS/dU of link (y, a): Gn + the staple terms Re Tr(W_l dC_l) of the links l
// whose plaquette staples contain it (six positions, three directions each)
__global__ void __launch_bounds__(kThreads) sforce_gather_kernel(Geom g, const void* U, const void* W, const void* Gn,
                                                                 void* G)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, a = blockIdx.y & 3;
    if (i >= g.Vh) return;
    const Walker y = link_coords(g, p, i);
    M3 out = ld_link(Gn, p, a, i, g.Vh);
#pragma unroll 1
    for (int d = 0; d < 4; ++d) {
        if (d == a) continue;
        Walker ya = y, yd = y, ymd = y;
        walk(g, ya, a, +1);
        walk(g, yd, d, +1);
        walk(g, ymd, d, -1);
        Walker ymda = ymd;
        walk(g, ymda, a, +1);
        // U_nu(x) of an upper staple of (x = y, d)
        m3_acc(out, m3_mul(m3_mul_adj(link_at(U, g, ya, d), link_at(U, g, yd, a)), link_at(W, g, y, d)));
        // U_mu(x+nu) of an upper staple of (x = y - d, a)
        m3_acc(out, m3_mul(m3_adj_mul(link_at(U, g, ymda, d), link_at(W, g, ymd, a)), link_at(U, g, ymd, d)));
        // U_nu(x+mu) of an upper staple of (x = y - d, d): (W U_a(x) U_d(x+a))^dag
        m3_acc(out, m3_adj(m3_mul(m3_mul(link_at(W, g, ymd, d), link_at(U, g, ymd, a)), link_at(U, g, ymda, d))));
        // U_nu(x-nu) of a lower staple of (x = y + a, d): (U_d(y) U_a(y+d) W)^dag
        m3_acc(out, m3_adj(m3_mul(m3_mul(link_at(U, g, y, d), link_at(U, g, yd, a)), link_at(W, g, ya, d))));
        // U_mu(x-nu) of a lower staple of (x = y + d, a)
        m3_acc(out, m3_mul_adj(m3_mul(link_at(U, g, ya, d), link_at(W, g, yd, a)), link_at(U, g, y, d)));
        // U_nu(x-nu+mu) of a lower staple of (x = y - d + a, d)
        m3_acc(out, m3_mul(m3_mul_adj(link_at(W, g, ymda, d), link_at(U, g, ymd, a)), link_at(U, g, ymd, d)));
    }
    st_link(G, p, a, i, g.Vh, out);
}

// F = TH(i U G) / 2
__global__ void __launch_bounds__(kThreads) sforce_bottom_kernel(Geom g, const void* U, const void* G, void* F)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    M3 t = m3_th(m3_scale(m3_mul(ld_link(U, p, mu, i, g.Vh), ld_link(G, p, mu, i, g.Vh)), Z{0.0, 0.5}));
    st_link(F, p, mu, i, g.Vh, t);
}

}  // namespace

// n stout levels; U is updated in place, tmp is one link field of scratch
cudaError_t launch_stout(const Geom& g, void* U, void* tmp, double rho, int n, int* err, cudaStream_t s)
{
    for (int k = 0; k < n; ++k) {
        stout_kernel<<<link_grid(g), kThreads, 0, s>>>(g, U, tmp, rho, err);
        cudaMemcpyAsync(U, tmp, (size_t)g.V * 4 * 9 * 16, cudaMemcpyDeviceToDevice, s);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The staple steps of HEX on their own, in the reference's flat tensor
// layouts (apply_step_1/3/5, Smearing.cpp:76-275): fields of 3x3 matrices
// indexed combo * V + s, s the lexicographic site, combo (4 mu + nu) 4 + rho
// (level 1 output, level 2 input), 4 mu + nu (level 2 output, level 3 input)
// or mu (level 3 output); level 1 reads the gauge field in its host layout
// [s][mu].  One thread per output matrix; a checking path for the fused
// kernels above, which keep only the decorated links the next level uses.
// ---------------------------------------------------------------------------
__device__ __forceinline__ M3 ld_mat(const double2* f, long k)
{
    M3 m;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        const double2 v = f[k * 9 + e];
        m.e[e] = {v.x, v.y};
    }
    return m;
}

__device__ __forceinline__ int lex_shift(const Geom& g, int s, int d, int dir)
{
    int c[4];
    int r = s;
    for (int k = 3; k >= 0; --k) {
        c[k] = r % g.L[k];
        r /= g.L[k];
    }
    c[d] = (c[d] + dir + g.L[d]) % g.L[d];
    return ((c[0] * g.L[1] + c[1]) * g.L[2] + c[2]) * g.L[3] + c[3];
}

// index of matrix (combo, s) of the level's input field
__device__ __forceinline__ long gamma_in(int level, const Geom& g, int a, int b, int c, int s)
{
    if (level == 1) return (long)s * 4 + a;                          // U_a(s)
    if (level == 2) return (long)((a * 4 + b) * 4 + c) * g.V + s;     // V1[a, b, c](s)
    return (long)(a * 4 + b) * g.V + s;                               // V2[a, b](s)
}

__global__ void __launch_bounds__(kThreads) hex_gamma_kernel(Geom g, int level, const double2* in, double2* out)
{
    const int ncombo = level == 1 ? 64 : (level == 2 ? 16 : 4);
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)ncombo * g.V) return;
    const int combo = (int)(idx / g.V), s = (int)(idx % g.V);
    int mu, nu = 0, rho = 0;
    if (level == 1) { mu = combo / 16; nu = (combo / 4) & 3; rho = combo & 3; }
    else if (level == 2) { mu = combo / 4; nu = combo & 3; }
    else { mu = combo; }
    M3 G = m3_zero();
    for (int sg = 0; sg < 4; ++sg) {
        if (sg == mu || (level < 3 && sg == nu) || (level == 1 && sg == rho)) continue;
        // side links S (direction sg) and middle link M (direction mu) of
        // the staple through sg: level 1 U_sg, U_mu; level 2 V1[sg, mu, nu],
        // V1[mu, nu, sg]; level 3 V2[sg, mu], V2[mu, sg]
        const int xs = lex_shift(g, s, sg, +1), xm = lex_shift(g, s, mu, +1);
        const int xd = lex_shift(g, s, sg, -1), xdm = lex_shift(g, xd, mu, +1);
        long sx, sxm, sxd, sxdm, mxs, mxd;
        if (level == 1) {
            sx = gamma_in(1, g, sg, 0, 0, s); sxm = gamma_in(1, g, sg, 0, 0, xm);
            sxd = gamma_in(1, g, sg, 0, 0, xd); sxdm = gamma_in(1, g, sg, 0, 0, xdm);
            mxs = gamma_in(1, g, mu, 0, 0, xs); mxd = gamma_in(1, g, mu, 0, 0, xd);
        } else if (level == 2) {
            sx = gamma_in(2, g, sg, mu, nu, s); sxm = gamma_in(2, g, sg, mu, nu, xm);
            sxd = gamma_in(2, g, sg, mu, nu, xd); sxdm = gamma_in(2, g, sg, mu, nu, xdm);
            mxs = gamma_in(2, g, mu, nu, sg, xs); mxd = gamma_in(2, g, mu, nu, sg, xd);
        } else {
            sx = gamma_in(3, g, sg, mu, 0, s); sxm = gamma_in(3, g, sg, mu, 0, xm);
            sxd = gamma_in(3, g, sg, mu, 0, xd); sxdm = gamma_in(3, g, sg, mu, 0, xdm);
            mxs = gamma_in(3, g, mu, sg, 0, xs); mxd = gamma_in(3, g, mu, sg, 0, xd);
        }
        M3 up = m3_mul_adj(m3_mul(ld_mat(in, sx), ld_mat(in, mxs)), ld_mat(in, sxm));
        M3 dn = m3_mul(m3_adj_mul(ld_mat(in, sxd), ld_mat(in, mxd)), ld_mat(in, sxdm));
        m3_acc(G, up);
        m3_acc(G, dn);
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) out[idx * 9 + e] = make_double2(G.e[e].re, G.e[e].im);
}

cudaError_t launch_hex_gamma(const Geom& g, int level, const void* in, void* out, cudaStream_t s)
{
    const long n = (long)(level == 1 ? 64 : (level == 2 ? 16 : 4)) * g.V;
    hex_gamma_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(g, level, (const double2*)in,
                                                                                    (double2*)out);
    return cudaGetLastError();
}

// n HEX passes; scratch holds six link fields (V1: 3, V2: 3)
cudaError_t launch_hex(const Geom& g, void* U, void* scratch, double a1, double a2, double a3, int n, int* err,
                       cudaStream_t s)
{
    char* V1 = (char*)scratch;
    char* V2 = V1 + (size_t)3 * g.V * 4 * 9 * 16;
    for (int k = 0; k < n; ++k) {
        hex1_kernel<<<link_grid(g), kThreads, 0, s>>>(g, U, V1, 0.5 * a3, err);
        hex2_kernel<<<link_grid(g), kThreads, 0, s>>>(g, U, V1, V2, 0.5 * a2, err);
        hex3_kernel<<<link_grid(g), kThreads, 0, s>>>(g, U, V2, 0.5 * a1, err);
    }
    return cudaGetLastError();
}

}  // namespace sfh

namespace sfh {

// levels: n + 1 link fields, levels[0] = thin U (in), levels[k] = stout^k(U) (out)
cudaError_t launch_stout_levels(const Geom& g, void* const* levels, double rho, int n, int* err, cudaStream_t s)
{
    for (int k = 0; k < n; ++k)
        stout_kernel<<<link_grid(g), kThreads, 0, s>>>(g, levels[k], levels[k + 1], rho, err);
    return cudaGetLastError();
}

// F (in: force on levels[n]; out: force on levels[0]); G, Gn, W: scratch link fields
cudaError_t launch_stout_force(const Geom& g, void* const* levels, int n, double rho, void* F, void* G, void* Gn,
                               void* W, int* err, cudaStream_t s)
{
    sforce_top_kernel<<<link_grid(g), kThreads, 0, s>>>(g, levels[n], F, G);
    for (int k = n - 1; k >= 0; --k) {
        sforce_level_kernel<<<link_grid(g), kThreads, 0, s>>>(g, levels[k], G, W, Gn, rho, err);
        sforce_gather_kernel<<<link_grid(g), kThreads, 0, s>>>(g, levels[k], W, Gn, G);
    }
    sforce_bottom_kernel<<<link_grid(g), kThreads, 0, s>>>(g, levels[0], G, F);
    return cudaGetLastError();
}

}  // namespace sfh

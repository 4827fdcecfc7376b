/*
 * sfh_oracle.c — CPU oracle (plain C restatement) of the reference's
 * staggered-fermion HMC hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  It is loaded by
 * tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and
 * by nothing else.  Every function cites the reference file:line it restates
 * (alexanderchasteen/Staggered_Fermions_HMC).  Parity of this restatement is
 * pinned against outputs of the unmodified reference sources (tests/golden)
 * and the reference's analytic known-answer tests.
 *
 * Layouts are the reference's AoS layouts (see sfh_oracle.h).  Dimensions are
 * runtime values; the reference uses compile-time constants with
 * Lx = Ly = Lz = Spatial_Size and Lt = temporal_size (Parameters.h:9-10).
 */
#include "sfh_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cx;

/* ------------------------------------------------------------------------ */
/* geometry                                                                  */
/* ------------------------------------------------------------------------ */

typedef struct {
    int L[4];
    long V;
    int* up;    /* [s*4+mu] neighbour s+mu                     */
    int* dn;    /* [s*4+mu] neighbour s-mu                     */
    int* bcup;  /* fermion boundary sign of the +mu hop        */
    int* bcdn;  /* fermion boundary sign of the -mu hop        */
    int* eta;   /* staggered phase eta_mu(x)                   */
} tab_t;

static long site_of(const int L[4], const int c[4])
{
    return (((long)c[0] * L[1] + c[1]) * L[2] + c[2]) * L[3] + c[3];
}

static void coords_of(const int L[4], long s, int c[4])
{
    c[3] = (int)(s % L[3]); s /= L[3];
    c[2] = (int)(s % L[2]); s /= L[2];
    c[1] = (int)(s % L[1]); s /= L[1];
    c[0] = (int)s;
}

/* Fermions.cpp:20-96.  eta_mu(x) = prod_{nu<mu} (-1)^{x_nu}; the +t hop that
 * wraps and the -t hop that wraps carry a -1 (anti-periodic in time); spatial
 * directions are periodic. */
static void tab_fill(const int L[4], int* up, int* dn, int* bcup, int* bcdn,
                     int* eta)
{
    long V = (long)L[0] * L[1] * L[2] * L[3];
    for (long s = 0; s < V; ++s) {
        int c[4];
        coords_of(L, s, c);
        for (int mu = 0; mu < 4; ++mu) {
            int e = 1;
            for (int nu = 0; nu < mu; ++nu)
                if (c[nu] & 1) e = -e;
            eta[s * 4 + mu] = e;

            int cu[4] = {c[0], c[1], c[2], c[3]};
            int bu = 1;
            cu[mu] += 1;
            if (cu[mu] >= L[mu]) {
                cu[mu] -= L[mu];
                if (mu == 3) bu = -1;
            }
            up[s * 4 + mu] = (int)site_of(L, cu);
            bcup[s * 4 + mu] = bu;

            int cd[4] = {c[0], c[1], c[2], c[3]};
            int bd = 1;
            if (cd[mu] == 0) {
                cd[mu] = L[mu] - 1;
                if (mu == 3) bd = -1;
            } else {
                cd[mu] -= 1;
            }
            dn[s * 4 + mu] = (int)site_of(L, cd);
            bcdn[s * 4 + mu] = bd;
        }
    }
}

static void tab_build(tab_t* t, const int dims[4])
{
    memcpy(t->L, dims, sizeof(int) * 4);
    t->V = (long)dims[0] * dims[1] * dims[2] * dims[3];
    size_t n = (size_t)t->V * 4;
    t->up = (int*)malloc(n * sizeof(int));
    t->dn = (int*)malloc(n * sizeof(int));
    t->bcup = (int*)malloc(n * sizeof(int));
    t->bcdn = (int*)malloc(n * sizeof(int));
    t->eta = (int*)malloc(n * sizeof(int));
    tab_fill(dims, t->up, t->dn, t->bcup, t->bcdn, t->eta);
}

static void tab_free(tab_t* t)
{
    free(t->up); free(t->dn); free(t->bcup); free(t->bcdn); free(t->eta);
}

void orc_tables(const int dims[4], int* up, int* dn, int* bc_up, int* bc_dn,
                int* eta)
{
    tab_fill(dims, up, dn, bc_up, bc_dn, eta);
}

/* ------------------------------------------------------------------------ */
/* 3x3 complex helpers (row-major, matching the [row][col][re,im] storage)   */
/* ------------------------------------------------------------------------ */

static const cx* link_at(const double* U, long s, int mu)
{
    return (const cx*)(U + (s * 4 + mu) * 18);
}

static void m_id(cx* a)
{
    for (int i = 0; i < 9; ++i) a[i] = 0;
    a[0] = a[4] = a[8] = 1;
}

static void m_mul(const cx* a, const cx* b, cx* out)   /* out = a b */
{
    cx t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            cx s = 0;
            for (int k = 0; k < 3; ++k) s += a[i * 3 + k] * b[k * 3 + j];
            t[i * 3 + j] = s;
        }
    memcpy(out, t, sizeof(t));
}

static void m_mul_adj(const cx* a, const cx* b, cx* out)  /* out = a b^dag */
{
    cx t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            cx s = 0;
            for (int k = 0; k < 3; ++k) s += a[i * 3 + k] * conj(b[j * 3 + k]);
            t[i * 3 + j] = s;
        }
    memcpy(out, t, sizeof(t));
}

static void m_adj(const cx* a, cx* out)
{
    cx t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[i * 3 + j] = conj(a[j * 3 + i]);
    memcpy(out, t, sizeof(t));
}

static cx m_tr(const cx* a) { return a[0] + a[4] + a[8]; }

static void mv(const cx* a, const cx* v, cx* out)   /* out = a v */
{
    for (int i = 0; i < 3; ++i)
        out[i] = a[i * 3 + 0] * v[0] + a[i * 3 + 1] * v[1] + a[i * 3 + 2] * v[2];
}

static void mdv(const cx* a, const cx* v, cx* out)  /* out = a^dag v */
{
    for (int i = 0; i < 3; ++i)
        out[i] = conj(a[0 * 3 + i]) * v[0] + conj(a[1 * 3 + i]) * v[1] +
                 conj(a[2 * 3 + i]) * v[2];
}

/* ------------------------------------------------------------------------ */
/* staggered operator                                                        */
/* ------------------------------------------------------------------------ */

/* Fermions.cpp:218-247 (sign=+1) and 254-283 (sign=-1). */
static void dirac_tab(const tab_t* t, double mass, int sign, const double* U,
                      const double* in, double* out)
{
    const cx* psi = (const cx*)in;
    cx* res = (cx*)out;
    long V = t->V;
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        cx r[3], tmp[3];
        for (int c = 0; c < 3; ++c) r[c] = mass * psi[s * 3 + c];
        for (int mu = 0; mu < 4; ++mu) {
            long k = s * 4 + mu;
            double cf = 0.5 * t->eta[k] * t->bcup[k] * sign;
            mv(link_at(U, s, mu), psi + (long)t->up[k] * 3, tmp);
            for (int c = 0; c < 3; ++c) r[c] += cf * tmp[c];
            long d = t->dn[k];
            double cb = 0.5 * t->eta[k] * t->bcdn[k] * sign;
            mdv(link_at(U, d, mu), psi + d * 3, tmp);
            for (int c = 0; c < 3; ++c) r[c] -= cb * tmp[c];
        }
        for (int c = 0; c < 3; ++c) res[s * 3 + c] = r[c];
    }
}

void orc_dirac(const int dims[4], double mass, int sign, const double* U,
               const double* in, double* out)
{
    tab_t t;
    tab_build(&t, dims);
    dirac_tab(&t, mass, sign >= 0 ? 1 : -1, U, in, out);
    tab_free(&t);
}

/* Fermions.cpp:530-547: temp = D^dag in; out = D temp. */
static void ddag_tab(const tab_t* t, double mass, const double* U,
                     const double* in, double* out, double* tmp)
{
    dirac_tab(t, mass, -1, U, in, tmp);
    dirac_tab(t, mass, +1, U, tmp, out);
}

void orc_ddag(const int dims[4], double mass, const double* U,
              const double* in, double* out)
{
    tab_t t;
    tab_build(&t, dims);
    double* tmp = (double*)malloc(sizeof(double) * 6 * t.V);
    ddag_tab(&t, mass, U, in, out, tmp);
    free(tmp);
    tab_free(&t);
}

/* Fermions.cpp:521-528 */
double orc_dot(long n, const double* a, const double* b)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* Fermions.cpp:553-617: plain CG with X0 = 0, stop when r^2 < tol^2 |phi|^2
 * (recursive residual), breakdown / non-finite checks as in the reference. */
static int cg_tab(const tab_t* t, double mass, const double* U,
                  const double* phi, double tol, int maxit, double* X,
                  int* iters, double* final_rsq)
{
    long n = 6 * t->V;
    double* r = (double*)malloc(sizeof(double) * n);
    double* p = (double*)malloc(sizeof(double) * n);
    double* v = (double*)malloc(sizeof(double) * n);
    double* tmp = (double*)malloc(sizeof(double) * n);
    int status = ORC_OK, it = 0;
    memset(X, 0, sizeof(double) * n);
    memcpy(r, phi, sizeof(double) * n);
    memcpy(p, phi, sizeof(double) * n);
    double rsq = orc_dot(n, r, r);
    double phisq = orc_dot(n, phi, phi);
    if (phisq < 1e-28) goto done;
    double target = tol * tol * phisq;
    for (it = 0; it < maxit; ++it) {
        if (rsq < target) break;
        ddag_tab(t, mass, U, p, v, tmp);
        double pv = orc_dot(n, p, v);
        if (!isfinite(pv) || fabs(pv) < 1e-30) { status = ORC_ERR_BREAKDOWN; goto done; }
        double alpha = rsq / pv;
        if (!isfinite(alpha)) { status = ORC_ERR_BREAKDOWN; goto done; }
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) {
            X[i] += alpha * p[i];
            r[i] -= alpha * v[i];
        }
        double rnew = orc_dot(n, r, r);
        double beta = rnew / rsq;
        if (!isfinite(beta)) { status = ORC_ERR_BREAKDOWN; goto done; }
        rsq = rnew;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
    }
    if (rsq >= target) status = ORC_ERR_NOCONV;
done:
    if (iters) *iters = it;
    if (final_rsq) *final_rsq = rsq;
    free(r); free(p); free(v); free(tmp);
    return status;
}

int orc_cg(const int dims[4], double mass, const double* U, const double* phi,
           double tol, int maxit, double* X, int* iters, double* final_rsq)
{
    tab_t t;
    tab_build(&t, dims);
    int st = cg_tab(&t, mass, U, phi, tol, maxit, X, iters, final_rsq);
    tab_free(&t);
    return st;
}

/* ------------------------------------------------------------------------ */
/* staples and gauge force                                                   */
/* ------------------------------------------------------------------------ */

/* Product of links along a lattice path.  step = +(mu+1) walks forward in mu
 * (multiplies U_mu(pos)), step = -(mu+1) walks backward (multiplies
 * U_mu(pos-mu)^dag).  Gauge links are periodic in every direction
 * (Lattice.cpp:213-235). */
static void path_product(const tab_t* t, const double* U, long start,
                         const int* steps, int nsteps, cx* out)
{
    cx m[9];
    m_id(m);
    long pos = start;
    for (int i = 0; i < nsteps; ++i) {
        int st = steps[i];
        int mu = (st > 0 ? st : -st) - 1;
        if (st > 0) {
            m_mul(m, link_at(U, pos, mu), m);
            pos = t->up[pos * 4 + mu];
        } else {
            pos = t->dn[pos * 4 + mu];
            m_mul_adj(m, link_at(U, pos, mu), m);
        }
    }
    memcpy(out, m, sizeof(m));
}

/* Plaquette staple sum A1 for link (s, mu), Lattice.cpp:249-313: the paths
 * from x+mu back to x, so that U_mu(x) A1 is a sum of closed plaquettes. */
static void staple_plaq(const tab_t* t, const double* U, long s, int mu,
                        cx* A1)
{
    long xp = t->up[s * 4 + mu];
    int M = mu + 1;
    for (int i = 0; i < 9; ++i) A1[i] = 0;
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        int N = nu + 1;
        const int top[3] = {+N, -M, -N};
        const int bot[3] = {-N, -M, +N};
        cx m[9];
        path_product(t, U, xp, top, 3, m);
        for (int i = 0; i < 9; ++i) A1[i] += m[i];
        path_product(t, U, xp, bot, 3, m);
        for (int i = 0; i < 9; ++i) A1[i] += m[i];
    }
}

/* Rectangle staple sum A2 for link (s, mu), Lattice.cpp:315-499: the six
 * 1x2 / 2x1 rectangles per orthogonal direction nu that contain the link,
 * each as the path from x+mu back to x (types 1..6 of the reference). */
static void staple_rect(const tab_t* t, const double* U, long s, int mu,
                        cx* A2)
{
    long xp = t->up[s * 4 + mu];
    int M = mu + 1;
    for (int i = 0; i < 9; ++i) A2[i] = 0;
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        int N = nu + 1;
        const int paths[6][5] = {
            {-N, -N, -M, +N, +N},  /* type 1: short side, below  */
            {+N, +N, -M, -N, -N},  /* type 2: short side, above  */
            {+M, -N, -M, -M, +N},  /* type 3: long side, below, link first */
            {+N, -M, -M, -N, +M},  /* type 4: long side, above, link second */
            {-N, -M, -M, +N, +M},  /* type 5: long side, below, link second */
            {+M, +N, -M, -M, -N},  /* type 6: long side, above, link first */
        };
        for (int k = 0; k < 6; ++k) {
            cx m[9];
            path_product(t, U, xp, paths[k], 5, m);
            for (int i = 0; i < 9; ++i) A2[i] += m[i];
        }
    }
}

void orc_staples(const int dims[4], const double* U, double* A1, double* A2)
{
    tab_t t;
    tab_build(&t, dims);
    long V = t.V;
#pragma omp parallel for schedule(static)
    for (long l = 0; l < 4 * V; ++l) {
        long s = l / 4;
        int mu = (int)(l % 4);
        staple_plaq(&t, U, s, mu, (cx*)(A1 + l * 18));
        staple_rect(&t, U, s, mu, (cx*)(A2 + l * 18));
    }
    tab_free(&t);
}

/* make a 3x3 traceless: a -= tr(a)/3 I */
static void m_traceless(cx* a)
{
    cx tr3 = m_tr(a) / 3.0;
    a[0] -= tr3; a[4] -= tr3; a[8] -= tr3;
}

/* Fermions.cpp:372-384: F = -i (beta/12) (Q - Q^dag), Q = U V,
 * V = c11 A1 + c12 A2 (Lattice.cpp:502-507); trace removed. */
static void gauge_force_link(const tab_t* t, double beta, double c11,
                             double c12, const double* U, long s, int mu,
                             cx* F)
{
    cx A1[9], A2[9], Vs[9], Q[9];
    staple_plaq(t, U, s, mu, A1);
    staple_rect(t, U, s, mu, A2);
    for (int i = 0; i < 9; ++i) Vs[i] = c11 * A1[i] + c12 * A2[i];
    m_mul(link_at(U, s, mu), Vs, Q);
    cx f = -I * (beta / 12.0);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            F[i * 3 + j] = f * (Q[i * 3 + j] - conj(Q[j * 3 + i]));
    m_traceless(F);
}

void orc_gauge_force(const int dims[4], double beta, double c11, double c12,
                     const double* U, double* F)
{
    tab_t t;
    tab_build(&t, dims);
#pragma omp parallel for schedule(static)
    for (long l = 0; l < 4 * t.V; ++l)
        gauge_force_link(&t, beta, c11, c12, U, l / 4, (int)(l % 4),
                         (cx*)(F + l * 18));
    tab_free(&t);
}

/* Fermions.cpp:443-515: c = eta bc / 4;
 * A_f = (U Y(x+mu)) X(x)^dag, A_b = Y(x) X(x+mu)^dag U^dag,
 * F = -i c [(A_f - A_f^dag) + (A_b - A_b^dag)], trace removed. */
static void fermion_force_link(const tab_t* t, const double* U,
                               const double* X, const double* Y, long s,
                               int mu, cx* F)
{
    long k = s * 4 + mu;
    long up = t->up[k];
    double c = 0.25 * t->eta[k] * t->bcup[k];
    const cx* Ux = link_at(U, s, mu);
    const cx* Xx = (const cx*)X + s * 3;
    const cx* Xu = (const cx*)X + up * 3;
    const cx* Yx = (const cx*)Y + s * 3;
    const cx* Yu = (const cx*)Y + up * 3;
    cx uy[3], Af[9], T[9], Ab[9];
    mv(Ux, Yu, uy);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            Af[i * 3 + j] = uy[i] * conj(Xx[j]);
            T[i * 3 + j] = Yx[i] * conj(Xu[j]);
        }
    m_mul_adj(T, Ux, Ab);
    cx f = -I * c;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            cx a = (Af[i * 3 + j] - conj(Af[j * 3 + i])) +
                   (Ab[i * 3 + j] - conj(Ab[j * 3 + i]));
            F[i * 3 + j] = f * a;
        }
    m_traceless(F);
}

void orc_fermion_force(const int dims[4], const double* U, const double* X,
                       const double* Y, double* F)
{
    tab_t t;
    tab_build(&t, dims);
#pragma omp parallel for schedule(static)
    for (long l = 0; l < 4 * t.V; ++l)
        fermion_force_link(&t, U, X, Y, l / 4, (int)(l % 4),
                           (cx*)(F + l * 18));
    tab_free(&t);
}

static void full_force_tab(const tab_t* t, double beta, double c11, double c12,
                           const double* U, const double* X, const double* Y,
                           double* F)
{
#pragma omp parallel for schedule(static)
    for (long l = 0; l < 4 * t->V; ++l) {
        cx fg[9], ff[9];
        gauge_force_link(t, beta, c11, c12, U, l / 4, (int)(l % 4), fg);
        fermion_force_link(t, U, X, Y, l / 4, (int)(l % 4), ff);
        cx* o = (cx*)(F + l * 18);
        for (int i = 0; i < 9; ++i) o[i] = fg[i] + ff[i];
    }
}

/* Fermions.cpp:640-659 */
void orc_full_force(const int dims[4], double beta, double c11, double c12,
                    const double* U, const double* X, const double* Y,
                    double* F)
{
    tab_t t;
    tab_build(&t, dims);
    full_force_tab(&t, beta, c11, c12, U, X, Y, F);
    tab_free(&t);
}

/* ------------------------------------------------------------------------ */
/* exp(iQ) by Cayley-Hamilton (Morningstar & Peardon, hep-lat/0311018)       */
/* ------------------------------------------------------------------------ */

/* Fermions.cpp:834-841 */
static double sinc_stable(double x)
{
    if (fabs(x) <= 0.05) {
        double x2 = x * x;
        return 1.0 - (x2 / 6.0) * (1.0 - (x2 / 20.0) * (1.0 - x2 / 42.0));
    }
    return sin(x) / x;
}

/* Fermions.cpp:843-902 */
static int expiq_cx(const cx* Q, cx* out)
{
    cx Q2[9], Q3[9];
    m_mul(Q, Q, Q2);
    m_mul(Q2, Q, Q3);
    cx t3 = m_tr(Q3);
    if (fabs(cimag(t3)) > 1e-10) return ORC_ERR_DOMAIN;
    double c0 = creal(t3) / 3.0;
    double c1 = 0.5 * creal(m_tr(Q2));
    if (c1 < 0.0) return ORC_ERR_DOMAIN;
    if (c1 < 1e-12) {
        for (int i = 0; i < 9; ++i) out[i] = I * Q[i] - 0.5 * Q2[i];
        out[0] += 1; out[4] += 1; out[8] += 1;
        return ORC_OK;
    }
    int neg = c0 < 0.0;
    c0 = fabs(c0);
    double c0max = 2.0 * sqrt(c1 * c1 * c1 / 27.0);
    double ratio = 1.0;
    if (c0max > 0.0) {
        ratio = c0 / c0max;
        if (ratio > 1.0) ratio = 1.0;
        if (ratio < -1.0) ratio = -1.0;
    }
    double theta = acos(ratio);
    double w = sqrt(c1) * sin(theta / 3.0);
    double u = sqrt(c1 / 3.0) * cos(theta / 3.0);
    double xi = sinc_stable(w), cw = cos(w);
    cx e2u = cexp(2.0 * I * u), emu = cexp(-I * u);
    cx h0 = (u * u - w * w) * e2u +
            emu * (8.0 * u * u * cw + 2.0 * I * u * (3.0 * u * u + w * w) * xi);
    cx h1 = 2.0 * u * e2u - emu * (2.0 * u * cw - I * (3.0 * u * u - w * w) * xi);
    cx h2 = e2u - emu * (cw + 3.0 * I * u * xi);
    double den = 9.0 * u * u - w * w;
    cx f0 = h0 / den, f1 = h1 / den, f2 = h2 / den;
    if (neg) {
        f0 = conj(f0);
        f1 = -conj(f1);
        f2 = conj(f2);
    }
    for (int i = 0; i < 9; ++i) out[i] = f1 * Q[i] + f2 * Q2[i];
    out[0] += f0; out[4] += f0; out[8] += f0;
    return ORC_OK;
}

int orc_expiq(const double* Q, double* out)
{
    cx o[9];
    int st = expiq_cx((const cx*)Q, o);
    if (st == ORC_OK) memcpy(out, o, sizeof(o));
    return st;
}

int orc_exp_field(long n, double eps, const double* H, double* U)
{
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (long i = 0; i < n; ++i) {
        cx q[9];
        const cx* h = (const cx*)(H + i * 18);
        for (int k = 0; k < 9; ++k) q[k] = eps * h[k];
        if (expiq_cx(q, (cx*)(U + i * 18)) != ORC_OK) bad = 1;
    }
    return bad ? ORC_ERR_DOMAIN : ORC_OK;
}

/* Fermions.cpp:984-994: U <- exp(i eps P) U for every link. */
static int link_update_V(long V, double eps, const double* P, double* U)
{
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (long l = 0; l < 4 * V; ++l) {
        cx q[9], e[9];
        const cx* p = (const cx*)(P + l * 18);
        cx* u = (cx*)(U + l * 18);
        for (int k = 0; k < 9; ++k) q[k] = eps * p[k];
        if (expiq_cx(q, e) != ORC_OK) { bad = 1; continue; }
        m_mul(e, u, u);
    }
    return bad ? ORC_ERR_DOMAIN : ORC_OK;
}

int orc_link_update(const int dims[4], double eps, const double* P, double* U)
{
    long V = (long)dims[0] * dims[1] * dims[2] * dims[3];
    return link_update_V(V, eps, P, U);
}

/* Fermions.cpp:662-678 */
double orc_trp2(const int dims[4], const double* P)
{
    long V = (long)dims[0] * dims[1] * dims[2] * dims[3];
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (long l = 0; l < 4 * V; ++l) {
        const cx* p = (const cx*)(P + l * 18);
        cx p2[9];
        m_mul(p, p, p2);
        acc += creal(m_tr(p2));
    }
    return acc;
}

/* Lattice.cpp:759-781 */
double orc_action(const int dims[4], double beta, double c11, double c12,
                  const double* U)
{
    tab_t t;
    tab_build(&t, dims);
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (long l = 0; l < 4 * t.V; ++l) {
        cx A1[9], A2[9], m[9];
        long s = l / 4;
        int mu = (int)(l % 4);
        staple_plaq(&t, U, s, mu, A1);
        staple_rect(&t, U, s, mu, A2);
        m_mul(link_at(U, s, mu), A1, m);
        double ap = creal(m_tr(m)) / 4.0;
        m_mul(link_at(U, s, mu), A2, m);
        double ar = creal(m_tr(m)) / 6.0;
        acc += -(beta / 3.0) * (c11 * ap + c12 * ar);
    }
    tab_free(&t);
    return acc;
}

/* Lattice.cpp:784-804 (sum over links of ReTr(U A1)/3, divided by 4V) */
double orc_avg_plaq(const int dims[4], const double* U)
{
    tab_t t;
    tab_build(&t, dims);
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (long l = 0; l < 4 * t.V; ++l) {
        cx A1[9], m[9];
        staple_plaq(&t, U, l / 4, (int)(l % 4), A1);
        m_mul(link_at(U, l / 4, (int)(l % 4)), A1, m);
        acc += creal(m_tr(m)) / 3.0;
    }
    double V = (double)t.V;
    tab_free(&t);
    return acc / (4.0 * V);
}

/* ------------------------------------------------------------------------ */
/* leapfrog: local_initial_half_step / local_leapfrog_steps /                */
/* local_final_step, Fermions.cpp:967-1028                                   */
/* ------------------------------------------------------------------------ */

static int force_and_kick(const tab_t* t, double mass, double beta, double c11,
                          double c12, double kick, double tol, int maxit,
                          const double* phi, double* P, const double* U,
                          double* X, double* Y, double* F, long* iters_total)
{
    int it = 0;
    int st = cg_tab(t, mass, U, phi, tol, maxit, X, &it, NULL);
    if (iters_total) *iters_total += it;
    if (st != ORC_OK) return st;
    dirac_tab(t, mass, -1, U, X, Y);                      /* Fermions.cpp:623-633 */
    full_force_tab(t, beta, c11, c12, U, X, Y, F);
    long n = 72 * t->V;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) P[i] -= kick * F[i];
    return ORC_OK;
}

int orc_leapfrog(const int dims[4], double mass, double beta, double c11,
                 double c12, double eps, int n_steps, double tol, int maxit,
                 const double* phi, double* P, double* U, double* X,
                 long* cg_iters_total)
{
    tab_t t;
    tab_build(&t, dims);
    double* Y = (double*)malloc(sizeof(double) * 6 * t.V);
    double* F = (double*)malloc(sizeof(double) * 72 * t.V);
    if (cg_iters_total) *cg_iters_total = 0;
    int st = force_and_kick(&t, mass, beta, c11, c12, eps * 0.5, tol, maxit,
                            phi, P, U, X, Y, F, cg_iters_total);
    for (int n = 1; st == ORC_OK && n < n_steps; ++n) {
        st = link_update_V(t.V, eps, P, U);
        if (st != ORC_OK) break;
        st = force_and_kick(&t, mass, beta, c11, c12, eps, tol, maxit, phi, P,
                            U, X, Y, F, cg_iters_total);
    }
    if (st == ORC_OK) st = link_update_V(t.V, eps, P, U);
    if (st == ORC_OK)
        st = force_and_kick(&t, mass, beta, c11, c12, eps * 0.5, tol, maxit,
                            phi, P, U, X, Y, F, cg_iters_total);
    free(Y); free(F);
    tab_free(&t);
    return st;
}

/* ------------------------------------------------------------------------ */
/* Polyakov loop                                                             */
/* ------------------------------------------------------------------------ */

/* Lattice.cpp:849-882 */
void orc_polyakov_grid(const int dims[4], const double* U, double* out)
{
    int Lx = dims[0], Ly = dims[1], Lz = dims[2], Lt = dims[3];
#pragma omp parallel for schedule(static)
    for (long g = 0; g < (long)Lx * Ly * Lz; ++g) {
        int c[4] = {(int)(g / ((long)Ly * Lz)), (int)((g / Lz) % Ly),
                    (int)(g % Lz), 0};
        cx w[9];
        m_id(w);
        for (int tt = 0; tt < Lt; ++tt) {
            c[3] = tt;
            m_mul(w, link_at(U, site_of(dims, c), 3), w);
        }
        cx tr = m_tr(w);
        out[2 * g] = creal(tr);
        out[2 * g + 1] = cimag(tr);
    }
}

/* Lattice.cpp:886-948: average of P(m) conj(P(m+d)) over m and over the
 * displacement vectors d with |d|^2 = r2 (|d_i| <= L/2, d_i != L/2 for even L).
 * Assumes a cubic spatial volume as the reference does. */
void orc_polyakov_corr(const int dims[4], const double* grid, int r2,
                       double* out2)
{
    int L = dims[0];
    int maxd = (int)sqrt((double)r2);
    if (maxd > L / 2) maxd = L / 2;
    const cx* P = (const cx*)grid;
    cx acc = 0;
    long n = 0;
    for (int x = 0; x < L; ++x)
        for (int y = 0; y < L; ++y)
            for (int z = 0; z < L; ++z) {
                cx pm = P[((long)x * L + y) * L + z];
                for (int dx = -maxd; dx <= maxd; ++dx) {
                    if (dx == L / 2 && L % 2 == 0) continue;
                    for (int dy = -maxd; dy <= maxd; ++dy) {
                        if (dy == L / 2 && L % 2 == 0) continue;
                        for (int dz = -maxd; dz <= maxd; ++dz) {
                            if (dz == L / 2 && L % 2 == 0) continue;
                            if (dx * dx + dy * dy + dz * dz != r2) continue;
                            int nx = (x + dx + L) % L, ny = (y + dy + L) % L,
                                nz = (z + dz + L) % L;
                            acc += pm * conj(P[((long)nx * L + ny) * L + nz]);
                            ++n;
                        }
                    }
                }
            }
    if (n > 0) acc /= (double)n;
    out2[0] = creal(acc);
    out2[1] = cimag(acc);
}

/* ------------------------------------------------------------------------ */
/* smearing                                                                  */
/* ------------------------------------------------------------------------ */

/* Smearing.cpp:126-129: traceless anti-Hermitian part */
static void proj_ah(const cx* m, cx* out)
{
    cx a[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            a[i * 3 + j] = 0.5 * (m[i * 3 + j] - conj(m[j * 3 + i]));
    cx tr3 = (1.0 / 3.0) * m_tr(a);
    for (int i = 0; i < 9; ++i) out[i] = a[i];
    out[0] -= tr3; out[4] -= tr3; out[8] -= tr3;
}

/* U' = exp(coef * proj(G U^dag)) U, with exp(A) = exp(i (-i A)). */
static int smear_link(const cx* G, const cx* Uold, double coef, cx* out)
{
    cx om[9], A[9], q[9], e[9];
    m_mul_adj(G, Uold, om);
    proj_ah(om, A);
    for (int i = 0; i < 9; ++i) q[i] = -I * (A[i] * coef);
    int st = expiq_cx(q, e);
    if (st != ORC_OK) return st;
    m_mul(e, Uold, out);
    return ORC_OK;
}

int orc_stout(const int dims[4], double rho, int n_levels, double* U)
{
    tab_t t;
    tab_build(&t, dims);
    long V = t.V;
    double* old = (double*)malloc(sizeof(double) * 72 * V);
    int bad = 0;
    for (int lev = 0; lev < n_levels && !bad; ++lev) {
        memcpy(old, U, sizeof(double) * 72 * V);
#pragma omp parallel for schedule(static) reduction(| : bad)
        for (long l = 0; l < 4 * V; ++l) {
            long s = l / 4;
            int mu = (int)(l % 4);
            cx C[9], m1[9], m2[9];
            for (int i = 0; i < 9; ++i) C[i] = 0;
            for (int nu = 0; nu < 4; ++nu) {
                if (nu == mu) continue;
                long xn = t.up[s * 4 + nu], xm = t.up[s * 4 + mu];
                long xd = t.dn[s * 4 + nu], xdm = t.up[xd * 4 + mu];
                m_mul(link_at(old, s, nu), link_at(old, xn, mu), m1);
                m_mul_adj(m1, link_at(old, xm, nu), m1);
                for (int i = 0; i < 9; ++i) C[i] += m1[i];
                m_adj(link_at(old, xd, nu), m2);
                m_mul(m2, link_at(old, xd, mu), m2);
                m_mul(m2, link_at(old, xdm, nu), m2);
                for (int i = 0; i < 9; ++i) C[i] += m2[i];
            }
            if (smear_link(C, link_at(old, s, mu), rho, (cx*)(U + l * 18)) !=
                ORC_OK)
                bad = 1;
        }
    }
    free(old);
    tab_free(&t);
    return bad ? ORC_ERR_DOMAIN : ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* smeared-link force: the chain rule through stout levels                   */
/* ------------------------------------------------------------------------ */
/*
 * No counterpart in the reference (it has no smeared-link HMC).  Method of
 * Morningstar & Peardon, Phys. Rev. D 69 (2004) 054501, restated:
 *
 *   level k:  C = sum of plaquette staples of U (orientation as orc_stout),
 *             Q = -i rho TA(C U^dag),  V = exp(iQ) U.
 *   With dS = sum_links Re Tr(G dV) (G = dS/dV), the generator form of the
 *   reference's force (dS/deps = 2 Tr(F H) under U -> exp(i eps H) U) gives
 *   G = -2i V^dag F at the top level and F = 1/2 TH(i U G) at the bottom.
 *   One level down:
 *     Re Tr(U G d exp(iQ)) = Re Tr(L dQ),  L = TH(b0 Q^2 + b1 Q + f1 B + f2 (Q B + B Q)),
 *       B = U G, b0 = sum_j Tr(B Q^j) df_j/dc0, b1 = sum_j Tr(B Q^j) df_j/dc1
 *       (exp(iQ) = f0 + f1 Q + f2 Q^2, c0 = det Q, c1 = Tr Q^2 / 2);
 *     K = -i rho L, W = U^dag K;
 *     dS/dU(link) = G exp(iQ) - C^dag K + the staple terms of W (stout_gather).
 */

/* xi1(w) = cos(w)/w^2 - sin(w)/w^3, series below 0.05 */
static double xi1_stable(double w)
{
    if (fabs(w) < 0.05) {
        double w2 = w * w;
        return -1.0 / 3.0 + w2 / 30.0 - w2 * w2 / 840.0 + w2 * w2 * w2 / 45360.0;
    }
    return (cos(w) - sin(w) / w) / (w * w);
}

/* f_j of exp(iQ) and df_j/dc0, df_j/dc1.  h_j as in expiq_cx; with
 * D = 9u^2 - w^2, f_j = h_j / D, dh_j/dw = w g_j (h_j are even in w),
 * c0 = 2u(u^2 - w^2), c1 = 3u^2 + w^2. */
static int expiq_coeffs(const cx* Q, cx f[3], cx d0[3], cx d1[3])
{
    cx Q2[9], Q3[9];
    m_mul(Q, Q, Q2);
    m_mul(Q2, Q, Q3);
    double c0 = creal(m_tr(Q3)) / 3.0;
    double c1 = 0.5 * creal(m_tr(Q2));
    if (c1 < 0.0) return ORC_ERR_DOMAIN;
    if (c1 < 1e-12) {  /* exp(iQ) = 1 + iQ - Q^2/2 to this order */
        f[0] = 1; f[1] = I; f[2] = -0.5;
        for (int j = 0; j < 3; ++j) d0[j] = d1[j] = 0;
        return ORC_OK;
    }
    int neg = c0 < 0.0;
    c0 = fabs(c0);
    double c0max = 2.0 * sqrt(c1 * c1 * c1 / 27.0);
    double ratio = c0max > 0.0 ? c0 / c0max : 1.0;
    if (ratio > 1.0) ratio = 1.0;
    double theta = acos(ratio);
    double w = sqrt(c1) * sin(theta / 3.0);
    double u = sqrt(c1 / 3.0) * cos(theta / 3.0);
    double u2 = u * u, w2 = w * w;
    double xi0 = sinc_stable(w), xi1 = xi1_stable(w), cw = cos(w);
    cx E = cexp(2.0 * I * u), e = cexp(-I * u);
    cx P0 = 8.0 * u2 * cw + 2.0 * I * u * (3.0 * u2 + w2) * xi0;
    cx P1 = 2.0 * u * cw - I * (3.0 * u2 - w2) * xi0;
    cx P2 = cw + 3.0 * I * u * xi0;
    cx h[3], hu[3], g[3];
    h[0] = (u2 - w2) * E + e * P0;
    h[1] = 2.0 * u * E - e * P1;
    h[2] = E - e * P2;
    hu[0] = 2.0 * u * E + 2.0 * I * (u2 - w2) * E - I * e * P0 +
            e * (16.0 * u * cw + 2.0 * I * (9.0 * u2 + w2) * xi0);
    hu[1] = 2.0 * E + 4.0 * I * u * E + I * e * P1 - e * (2.0 * cw - 6.0 * I * u * xi0);
    hu[2] = 2.0 * I * E + I * e * P2 - e * (3.0 * I * xi0);
    g[0] = -2.0 * E + e * (-8.0 * u2 * xi0 + 2.0 * I * u * (2.0 * xi0 + (3.0 * u2 + w2) * xi1));
    g[1] = e * (2.0 * u * xi0 - 2.0 * I * xi0 + I * (3.0 * u2 - w2) * xi1);
    g[2] = e * (xi0 - 3.0 * I * u * xi1);
    double D = 9.0 * u2 - w2;
    for (int j = 0; j < 3; ++j) {
        cx fu = (hu[j] * D - 18.0 * u * h[j]) / (D * D);
        cx k = (g[j] * D + 2.0 * h[j]) / (D * D);
        f[j] = h[j] / D;
        d0[j] = (fu - 3.0 * u * k) / (2.0 * D);
        d1[j] = (u * fu + 0.5 * (3.0 * u2 - w2) * k) / D;
    }
    if (neg) {  /* f_j(Q) = (-1)^j conj(f_j(-Q)); c0 changes sign */
        f[0] = conj(f[0]); f[1] = -conj(f[1]); f[2] = conj(f[2]);
        d1[0] = conj(d1[0]); d1[1] = -conj(d1[1]); d1[2] = conj(d1[2]);
        d0[0] = -conj(d0[0]); d0[1] = conj(d0[1]); d0[2] = -conj(d0[2]);
    }
    return ORC_OK;
}

/* traceless Hermitian part */
static void m_th(const cx* a, cx* out)
{
    cx t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[i * 3 + j] = 0.5 * (a[i * 3 + j] + conj(a[j * 3 + i]));
    cx tr = m_tr(t) / 3.0;
    for (int i = 0; i < 9; ++i) out[i] = t[i];
    out[0] -= tr; out[4] -= tr; out[8] -= tr;
}

/* plaquette staple sum of link (s, mu), orientation as orc_stout */
static void stout_staple(const tab_t* t, const double* U, long s, int mu, cx* C)
{
    cx m1[9], m2[9];
    for (int i = 0; i < 9; ++i) C[i] = 0;
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        long xn = t->up[s * 4 + nu], xm = t->up[s * 4 + mu];
        long xd = t->dn[s * 4 + nu], xdm = t->up[xd * 4 + mu];
        m_mul(link_at(U, s, nu), link_at(U, xn, mu), m1);
        m_mul_adj(m1, link_at(U, xm, nu), m1);
        for (int i = 0; i < 9; ++i) C[i] += m1[i];
        m_adj(link_at(U, xd, nu), m2);
        m_mul(m2, link_at(U, xd, mu), m2);
        m_mul(m2, link_at(U, xdm, nu), m2);
        for (int i = 0; i < 9; ++i) C[i] += m2[i];
    }
}

/* out += a b c with each factor optionally adjoint */
static void acc3(cx* out, const cx* a, int ad, const cx* b, int bd, const cx* c, int cd)
{
    cx A[9], B[9], Cm[9], t1[9], t2[9];
    if (ad) m_adj(a, A); else memcpy(A, a, sizeof(A));
    if (bd) m_adj(b, B); else memcpy(B, b, sizeof(B));
    if (cd) m_adj(c, Cm); else memcpy(Cm, c, sizeof(Cm));
    m_mul(A, B, t1);
    m_mul(t1, Cm, t2);
    for (int i = 0; i < 9; ++i) out[i] += t2[i];
}

/* dS/dU of link m = (y, a) from the staple terms Re Tr(W_l dC_l) of every
 * link l whose staple contains m (six positions, three directions each). */
static void stout_gather(const tab_t* t, const double* U, const cx* W, long y, int a, cx* out)
{
#define LK(s, d) link_at(U, (s), (d))
#define WK(s, d) (W + ((s) * 4 + (d)) * 9)
#define UP(s, d) ((long)t->up[(s) * 4 + (d)])
#define DN(s, d) ((long)t->dn[(s) * 4 + (d)])
    for (int m = 0; m < 4; ++m) {
        if (m == a) continue;
        /* m is U_nu(x) of an upper staple of (x, mu): nu = a, x = y */
        acc3(out, LK(UP(y, a), m), 0, LK(UP(y, m), a), 1, WK(y, m), 0);
        /* m is U_mu(x+nu) of an upper staple: mu = a, x = y - nu */
        {
            long x = DN(y, m);
            acc3(out, LK(UP(x, a), m), 1, WK(x, a), 0, LK(x, m), 0);
        }
        /* m is U_nu(x+mu) of an upper staple: nu = a, x = y - mu */
        {
            long x = DN(y, m);
            cx t1[9];
            for (int i = 0; i < 9; ++i) t1[i] = 0;
            acc3(t1, WK(x, m), 0, LK(x, a), 0, LK(UP(x, a), m), 0);  /* (B^dag A^dag W^dag)^dag = W A B */
            cx t2[9];
            m_adj(t1, t2);
            for (int i = 0; i < 9; ++i) out[i] += t2[i];
        }
        /* m is U_nu(x-nu) of a lower staple: nu = a, x = y + a */
        {
            long x = UP(y, a);
            cx t1[9];
            for (int i = 0; i < 9; ++i) t1[i] = 0;
            acc3(t1, LK(y, m), 0, LK(UP(y, m), a), 0, WK(x, m), 0);  /* (W^dag G^dag F^dag)^dag = F G W */
            cx t2[9];
            m_adj(t1, t2);
            for (int i = 0; i < 9; ++i) out[i] += t2[i];
        }
        /* m is U_mu(x-nu) of a lower staple: mu = a, x = y + nu */
        acc3(out, LK(UP(y, a), m), 0, WK(UP(y, m), a), 0, LK(y, m), 1);
        /* m is U_nu(x-nu+mu) of a lower staple: nu = a, x = y + a - mu */
        {
            long z = DN(y, m); /* y - mu */
            long x = UP(z, a); /* y - mu + a */
            acc3(out, WK(x, m), 0, LK(z, a), 1, LK(z, m), 0);
        }
    }
#undef LK
#undef WK
#undef UP
#undef DN
}

int orc_stout_force(const int dims[4], double rho, int n_levels, const double* U_thin, const double* F_top,
                    double* F_thin)
{
    tab_t t;
    tab_build(&t, dims);
    long V = t.V, nl = 4 * V;
    double** lev = (double**)malloc(sizeof(double*) * (n_levels + 1));
    for (int k = 0; k <= n_levels; ++k) lev[k] = (double*)malloc(sizeof(double) * 72 * V);
    memcpy(lev[0], U_thin, sizeof(double) * 72 * V);
    int bad = 0;
    for (int k = 0; k < n_levels && !bad; ++k) {
        memcpy(lev[k + 1], lev[k], sizeof(double) * 72 * V);
        bad = orc_stout(dims, rho, 1, lev[k + 1]);
    }
    cx* G = (cx*)malloc(sizeof(cx) * 9 * nl);
    cx* Gn = (cx*)malloc(sizeof(cx) * 9 * nl);
    cx* W = (cx*)malloc(sizeof(cx) * 9 * nl);
    /* top: G = -2i V^dag F */
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nl; ++l) {
        cx vd[9], g[9];
        m_adj((const cx*)(lev[n_levels] + l * 18), vd);
        m_mul(vd, (const cx*)(F_top + l * 18), g);
        for (int i = 0; i < 9; ++i) G[l * 9 + i] = -2.0 * I * g[i];
    }
    for (int k = n_levels - 1; k >= 0 && !bad; --k) {
        const double* Uk = lev[k];
#pragma omp parallel for schedule(static) reduction(| : bad)
        for (long l = 0; l < nl; ++l) {
            long s = l / 4;
            int mu = (int)(l % 4);
            const cx* u = (const cx*)(Uk + l * 18);
            cx C[9], om[9], A[9], Q[9], Q2[9], B[9], eq[9];
            stout_staple(&t, Uk, s, mu, C);
            m_mul_adj(C, u, om);
            proj_ah(om, A);
            for (int i = 0; i < 9; ++i) Q[i] = -I * rho * A[i];
            cx f[3], d0[3], d1[3];
            if (expiq_coeffs(Q, f, d0, d1) != ORC_OK) { bad = 1; continue; }
            m_mul(Q, Q, Q2);
            for (int i = 0; i < 9; ++i) eq[i] = f[1] * Q[i] + f[2] * Q2[i];
            eq[0] += f[0]; eq[4] += f[0]; eq[8] += f[0];
            m_mul(u, G + l * 9, B);
            cx BQ[9], BQ2[9];
            m_mul(B, Q, BQ);
            m_mul(B, Q2, BQ2);
            cx tr[3] = {m_tr(B), m_tr(BQ), m_tr(BQ2)};
            cx b0 = 0, b1 = 0;
            for (int j = 0; j < 3; ++j) { b0 += tr[j] * d0[j]; b1 += tr[j] * d1[j]; }
            cx QB[9], Lh[9], L[9];
            m_mul(Q, B, QB);
            for (int i = 0; i < 9; ++i) Lh[i] = b0 * Q2[i] + b1 * Q[i] + f[1] * B[i] + f[2] * (QB[i] + BQ[i]);
            m_th(Lh, L);
            cx K[9], ud[9], w[9], g1[9], cd[9], g2[9];
            for (int i = 0; i < 9; ++i) K[i] = -I * rho * L[i];
            m_adj(u, ud);
            m_mul(ud, K, w);
            for (int i = 0; i < 9; ++i) W[l * 9 + i] = w[i];
            m_mul(G + l * 9, eq, g1);
            m_adj(C, cd);
            m_mul(cd, K, g2);
            for (int i = 0; i < 9; ++i) Gn[l * 9 + i] = g1[i] - g2[i];
        }
        if (bad) break;
#pragma omp parallel for schedule(static)
        for (long l = 0; l < nl; ++l) {
            cx acc[9];
            for (int i = 0; i < 9; ++i) acc[i] = 0;
            stout_gather(&t, Uk, W, l / 4, (int)(l % 4), acc);
            for (int i = 0; i < 9; ++i) G[l * 9 + i] = Gn[l * 9 + i] + acc[i];
        }
    }
    if (!bad) {
#pragma omp parallel for schedule(static)
        for (long l = 0; l < nl; ++l) {
            cx ug[9], iug[9], f[9];
            m_mul((const cx*)(lev[0] + l * 18), G + l * 9, ug);
            for (int i = 0; i < 9; ++i) iug[i] = I * ug[i];
            m_th(iug, f);
            for (int i = 0; i < 9; ++i) ((cx*)(F_thin + l * 18))[i] = 0.5 * f[i];
        }
    }
    free(G); free(Gn); free(W);
    for (int k = 0; k <= n_levels; ++k) free(lev[k]);
    free(lev);
    tab_free(&t);
    return bad ? ORC_ERR_DOMAIN : ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* heatbath: Cabibbo-Marinari SU(2) subgroups (Lattice.cpp:614-757,          */
/* SU3_Sampling.cpp:17-199)                                                  */
/* ------------------------------------------------------------------------ */
/*
 * single_link_heatbath restated per link: A = c11 A1 + c12 A2; for the
 * subgroups R (rows/cols 0,1), S (0,2), T (1,2) in turn: W = the SU(2)
 * projection of that 2x2 block of U A, a = sqrt(det W); a <= 1e-14: R a
 * uniform SU(2) element, else X from the sampler with (a, 2 beta / 3) and
 * R = X (W/a)^dag; U <- R U.
 * Order: the reference sweeps lexicographically; here (as on the GPU) one
 * direction mu at a time and, within it, eight colours
 * (x_mu mod 2) * 4 + (sum_{nu != mu} x_nu mod 4) of links whose staples do not
 * contain each other (needs every extent divisible by 4).  The uniforms are
 * Philox-4x32-10 (Salmon et al., SC'11) keyed by the seed, counter
 * (link, draw, sweep, 0x48420000 + subgroup), 53-bit doubles in [0, 1);
 * the reference's generator is unseeded, so parity with it is statistical.
 */
static void philox_4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1, n3 = (uint32_t)p0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

typedef struct {
    uint32_t k0, k1, link, sweep, tag, draw;
    double buf[2];
    int have;
} hb_rng;

static double hb_u(hb_rng* r)  /* uniform in [0, 1) */
{
    if (r->have == 0) {
        uint32_t c[4] = {r->link, r->draw++, r->sweep, r->tag};
        philox_4x32_10(c, r->k0, r->k1);
        uint64_t a = (((uint64_t)c[0] << 21) ^ (uint64_t)(c[1] >> 11)) & ((1ull << 53) - 1);
        uint64_t b = (((uint64_t)c[2] << 21) ^ (uint64_t)(c[3] >> 11)) & ((1ull << 53) - 1);
        r->buf[0] = (double)a * (1.0 / 9007199254740992.0);
        r->buf[1] = (double)b * (1.0 / 9007199254740992.0);
        r->have = 2;
    }
    return r->buf[2 - r->have--];
}

/* SU3_Sampling.cpp:17-31 (generate_x0) */
static double hb_x0(hb_rng* r, double a, double beta)
{
    for (;;) {
        double r1 = 1.0 - hb_u(r), r2 = 1.0 - hb_u(r), r3 = 1.0 - hb_u(r);
        double c = cos(2.0 * 3.14159265358979323846 * r2);
        double l2 = -1.0 / (2.0 * a * beta) * (log(r1) + c * c * log(r3));
        double x = 1.0 - l2;
        double rr = hb_u(r);
        if (rr * rr <= x && x >= -1.0 && x <= 1.0) return 1.0 - 2.0 * l2;
    }
}

/* SU3_Sampling.cpp:42-58 / 152-168: uniform unit vector by rejection */
static void hb_unit(hb_rng* r, double* v, int n)
{
    for (;;) {
        double len2 = 0.0;
        for (int k = 0; k < n; ++k) {
            v[k] = 2.0 * hb_u(r) - 1.0;
            len2 += v[k] * v[k];
        }
        double len = sqrt(len2);
        if (len <= 1.0 && len > 0.0) {
            for (int k = 0; k < n; ++k) v[k] /= len;
            return;
        }
    }
}

/* 2x2 (row-major) from quaternion q: q0 I + i (q1 sx + q2 sy + q3 sz) */
static void quat_su2(const double q[4], cx m[4])
{
    m[0] = q[0] + I * q[3];
    m[1] = q[2] + I * q[1];
    m[2] = -q[2] + I * q[1];
    m[3] = q[0] - I * q[3];
}

static void hb_subgroup(hb_rng* r, cx* U, const cx* A, int i, int j, double beta)
{
    cx UA[9];
    m_mul(U, A, UA);
    cx b[4] = {UA[i * 3 + i], UA[i * 3 + j], UA[j * 3 + i], UA[j * 3 + j]};
    /* SU(2) projection (Lattice.cpp:570-598): w0 = Re tr/2, w_k from the
     * anti-Hermitian part */
    double w0 = 0.5 * creal(b[0] + b[3]);
    double w1 = 0.5 * cimag(b[1] + b[2]);
    double w2 = 0.5 * creal(b[1] - b[2]);
    double w3 = 0.5 * cimag(b[0] - b[3]);
    double a = sqrt(w0 * w0 + w1 * w1 + w2 * w2 + w3 * w3);
    cx R[4];
    if (a <= 1e-14) {
        double q[4];
        hb_unit(r, q, 4);
        quat_su2(q, R);
    } else {
        double x0 = hb_x0(r, a, 2.0 * beta / 3.0);
        double v[3];
        hb_unit(r, v, 3);
        double nx = sqrt(1.0 - x0 * x0);
        double qx[4] = {x0, nx * v[0], nx * v[1], nx * v[2]};
        double qw[4] = {w0 / a, -w1 / a, -w2 / a, -w3 / a};  /* (W/a)^dag */
        cx X[4], Wd[4];
        quat_su2(qx, X);
        quat_su2(qw, Wd);
        R[0] = X[0] * Wd[0] + X[1] * Wd[2];
        R[1] = X[0] * Wd[1] + X[1] * Wd[3];
        R[2] = X[2] * Wd[0] + X[3] * Wd[2];
        R[3] = X[2] * Wd[1] + X[3] * Wd[3];
    }
    cx E[9], out[9];
    m_id(E);
    E[i * 3 + i] = R[0]; E[i * 3 + j] = R[1];
    E[j * 3 + i] = R[2]; E[j * 3 + j] = R[3];
    m_mul(E, U, out);
    memcpy(U, out, sizeof(out));
}

int orc_heatbath(const int dims[4], double beta, double c11, double c12, unsigned long long seed, int sweep0,
                 int nsweeps, double* U)
{
    for (int k = 0; k < 4; ++k)
        if (dims[k] % 4) return ORC_ERR_DOMAIN;
    tab_t t;
    tab_build(&t, dims);
    long V = t.V;
    for (int sw = sweep0; sw < sweep0 + nsweeps; ++sw)
        for (int mu = 0; mu < 4; ++mu)
            for (int col = 0; col < 8; ++col)
#pragma omp parallel for schedule(static)
                for (long s = 0; s < V; ++s) {
                    int c[4];
                    coords_of(t.L, s, c);
                    int sum = 0;
                    for (int nu = 0; nu < 4; ++nu)
                        if (nu != mu) sum += c[nu];
                    if ((c[mu] & 1) * 4 + (sum & 3) != col) continue;
                    cx A1[9], A2[9], A[9];
                    staple_plaq(&t, U, s, mu, A1);
                    staple_rect(&t, U, s, mu, A2);
                    for (int i = 0; i < 9; ++i) A[i] = c11 * A1[i] + c12 * A2[i];
                    cx* u = (cx*)(U + (s * 4 + mu) * 18);
                    const int sub[3][2] = {{0, 1}, {0, 2}, {1, 2}};
                    for (int g = 0; g < 3; ++g) {
                        hb_rng r = {(uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)(s * 4 + mu),
                                    (uint32_t)sw, 0x48420000u + (uint32_t)g, 0, {0, 0}, 0};
                        hb_subgroup(&r, u, A, sub[g][0], sub[g][1], beta);
                    }
                }
    tab_free(&t);
    return ORC_OK;
}

/* HEX, Smearing.cpp:76-311.  Decorated fields are stored as
 * [combo][site][9] with combo = (4 mu + nu) 4 + rho (level 1),
 * 4 mu + nu (level 2), mu (level 3), as in the reference's flat indices
 * (Smearing.cpp:14-73).  The staple steps are exposed on their own
 * (orc_hex_gamma1/2/3) so that they can be checked against the reference's
 * apply_step_1/3/5, which run unmodified; the exp steps cannot (see
 * orc_hex). */
#define LNK(s, mu) (Uc + ((long)(s) * 4 + (mu)) * 9)
#define F3(arr, a, b, c, s) ((arr) + ((((long)(a) * 4 + (b)) * 4 + (c)) * V + (s)) * 9)
#define F2(arr, a, b, s) ((arr) + (((long)(a) * 4 + (b)) * V + (s)) * 9)

/* step 1 (Smearing.cpp:76-123): G1[mu,nu,rho](x) = sum over sigma not in
 * {mu, nu, rho} of the up and down staples of U from x to x+mu */
static void hex_gamma1(const tab_t* t, const cx* Uc, cx* G1)
{
    const long V = t->V;
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s)
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = 0; nu < 4; ++nu)
                for (int rh = 0; rh < 4; ++rh) {
                    cx* g = F3(G1, mu, nu, rh, s);
                    for (int i = 0; i < 9; ++i) g[i] = 0;
                    for (int sg = 0; sg < 4; ++sg) {
                        if (sg == mu || sg == nu || sg == rh) continue;
                        long xs = t->up[s * 4 + sg], xm = t->up[s * 4 + mu];
                        long xd = t->dn[s * 4 + sg], xdm = t->up[xd * 4 + mu];
                        cx a[9], b[9];
                        m_mul(LNK(s, sg), LNK(xs, mu), a);
                        m_mul_adj(a, LNK(xm, sg), a);
                        m_adj(LNK(xd, sg), b);
                        m_mul(b, LNK(xd, mu), b);
                        m_mul(b, LNK(xdm, sg), b);
                        for (int i = 0; i < 9; ++i) g[i] += a[i] + b[i];
                    }
                }
}

/* step 3 (Smearing.cpp:157-209): G2[mu,nu](x) = sum over sigma not in
 * {mu, nu} of staples with side links V1[sigma,mu,nu] and middle link
 * V1[mu,nu,sigma] */
static void hex_gamma2(const tab_t* t, const cx* V1, cx* G2)
{
    const long V = t->V;
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s)
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = 0; nu < 4; ++nu) {
                cx* g = F2(G2, mu, nu, s);
                for (int i = 0; i < 9; ++i) g[i] = 0;
                for (int sg = 0; sg < 4; ++sg) {
                    if (sg == mu || sg == nu) continue;
                    long xs = t->up[s * 4 + sg], xm = t->up[s * 4 + mu];
                    long xd = t->dn[s * 4 + sg], xdm = t->up[xd * 4 + mu];
                    cx a[9], b[9];
                    m_mul(F3(V1, sg, mu, nu, s), F3(V1, mu, nu, sg, xs), a);
                    m_mul_adj(a, F3(V1, sg, mu, nu, xm), a);
                    m_adj(F3(V1, sg, mu, nu, xd), b);
                    m_mul(b, F3(V1, mu, nu, sg, xd), b);
                    m_mul(b, F3(V1, sg, mu, nu, xdm), b);
                    for (int i = 0; i < 9; ++i) g[i] += a[i] + b[i];
                }
            }
}

/* step 5 (Smearing.cpp:236-275), Gamma_3 starting at zero: G3[mu](x) =
 * sum over nu != mu of staples with side links V2[nu,mu] and middle link
 * V2[mu,nu]; G3 as [mu][site][9] */
static void hex_gamma3(const tab_t* t, const cx* V2, cx* G3)
{
    const long V = t->V;
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s)
        for (int mu = 0; mu < 4; ++mu) {
            cx* g = G3 + ((long)mu * V + s) * 9;
            for (int i = 0; i < 9; ++i) g[i] = 0;
            for (int nu = 0; nu < 4; ++nu) {
                if (nu == mu) continue;
                long xn = t->up[s * 4 + nu], xm = t->up[s * 4 + mu];
                long xd = t->dn[s * 4 + nu], xdm = t->up[xd * 4 + mu];
                cx a[9], b[9];
                m_mul(F2(V2, nu, mu, s), F2(V2, mu, nu, xn), a);
                m_mul_adj(a, F2(V2, nu, mu, xm), a);
                m_adj(F2(V2, nu, mu, xd), b);
                m_mul(b, F2(V2, mu, nu, xd), b);
                m_mul(b, F2(V2, nu, mu, xdm), b);
                for (int i = 0; i < 9; ++i) g[i] += a[i] + b[i];
            }
        }
}

void orc_hex_gamma1(const int dims[4], const double* U, double* G1)
{
    tab_t t;
    tab_build(&t, dims);
    hex_gamma1(&t, (const cx*)U, (cx*)G1);
    tab_free(&t);
}

void orc_hex_gamma2(const int dims[4], const double* V1, double* G2)
{
    tab_t t;
    tab_build(&t, dims);
    hex_gamma2(&t, (const cx*)V1, (cx*)G2);
    tab_free(&t);
}

void orc_hex_gamma3(const int dims[4], const double* V2, double* G3)
{
    tab_t t;
    tab_build(&t, dims);
    hex_gamma3(&t, (const cx*)V2, (cx*)G3);
    tab_free(&t);
}

int orc_hex(const int dims[4], const double alphas[3], double* U)
{
    tab_t t;
    tab_build(&t, dims);
    long V = t.V;
    const cx* Uc = (const cx*)U;
    cx* G1 = (cx*)malloc(sizeof(cx) * 9 * 64 * V);
    cx* V1 = (cx*)malloc(sizeof(cx) * 9 * 64 * V);
    cx* G2 = (cx*)malloc(sizeof(cx) * 9 * 16 * V);
    cx* V2 = (cx*)malloc(sizeof(cx) * 9 * 16 * V);
    cx* G3 = (cx*)malloc(sizeof(cx) * 9 * 4 * V);
    cx* Unew = (cx*)malloc(sizeof(cx) * 9 * 4 * V);
    int bad = 0;
    hex_gamma1(&t, Uc, G1);
    /* step 2 (Smearing.cpp:132-155) */
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (long s = 0; s < V; ++s)
        for (int c = 0; c < 64; ++c) {
            int mu = c / 16;
            if (smear_link(G1 + ((long)c * V + s) * 9, LNK(s, mu),
                           alphas[2] * 0.5, V1 + ((long)c * V + s) * 9) != ORC_OK)
                bad = 1;
        }
    hex_gamma2(&t, V1, G2);
    /* step 4 (Smearing.cpp:213-234) */
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (long s = 0; s < V; ++s)
        for (int c = 0; c < 16; ++c) {
            int mu = c / 4;
            if (smear_link(G2 + ((long)c * V + s) * 9, LNK(s, mu),
                           alphas[1] * 0.5, V2 + ((long)c * V + s) * 9) != ORC_OK)
                bad = 1;
        }
    hex_gamma3(&t, V2, G3);
    /* step 6 (Smearing.cpp:278-301) */
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (long s = 0; s < V; ++s)
        for (int mu = 0; mu < 4; ++mu)
            if (smear_link(G3 + ((long)mu * V + s) * 9, LNK(s, mu), alphas[0] * 0.5,
                           Unew + ((long)s * 4 + mu) * 9) != ORC_OK)
                bad = 1;
    if (!bad) memcpy(U, Unew, sizeof(cx) * 9 * 4 * V);
    free(G1); free(V1); free(G2); free(V2); free(G3); free(Unew);
    tab_free(&t);
    return bad ? ORC_ERR_DOMAIN : ORC_OK;
}
#undef LNK
#undef F3
#undef F2

/* ------------------------------------------------------------------------ */
/* seeded generators (the library's, restated on the CPU)                   */
/* ------------------------------------------------------------------------ */
/*
 * The reference draws its fields from an unseeded std::mt19937
 * (rng.cpp:7-15): the Gaussian Hermitian generator of
 * random_traceless_hermitian_SU3 (Lattice.cpp:1001-1033), complex Gaussian
 * spinors (generateGaussianComplex, Fermions.cpp:207-212) and momenta
 * P = sum_a 1/2 p_a lambda_a (generate_conjugate_field_configuration,
 * Fermions.cpp:342-360).  The library keeps those distributions but draws
 * from Philox-4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11; checked here
 * against the published known-answer vectors) keyed by the seed, with one
 * counter per object: (id_lo, id_hi, k, stream), id = site (spinors) or
 * 4 site + mu (links), k = pair index, stream 1 gauge, 2 spinor, 3 momenta.
 * Each block gives two N(0,1) by Box-Muller from two 53-bit uniforms in
 * (0, 1).  These functions give the same fields on the CPU, so both sides
 * of a comparison start from identical inputs (to the last few ulps: the
 * log and sin/cos of the C library and of CUDA may differ in the last bit).
 */
void orc_philox4x32_10(const unsigned ctr[4], const unsigned key[2], unsigned out[4])
{
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox_4x32_10(c, key[0], key[1]);
    for (int i = 0; i < 4; ++i) out[i] = c[i];
}

static void gen_normals(unsigned long long seed, uint32_t stream, unsigned long long id, int n, double* z)
{
    const double inv53 = 1.0 / 9007199254740992.0;
    for (int k = 0; k < (n + 1) / 2; ++k) {
        uint32_t c[4] = {(uint32_t)id, (uint32_t)(id >> 32), (uint32_t)k, stream};
        philox_4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        uint64_t a = (((uint64_t)c[0] << 21) ^ (uint64_t)(c[1] >> 11)) & ((1ull << 53) - 1);
        uint64_t b = (((uint64_t)c[2] << 21) ^ (uint64_t)(c[3] >> 11)) & ((1ull << 53) - 1);
        double u1 = ((double)a + 0.5) * inv53, u2 = ((double)b + 0.5) * inv53;
        double rad = sqrt(-2.0 * log(u1));
        double ang = 2.0 * 3.14159265358979323846 * u2;
        z[2 * k] = rad * cos(ang);
        if (2 * k + 1 < n) z[2 * k + 1] = rad * sin(ang);
    }
}

void orc_gen_normals(unsigned long long seed, unsigned stream, unsigned long long id, int n, double* z)
{
    gen_normals(seed, stream, id, n, z);
}

int orc_gen_gauge(const int dims[4], double eps, unsigned long long seed, double* U)
{
    const long n = 4L * dims[0] * dims[1] * dims[2] * dims[3];
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (long l = 0; l < n; ++l) {  /* l = 4 s + mu */
        double z[9];
        gen_normals(seed, 1u, (unsigned long long)l, 9, z);
        const double tr3 = (z[0] + z[1] + z[2]) / 3.0;
        cx H[9];
        H[0] = z[0] - tr3;
        H[4] = z[1] - tr3;
        H[8] = z[2] - tr3;
        H[1] = z[3] + I * z[4];
        H[3] = z[3] - I * z[4];
        H[2] = z[5] + I * z[6];
        H[6] = z[5] - I * z[6];
        H[5] = z[7] + I * z[8];
        H[7] = z[7] - I * z[8];
        for (int k = 0; k < 9; ++k) H[k] *= eps;
        if (expiq_cx(H, (cx*)(U + l * 18)) != ORC_OK) bad = 1;
    }
    return bad ? ORC_ERR_DOMAIN : ORC_OK;
}

void orc_gen_spinor(const int dims[4], double sigma, unsigned long long seed, double* out)
{
    const long V = (long)dims[0] * dims[1] * dims[2] * dims[3];
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        double z[6];
        gen_normals(seed, 2u, (unsigned long long)s, 6, z);
        for (int k = 0; k < 6; ++k) out[s * 6 + k] = sigma * z[k];
    }
}

void orc_gen_momenta(const int dims[4], unsigned long long seed, double* P)
{
    const long n = 4L * dims[0] * dims[1] * dims[2] * dims[3];
    const double a8 = 1.0 / sqrt(3.0);
#pragma omp parallel for schedule(static)
    for (long l = 0; l < n; ++l) {
        double z[8];
        gen_normals(seed, 3u, (unsigned long long)l, 8, z);
        /* 1/2 sum_a p_a lambda_a, Gell-Mann basis of Fermions.cpp:321-340 */
        cx M[9];
        M[0] = z[2] + a8 * z[7];
        M[4] = -z[2] + a8 * z[7];
        M[8] = -2.0 * a8 * z[7];
        M[1] = z[0] - I * z[1];
        M[3] = z[0] + I * z[1];
        M[2] = z[3] - I * z[4];
        M[6] = z[3] + I * z[4];
        M[5] = z[5] - I * z[6];
        M[7] = z[5] + I * z[6];
        cx* o = (cx*)(P + l * 18);
        for (int k = 0; k < 9; ++k) o[k] = 0.5 * M[k];
    }
}

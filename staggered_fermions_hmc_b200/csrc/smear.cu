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

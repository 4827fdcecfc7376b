// generate.cu — seeded device generators for gauge fields, spinors and
// momenta.  The reference seeds from std::random_device (rng.cpp:7-15) and is
// not reproducible; these generators are keyed by (seed, object id) with
// Philox-4x32-10, so a field does not depend on the launch shape.
//
//   gauge:    U = exp(i eps H), H traceless Hermitian with N(0,1) entries
//             (the distribution of Lattice.cpp:1001-1033)
//   spinor:   iid N(0, sigma^2) per real component
//   momenta:  P = sum_a 1/2 p_a lambda_a, p_a ~ N(0,1) (Fermions.cpp:342-360)
#include "sfh_internal.h"
#include "su3.cuh"

namespace sfh {

namespace {

enum { STREAM_GAUGE = 1, STREAM_SPINOR = 2, STREAM_MOMENTA = 3 };

__global__ void random_gauge_kernel(Geom g, double eps, unsigned long long seed, void* U, int* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    Coord c = eo_coords(g, p, i);
    M3 H = random_hermitian(seed, STREAM_GAUGE, (unsigned long long)c.lex * 4 + mu);
#pragma unroll
    for (int k = 0; k < 9; ++k) H.e[k] = cscale(H.e[k], eps);
    M3 E;
    if (!expiq(H, E)) {
        atomicOr(err, DEV_ERR_DOMAIN);
        E = m3_id();
    }
    st_link(U, p, mu, i, g.Vh, E);
}

__global__ void random_spinor_kernel(Geom g, double sigma, unsigned long long seed, double2* out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y;
    if (i >= g.Vh) return;
    Coord c = eo_coords(g, p, i);
    double z[6];
    normals<6>(seed, STREAM_SPINOR, (unsigned long long)c.lex, z);
    double2* b = out + (size_t)p * 3 * g.Vh + i;
#pragma unroll
    for (int k = 0; k < 3; ++k) b[(size_t)k * g.Vh] = make_double2(sigma * z[2 * k], sigma * z[2 * k + 1]);
}

__global__ void random_momenta_kernel(Geom g, unsigned long long seed, void* P)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    Coord c = eo_coords(g, p, i);
    double z[8];
    normals<8>(seed, STREAM_MOMENTA, (unsigned long long)c.lex * 4 + mu, z);
    // P = 1/2 sum_a p_a lambda_a with the Gell-Mann basis (Fermions.cpp:321-340)
    const double a8 = 1.0 / sqrt(3.0);
    M3 M = m3_zero();
    M.e[1] = {z[0], -z[1]};
    M.e[3] = {z[0], z[1]};
    M.e[0].re = z[2] + a8 * z[7];
    M.e[4].re = -z[2] + a8 * z[7];
    M.e[2] = {z[3], -z[4]};
    M.e[6] = {z[3], z[4]};
    M.e[5] = {z[5], -z[6]};
    M.e[7] = {z[5], z[6]};
    M.e[8].re = -2.0 * a8 * z[7];
#pragma unroll
    for (int k = 0; k < 9; ++k) M.e[k] = cscale(M.e[k], 0.5);
    st_link(P, p, mu, i, g.Vh, M);
}

}  // namespace

cudaError_t launch_random_gauge(const Geom& g, double eps, unsigned long long seed, void* U, int* d_err,
                                cudaStream_t s)
{
    random_gauge_kernel<<<dim3((g.Vh + 127) / 128, 8), 128, 0, s>>>(g, eps, seed, U, d_err);
    return cudaGetLastError();
}

cudaError_t launch_random_spinor(const Geom& g, double sigma, unsigned long long seed, void* out,
                                 cudaStream_t s)
{
    random_spinor_kernel<<<dim3((g.Vh + 255) / 256, 2), 256, 0, s>>>(g, sigma, seed, (double2*)out);
    return cudaGetLastError();
}

cudaError_t launch_random_momenta(const Geom& g, unsigned long long seed, void* P, cudaStream_t s)
{
    random_momenta_kernel<<<dim3((g.Vh + 127) / 128, 8), 128, 0, s>>>(g, seed, P);
    return cudaGetLastError();
}

}  // namespace sfh

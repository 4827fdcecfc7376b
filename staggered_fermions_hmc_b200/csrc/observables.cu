// observables.cu — Polyakov loop grid and correlator, gauge checkpoint files.
//
// Polyakov loop P(x,y,z) = Tr prod_{t=0}^{Lt-1} U_t(x,y,z,t), right-multiplied
// and not normalised (poly_loop_at_spat_coord, Lattice.cpp:849-865); the grid
// is precompute_polyakov_grid (Lattice.cpp:869-882).  The correlator at
// squared distance r2 averages P(m) conj(P(m+d)) over all spatial sites m and
// displacements d with |d|^2 = r2, |d_i| <= min(floor(sqrt(r2)), L_i/2) and
// d_i != L_i/2 for even L_i (correlator_over_fixed_distance_fast,
// Lattice.cpp:886-948; the reference has one spatial size, here each
// direction uses its own).
//
// Checkpoints are the reference's raw format: the link array in its own
// layout as native doubles (save_all_lattice_configs / load_all_lattice_configs
// for one coupling, Lattice.cpp:810-847).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "sfh_internal.h"
#include "walk.cuh"

namespace sfh {
int set_error(sfh_ctx* c, int code, const std::string& msg);
int cuda_check(sfh_ctx* c, cudaError_t e, const char* what);
}  // namespace sfh

using namespace sfh;

namespace {

__global__ void polyakov_grid_kernel(Geom g, const void* U, double2* out)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    int ns = g.L[0] * g.L[1] * g.L[2];
    if (s >= ns) return;
    Walker w;
    w.x[2] = s % g.L[2];
    w.x[1] = (s / g.L[2]) % g.L[1];
    w.x[0] = s / (g.L[1] * g.L[2]);
    w.x[3] = 0;
    M3 m = m3_id();
    for (int t = 0; t < g.L[3]; ++t) {
        w.x[3] = t;
        m = m3_mul(m, link_at(U, g, w, 3));
    }
    Cx<double> tr = m3_tr(m);
    out[s] = make_double2(tr.re, tr.im);
}

// per spatial site m: sum over displacements of P(m) conj(P(m+d))
__global__ void polyakov_corr_kernel(Geom g, const double2* grid, const int* disp, int ndisp, double2* partial)
{
    __shared__ double sre[256], sim[256];
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    int ns = g.L[0] * g.L[1] * g.L[2];
    double re = 0.0, im = 0.0;
    if (s < ns) {
        int z = s % g.L[2], y = (s / g.L[2]) % g.L[1], x = s / (g.L[1] * g.L[2]);
        double2 pm = grid[s];
        for (int k = 0; k < ndisp; ++k) {
            int nx = (x + disp[3 * k] + g.L[0]) % g.L[0];
            int ny = (y + disp[3 * k + 1] + g.L[1]) % g.L[1];
            int nz = (z + disp[3 * k + 2] + g.L[2]) % g.L[2];
            double2 pn = grid[(nx * g.L[1] + ny) * g.L[2] + nz];
            re += pm.x * pn.x + pm.y * pn.y;  // P_m conj(P_n)
            im += pm.y * pn.x - pm.x * pn.y;
        }
    }
    sre[threadIdx.x] = re;
    sim[threadIdx.x] = im;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sre[threadIdx.x] += sre[threadIdx.x + o];
            sim[threadIdx.x] += sim[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(sre[0], sim[0]);
}

}  // namespace

extern "C" int sfh_polyakov_grid(sfh_ctx* c, double* out)
{
    if (!c || !out) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int ns = c->g.L[0] * c->g.L[1] * c->g.L[2];
    double2* d = (double2*)c->stage;
    polyakov_grid_kernel<<<(ns + 127) / 128, 128, 0, c->stream>>>(c->g, c->U64, d);
    int st = cuda_check(c, cudaGetLastError(), "polyakov grid");
    if (!st) st = cuda_check(c, cudaMemcpyAsync(out, d, sizeof(double2) * ns, cudaMemcpyDeviceToHost, c->stream),
                             "polyakov grid");
    if (!st) st = cuda_check(c, cudaStreamSynchronize(c->stream), "polyakov grid");
    return st;
}

namespace {

// displacements d with |d|^2 = r2, |d_i| <= min(floor(sqrt(r2)), L_i/2) and
// d_i != L_i/2 for even L_i (Lattice.cpp:893-915)
std::vector<int> correlator_displacements(const int* L, int r2)
{
    std::vector<int> disp;
    int root = (int)std::sqrt((double)r2);
    int md[3];
    for (int k = 0; k < 3; ++k) md[k] = std::min(root, L[k] / 2);
    for (int dx = -md[0]; dx <= md[0]; ++dx) {
        if (dx == L[0] / 2 && L[0] % 2 == 0) continue;
        for (int dy = -md[1]; dy <= md[1]; ++dy) {
            if (dy == L[1] / 2 && L[1] % 2 == 0) continue;
            for (int dz = -md[2]; dz <= md[2]; ++dz) {
                if (dz == L[2] / 2 && L[2] % 2 == 0) continue;
                if (dx * dx + dy * dy + dz * dz == r2) {
                    disp.push_back(dx);
                    disp.push_back(dy);
                    disp.push_back(dz);
                }
            }
        }
    }
    return disp;
}

// correlator over the grid already in stage (or copied there from host_grid)
int correlator_on_stage(sfh_ctx* c, const double* host_grid, int r2, double* out2)
{
    const int* L = c->g.L;
    std::vector<int> disp = correlator_displacements(L, r2);
    out2[0] = out2[1] = 0.0;
    int nd = (int)disp.size() / 3;
    if (nd == 0) return SFH_OK;  // Lattice.cpp:910
    int ns = L[0] * L[1] * L[2];
    int nb = (ns + 255) / 256;
    double2* grid = (double2*)c->stage;
    double2* part = grid + ns;
    int* ddisp = (int*)(part + nb);
    int st = SFH_OK;
    if (host_grid)
        st = cuda_check(c, cudaMemcpyAsync(grid, host_grid, sizeof(double2) * ns, cudaMemcpyHostToDevice, c->stream),
                        "polyakov correlator");
    else
        polyakov_grid_kernel<<<(ns + 127) / 128, 128, 0, c->stream>>>(c->g, c->U64, grid);
    if (!st) st = cuda_check(c, cudaMemcpyAsync(ddisp, disp.data(), sizeof(int) * disp.size(), cudaMemcpyHostToDevice,
                                               c->stream), "polyakov correlator");
    if (st) return st;
    polyakov_corr_kernel<<<nb, 256, 0, c->stream>>>(c->g, grid, ddisp, nd, part);
    std::vector<double2> hp(nb);
    st = cuda_check(c, cudaMemcpyAsync(hp.data(), part, sizeof(double2) * nb, cudaMemcpyDeviceToHost, c->stream),
                    "polyakov correlator");
    if (!st) st = cuda_check(c, cudaStreamSynchronize(c->stream), "polyakov correlator");
    if (st) return st;
    double re = 0.0, im = 0.0;
    for (const double2& v : hp) {
        re += v.x;
        im += v.y;
    }
    double n = (double)ns * nd;
    out2[0] = re / n;
    out2[1] = im / n;
    return SFH_OK;
}

}  // namespace

extern "C" int sfh_polyakov_correlator(sfh_ctx* c, int r2, double* out2)
{
    if (!c || !out2 || r2 < 0) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    return correlator_on_stage(c, nullptr, r2, out2);
}

extern "C" int sfh_polyakov_correlator_grid(sfh_ctx* c, const double* grid, int r2, double* out2)
{
    if (!c || !grid || !out2 || r2 < 0) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    return correlator_on_stage(c, grid, r2, out2);
}

extern "C" int sfh_save_gauge(sfh_ctx* c, const char* path)
{
    if (!c || !path) return SFH_ERR_INVALID;
    std::vector<double> h((size_t)c->g.V * 72);
    int st = sfh_download_gauge(c, h.data());
    if (st) return st;
    FILE* f = std::fopen(path, "wb");
    if (!f) return set_error(c, SFH_ERR_IO, std::string("Error opening file for writing: ") + path);
    size_t n = std::fwrite(h.data(), sizeof(double), h.size(), f);
    int closed = std::fclose(f);
    if (n != h.size() || closed != 0)
        return set_error(c, SFH_ERR_IO, std::string("Error writing complete binary data to: ") + path);
    return SFH_OK;
}

extern "C" int sfh_load_gauge(sfh_ctx* c, const char* path)
{
    if (!c || !path) return SFH_ERR_INVALID;
    std::vector<double> h((size_t)c->g.V * 72);
    FILE* f = std::fopen(path, "rb");
    if (!f) return set_error(c, SFH_ERR_IO, std::string("Error opening file for reading: ") + path);
    size_t n = std::fread(h.data(), sizeof(double), h.size(), f);
    std::fclose(f);
    if (n != h.size())
        return set_error(c, SFH_ERR_IO, std::string("Error reading complete binary data from: ") + path);
    return sfh_upload_gauge(c, h.data());
}

// layout.cu — conversion between the reference's host layouts and the
// device even-odd structure-of-arrays layouts, and derivation of the
// reduced-precision gauge copies.
//
// Reference layouts (converted only at the C ABI boundary):
//   links / momenta / forces : [site][mu][row][col][re,im]  (Lattice.cpp:135-168)
//   spinors                  : [site][color][re,im]          (Fermions.cpp:99-116)
#include "sfh_internal.h"

namespace sfh {

namespace {

constexpr int kThreads = 256;

inline int blocks_for(long n) { return (int)((n + kThreads - 1) / kThreads); }

// one thread per (parity, checkerboard site)
__global__ void spinor_aos_to_eo(Geom g, const double* __restrict__ aos, double2* __restrict__ eo)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y;
    if (i >= g.Vh) return;
    Coord c = eo_coords(g, p, i);
    const double2* src = reinterpret_cast<const double2*>(aos) + (size_t)c.lex * 3;
    double2* dst = eo + (size_t)p * 3 * g.Vh + i;
#pragma unroll
    for (int k = 0; k < 3; ++k) dst[(size_t)k * g.Vh] = src[k];
}

__global__ void spinor_eo_to_aos(Geom g, const double2* __restrict__ eo, double* __restrict__ aos)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y;
    if (i >= g.Vh) return;
    Coord c = eo_coords(g, p, i);
    double2* dst = reinterpret_cast<double2*>(aos) + (size_t)c.lex * 3;
    const double2* src = eo + (size_t)p * 3 * g.Vh + i;
#pragma unroll
    for (int k = 0; k < 3; ++k) dst[k] = src[(size_t)k * g.Vh];
}

// one thread per (parity, site, mu)
__global__ void links_aos_to_eo(Geom g, const double* __restrict__ aos, double2* __restrict__ eo)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    Coord c = eo_coords(g, p, i);
    const double2* src = reinterpret_cast<const double2*>(aos) + ((size_t)c.lex * 4 + mu) * 9;
    double2* dst = eo + ((size_t)(p * 4 + mu) * 9) * g.Vh + i;
#pragma unroll
    for (int k = 0; k < 9; ++k) dst[(size_t)k * g.Vh] = src[k];
}

__global__ void links_eo_to_aos(Geom g, const double2* __restrict__ eo, double* __restrict__ aos)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int p = blockIdx.y >> 2, mu = blockIdx.y & 3;
    if (i >= g.Vh) return;
    Coord c = eo_coords(g, p, i);
    double2* dst = reinterpret_cast<double2*>(aos) + ((size_t)c.lex * 4 + mu) * 9;
    const double2* src = eo + ((size_t)(p * 4 + mu) * 9) * g.Vh + i;
#pragma unroll
    for (int k = 0; k < 9; ++k) dst[k] = src[(size_t)k * g.Vh];
}

// FP64 18-real -> FP32 12-real (float4 x3), FP16 / BF16 12-real (uint2 x3)
// and FP32 18-real, each where its output is given
__global__ void make_lowp(Geom g, const double2* __restrict__ U64, float4* __restrict__ U32,
                          uint2* __restrict__ U16, float2* __restrict__ U32_18, uint2* __restrict__ Ubf16)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int pm = blockIdx.y;  // p*4+mu
    if (i >= g.Vh) return;
    const double2* src = U64 + (size_t)pm * 9 * g.Vh + i;
    if (U32_18)
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            double2 a = src[(size_t)k * g.Vh];
            U32_18[((size_t)pm * 9 + k) * g.Vh + i] = make_float2((float)a.x, (float)a.y);
        }
    double2 e[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) e[k] = src[(size_t)k * g.Vh];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double2 a = e[2 * k], b = e[2 * k + 1];
        if (U32)
            U32[((size_t)pm * 3 + k) * g.Vh + i] =
                make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
        if (U16)
            U16[((size_t)pm * 3 + k) * g.Vh + i] =
                make_uint2(Pair16<SP_F16>::from_floats((float)a.x, (float)a.y),
                           Pair16<SP_F16>::from_floats((float)b.x, (float)b.y));
        if (Ubf16)
            Ubf16[((size_t)pm * 3 + k) * g.Vh + i] =
                make_uint2(Pair16<SP_BF16>::from_floats((float)a.x, (float)a.y),
                           Pair16<SP_BF16>::from_floats((float)b.x, (float)b.y));
    }
}

}  // namespace

void launch_spinor_aos_to_eo(const Geom& g, const double* aos, void* eo, cudaStream_t s)
{
    spinor_aos_to_eo<<<dim3(blocks_for(g.Vh), 2), kThreads, 0, s>>>(g, aos, (double2*)eo);
}

void launch_spinor_eo_to_aos(const Geom& g, const void* eo, double* aos, cudaStream_t s)
{
    spinor_eo_to_aos<<<dim3(blocks_for(g.Vh), 2), kThreads, 0, s>>>(g, (const double2*)eo, aos);
}

void launch_links_aos_to_eo(const Geom& g, const double* aos, void* eo, cudaStream_t s)
{
    links_aos_to_eo<<<dim3(blocks_for(g.Vh), 8), kThreads, 0, s>>>(g, aos, (double2*)eo);
}

void launch_links_eo_to_aos(const Geom& g, const void* eo, double* aos, cudaStream_t s)
{
    links_eo_to_aos<<<dim3(blocks_for(g.Vh), 8), kThreads, 0, s>>>(g, (const double2*)eo, aos);
}

void launch_make_lowp_gauge(const Geom& g, const void* U64, void* U32, void* U16, cudaStream_t s, void* U32_18,
                            void* Ubf16)
{
    make_lowp<<<dim3(blocks_for(g.Vh), 8), kThreads, 0, s>>>(g, (const double2*)U64, (float4*)U32,
                                                              (uint2*)U16, (float2*)U32_18, (uint2*)Ubf16);
}

}  // namespace sfh

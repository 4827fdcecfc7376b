// walk.cuh — walking the periodic lattice by coordinates and reading FP64
// link fields at arbitrary sites (gauge links are periodic in every
// direction, Lattice.cpp:213-235).
#pragma once

#include "su3.cuh"

namespace sfh {

struct Walker {
    int x[4];
};

__device__ __forceinline__ void walk(const Geom& g, Walker& w, int mu, int dir)
{
    int v = w.x[mu] + dir;
    if (v < 0) v += g.L[mu];
    if (v >= g.L[mu]) v -= g.L[mu];
    w.x[mu] = v;
}

__device__ __forceinline__ int lex_of(const Geom& g, const Walker& w)
{
    return ((w.x[0] * g.L[1] + w.x[1]) * g.L[2] + w.x[2]) * g.L[3] + w.x[3];
}

__device__ __forceinline__ M3 link_at(const void* U, const Geom& g, const Walker& w, int mu)
{
    int par = (w.x[0] + w.x[1] + w.x[2] + w.x[3]) & 1;
    int i = lex_of(g, w) >> 1;
    const double2* b = (const double2*)U + ((size_t)(par * 4 + mu) * 9) * g.Vh + i;
    M3 m;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        double2 v = __ldg(b + (size_t)k * g.Vh);
        m.e[k] = {v.x, v.y};
    }
    return m;
}

__device__ __forceinline__ Walker link_coords(const Geom& g, int p, int i)
{
    Coord c = eo_coords(g, p, i);
    Walker w;
#pragma unroll
    for (int k = 0; k < 4; ++k) w.x[k] = c.x[k];
    return w;
}


}  // namespace sfh

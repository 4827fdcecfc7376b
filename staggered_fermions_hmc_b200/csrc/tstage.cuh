// tstage.cuh — neighbour vectors staged along the time direction.
//
// The even-odd index of a site is lex >> 1 with time the fastest coordinate
// (sfh_core.cuh), so for a tile of output sites [i0, i0 + n) of one parity
// the time and z neighbours lie in [i0 - Lt/2, i0 + n + Lt/2) of the other
// parity: a z hop moves the index by Lt/2, a time hop by 0 or 1, a time wrap
// by at most Lt/2 - 1; only z wraps leave the range.  One thread copies that
// range of a one-word-per-site vector field (the 16-bit storages: one uint4
// per site) into shared memory with one bulk asynchronous copy (the TMA
// engine, cp.async.bulk, completing on an mbarrier) while the tile computes
// its coordinates and loads its links; the x and y neighbours come from
// global memory.
//
// Every wait on the mbarrier is bounded (test_wait polls with a short sleep,
// kStageTries times): a thread whose copy has not landed raises
// DEV_ERR_TIMEOUT, waits once more with the same bound for the copy in
// flight, and reads its neighbours from global memory instead, so results do
// not depend on the staging.
#pragma once

#include <cstdint>

#include "sfh_core.cuh"

namespace sfh {
namespace {

constexpr int kStageTries = 1 << 20;  // polls of ~32 ns: a bound of ~0.1 s per wait

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    // the initialised barrier visible to the asynchronous (TMA) proxy
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// one arrival on the barrier that also announces `bytes` of transactions
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// bulk copy global -> shared of `bytes` (a multiple of 16, both addresses
// 16-byte aligned), completing that many transactions on the barrier
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// one copy announced and issued
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    mbar_arrive_expect_tx(bar, bytes);
    bulk_copy_g2s(dst, src, bytes, bar);
}

// wait for the barrier's phase `parity` to complete, at most kStageTries
// polls; true when it did
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity)
{
    for (int k = 0; k < kStageTries; ++k) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        __nanosleep(32);
    }
    return false;
}

// the staged range of a tile [i0, i0 + n) of parity-index space [0, Vh)
struct TRange {
    int lo, cnt;
};

__device__ __forceinline__ TRange trange(const Geom& g, int i0, int n)
{
    const int h = g.L[3] >> 1;
    const int lo = max(0, i0 - h);
    const int hi = min(g.Vh, i0 + n + h);
    return {lo, hi - lo};
}

// shared-memory words of a tile of n sites: n + Lt
__host__ __device__ __forceinline__ int tstage_words(int n, int Lt) { return n + Lt; }

// the word of neighbour j: from the staged range when it holds j (and the
// copy landed), else from global memory
__device__ __forceinline__ uint4 nbr_word(const uint4* s, const TRange& r, bool ok, const uint4* src, int j)
{
    const unsigned d = (unsigned)(j - r.lo);
    return (ok && d < (unsigned)r.cnt) ? s[d] : __ldg(src + j);
}

}  // namespace
}  // namespace sfh

// Block-wide scans used by the WZP codec and the side-record compaction.
#pragma once
#include "common.cuh"

namespace wb {

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += t;
    }
    return v;
}

// Exclusive scan over the block; `total` receives the block sum. `tmp` must
// hold 33 words of shared memory. Contains three __syncthreads().
template <int NT>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* tmp, uint32_t& total) {
    static_assert(NT % 32 == 0 && NT <= 1024, "block size");
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t inc = warp_incl_scan(v);
    __syncthreads(); // tmp may still be read by a previous scan
    if (lane == 31) tmp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < NW ? tmp[lane] : 0;
        const uint32_t wi = warp_incl_scan(w);
        if (lane < NW) tmp[lane] = wi - w;
        if (lane == NW - 1) tmp[32] = wi;
    }
    __syncthreads();
    total = tmp[32];
    return tmp[warp] + inc - v;
}

template <int NT>
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* tmp) {
    uint32_t total;
    block_excl_scan<NT>(v, tmp, total);
    return total;
}

} // namespace wb

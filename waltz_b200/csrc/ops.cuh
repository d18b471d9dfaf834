// Kernel launch forms shared by every pipeline stage.
//
// A stage is an Op type: its block size, a Params struct and
// `run(params, block, blocks)`, the body of one CTA given its block index
// within the stage's own grid. Two launch forms use the same body:
//  * op_kernel_for<Op>(): one launch for one field (grid = the stage's blocks);
//  * op_batch_kernel<Op>: one launch for the stage of many fields — a table
//    of Params in device memory and the first block of each entry; a CTA
//    finds its entry by binary search over the block starts and runs the
//    body with its block index inside that entry (a chunk-tile work list).
// Ops whose Params hold tensor maps use them in place: in kernel-parameter
// space (grid constant) for op_kernel, in global memory for op_batch_kernel.
#pragma once
#include "common.cuh"

namespace wb {

// Ops that hand the address of a parameter to the hardware (tensor maps)
// declare kGridConstant and get their parameters in grid-constant space;
// the others take them by value, so the body reads fields as constant-bank
// operands.
template <class Op, class = void> struct GridConstant {
    static constexpr bool value = false;
};
template <class Op> struct GridConstant<Op, decltype(void(Op::kGridConstant))> {
    static constexpr bool value = Op::kGridConstant;
};

template <class Op>
__global__ void __launch_bounds__(Op::kThreads, Op::kMinBlocks)
    op_kernel_gc(const __grid_constant__ typename Op::Params p) {
    Op::run(p, blockIdx.x, gridDim.x);
}

template <class Op>
__global__ void __launch_bounds__(Op::kThreads, Op::kMinBlocks) op_kernel_val(const typename Op::Params p) {
    Op::run(p, blockIdx.x, gridDim.x);
}

template <class Op> constexpr auto op_kernel_for() {
    if constexpr (GridConstant<Op>::value) return &op_kernel_gc<Op>;
    else return &op_kernel_val<Op>;
}

template <class Op>
__global__ void __launch_bounds__(Op::kThreads, Op::kMinBlocks)
    op_batch_kernel(const typename Op::Params* __restrict__ table, const uint32_t* __restrict__ starts,
                    uint32_t count) {
    const uint32_t b = blockIdx.x;
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(starts + mid) <= b) lo = mid;
        else hi = mid;
    }
    const uint32_t first = __ldg(starts + lo);
    if constexpr (GridConstant<Op>::value) {
        if (threadIdx.x == 0) Op::acquire_maps(table[lo]); // thread 0 issues the tensor copies
    }
    Op::run(table[lo], b - first, __ldg(starts + lo + 1) - first);
}

// The same stage as a persistent work queue: a grid of resident CTAs, each
// pulling chunk-tile items (a field's block) from a device ticket until the
// stage's items run out; an item runs the body exactly as op_batch_kernel
// runs it, and the CTA synchronises before its next item reuses shared
// memory. Items are taken in increasing order, so a stage whose blocks wait
// on earlier blocks of the same field (the WZP lookback) only waits on items
// already running on resident CTAs. The ticket is zeroed before each launch.
template <class Op>
__global__ void __launch_bounds__(Op::kThreads, Op::kMinBlocks)
    op_queue_kernel(const typename Op::Params* __restrict__ table, const uint32_t* __restrict__ starts,
                    uint32_t count, uint32_t* ticket) {
    __shared__ uint32_t item;
    const uint32_t total = __ldg(starts + count);
    for (;;) {
        if (threadIdx.x == 0) item = atomicAdd(ticket, 1u);
        __syncthreads();
        const uint32_t b = item;
        if (b >= total) break;
        uint32_t lo = 0, hi = count;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(starts + mid) <= b) lo = mid;
            else hi = mid;
        }
        const uint32_t first = __ldg(starts + lo);
        if constexpr (GridConstant<Op>::value) {
            if (threadIdx.x == 0) Op::acquire_maps(table[lo]);
        }
        Op::run(table[lo], b - first, __ldg(starts + lo + 1) - first);
        __syncthreads(); // the item's shared memory and `item` are free again
    }
}

// Zero fill of one byte range (16-byte stores for the aligned bulk).
struct ZeroOp {
    static constexpr int kThreads = 256, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        void* ptr;
        uint64_t bytes;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t blocks) {
        uint8_t* p = static_cast<uint8_t*>(P.ptr);
        const uint64_t n = P.bytes;
        const uint64_t head = (16 - (reinterpret_cast<uintptr_t>(p) & 15)) & 15;
        const uint64_t lead = head < n ? head : n;
        const uint64_t vec = (n - lead) / 16;
        const uint64_t stride = uint64_t(blocks) * kThreads;
        const uint64_t t = uint64_t(block) * kThreads + threadIdx.x;
        if (t < lead) p[t] = 0;
        uint4* v = reinterpret_cast<uint4*>(p + lead);
        for (uint64_t i = t; i < vec; i += stride) v[i] = make_uint4(0, 0, 0, 0);
        for (uint64_t i = lead + vec * 16 + t; i < n; i += stride) p[i] = 0;
    }
};

} // namespace wb

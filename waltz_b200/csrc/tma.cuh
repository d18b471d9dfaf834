// Tensor-memory-accelerator (TMA) staging: tiled bulk copies from global to
// shared memory, completed on an mbarrier (sm_90+ PTX, used here on sm_100a).
//
// Device side: one elected thread arms the barrier with the expected byte
// count and issues the copies; every thread waits on the barrier's phase with
// an iteration bound, after which the block agrees (barrier vote) to stop and
// records ST_WAIT_TIMEOUT instead of hanging. Copies are plain, one CTA
// each: every CTA reads its own boxes into its own shared memory.
// Host side: tensor maps are encoded with the driver's cuTensorMapEncodeTiled,
// reached through the runtime's driver entry point (no link-time libcuda).
#pragma once
#include <cuda.h>

#include "common.cuh"

namespace wb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes the initialised barrier visible to the asynchronous (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's generic-proxy shared-memory accesses before later
// asynchronous-proxy accesses (a TMA write into a buffer just read or written).
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Waits for phase `parity` of the barrier to complete; false after `bound`
// polls (each poll may suspend the thread for a short hardware time slice).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t bound) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t i = 0; i < bound; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Poll bound of every wait for a TMA copy or an MMA. A CTA whose wait runs
// out records ST_WAIT_TIMEOUT and returns, and the host rejects the call. The
// bulk copy it waited on may still be in flight into the CTA's shared memory
// at that point. A healthy device lands a tile in microseconds, far inside
// 2^22 polls, so this path only runs on a device that has already failed.
constexpr uint32_t kWaitBound = 1u << 22;

// A tensor map read from global memory (a batched launch's parameter table)
// is acquired by the tensor-map proxy before its first use, by the thread
// that issues the copies; maps in kernel parameter space need nothing.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
                 : "memory");
}

// ------------------------------------------------------------------ host
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// 3-D tiled map of a T array with x fastest (strides in elements). Returns
// false when the array does not meet the copy engine's rules (16-byte base
// and row strides) or the encoder is unavailable; callers then stage with
// ordinary loads.
template <class T>
inline bool make_map_3d(CUtensorMap* map, const T* base, uint64_t nx, uint64_t ny, uint64_t nz, uint64_t sy,
                        uint64_t sz, uint32_t bx, uint32_t by, uint32_t bz,
                        CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_NONE) {
    const EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (sy * sizeof(T)) % 16 || (sz * sizeof(T)) % 16) return false;
    if ((bx * sizeof(T)) % 16 || bx > 256 || by > 256 || bz > 256) return false;
    const cuuint64_t dims[3] = {nx, ny, nz};
    const cuuint64_t strides[2] = {sy * sizeof(T), sz * sizeof(T)};
    const cuuint32_t box[3] = {bx, by, bz};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapDataType type = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    if (swizzle == CU_TENSOR_MAP_SWIZZLE_128B && bx * sizeof(T) > 128) return false;
    return fn(map, type, 3, const_cast<T*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

} // namespace wb

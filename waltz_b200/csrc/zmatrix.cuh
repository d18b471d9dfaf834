// Tensor-core Z transform (the precision form's matrix arithmetic).
//
// All levels of the CDF 9/7 analysis (or synthesis) along z of a plane
// schedule form one dense nz x nz matrix Mz: coefficient n of a column is
// sum_k Mz[n][k] * x[k]. For a field stored z-major (plane z = nx*ny
// contiguous columns) the whole Z stage is the GEMM  D = X^T * Mz^T  with one
// row of D per column of the field, computed here on the 5th-generation
// tensor cores:
//   * a CTA takes 128 field columns at a time (UMMA M = 128): its threads
//     read the K = nz planes of those columns (coalesced rows of 128) in
//     chunks of up to 64 planes and split every value into TF32 halves
//     (hi = fp32 truncated to TF32, lo = x - hi, exact) written transposed
//     into the K-major no-swizzle operand layout (8-row x 16-byte core
//     matrices); chunks accumulate into the same tensor-memory tile. Double
//     fields are rounded to fp32 first (the precision form's transform is
//     fp32-accurate for both types; the quantisation and repair decisions of
//     double fields stay in double, outside this kernel);
//   * Mz's halves are prepared on the host in the same layout and loaded once
//     per CTA; D = Ahi*Bhi + Ahi*Blo + Alo*Bhi, three tcgen05.mma kind::tf32
//     per 8-deep K step, FP32 accumulation in tensor memory;
//   * the epilogue reads D from tensor memory (lane = field column, column =
//     coefficient) and writes it back z-major, or hands it to an emitter.
// One thread issues the MMAs and commits them to an mbarrier; every wait is
// bounded and a block that gives up records ST_WAIT_TIMEOUT, frees its tensor
// memory and returns. Every copy and load targets only this CTA.
#pragma once
#include "common.cuh"

#include <cuda_bf16.h>

#include <cfloat>
#include "tma.cuh"

namespace wb {

// Split forms of the precision form's arithmetic (the archive records the
// form in its header flags): TF32x3, BF16x3, and exact bf16 slices.
enum : int { kZsNone = 0, kZsTf32x3 = 1, kZsBf16x3 = 2, kZsExact = 3 };

constexpr int kZmCols = 128;   // field columns per tile (UMMA M)
constexpr int kZmMaxK = 128;   // largest nz handled (the whole matrix stays in shared memory)
constexpr int kZmChunk = 64;   // planes of A staged per MMA pass
constexpr int kZmThreads = 256;

// Instruction descriptor of tcgen05.mma kind::tf32: D f32, A and B tf32,
// both K-major, M = 128, N = np (bit layout of the UMMA instruction
// descriptor: c_format [4,6), a_format [7,10), b_format [10,13), a_major 15,
// b_major 16, N >> 3 at [17,23), M >> 4 at [24,29)).
__host__ __device__ constexpr uint32_t zm_idesc(uint32_t np) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((np >> 3) << 17) | ((128u >> 4) << 24);
}

// Shared-memory matrix descriptor: start >> 4 at [0,14), LBO >> 4 at
// [16,30), SBO >> 4 at [32,46), version 1 at [46,48), layout at [61,64).
__device__ __forceinline__ uint64_t zm_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
    return uint64_t((saddr >> 4) & 0x3fffu) | (uint64_t((lbo >> 4) & 0x3fffu) << 16) |
           (uint64_t((sbo >> 4) & 0x3fffu) << 32) | (uint64_t(1) << 46) | (uint64_t(layout) << 61);
}

__device__ __forceinline__ void zm_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    const uint32_t mask = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(mask), "r"(mask), "r"(mask), "r"(mask));
}

__device__ __forceinline__ void zm_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// Shared-memory plan of one CTA (bytes from a 1024-byte aligned base): the
// A halves (128 x one chunk of up to 64 planes each) and the B halves
// (np x kp each), all fp32.
struct ZmPlan {
    uint32_t kp, np;          // padded K (multiple of 8) and N (multiple of 16)
    uint32_t kc;              // planes per A chunk (multiple of 8, <= kZmChunk)
    uint32_t a_bytes;         // one A half: 128 x kc x 4 B
    uint32_t b_bytes;         // one B half: np x kp x 4 B
    __host__ __device__ static ZmPlan make(uint32_t nz) {
        ZmPlan p;
        p.kp = (nz + 7) / 8 * 8;
        p.np = (nz + 15) / 16 * 16;
        p.kc = p.kp < uint32_t(kZmChunk) ? p.kp : uint32_t(kZmChunk);
        p.a_bytes = 128 * p.kc * 4;
        p.b_bytes = p.np * p.kp * 4;
        return p;
    }
    __host__ __device__ uint32_t smem() const { return 1024 + 2 * a_bytes + 2 * b_bytes + 64; }
};

// Destination of the Z stage: z-major store, or a per-sample emitter. The
// epilogue hands over one column's group of 16 consecutive z values
// (z0 .. z0+15, those below nz).
// The values arrive as float (fp32-accurate forms) or double (the exact
// slice form), and are rounded to the field's type T.
template <class T> struct ZmStore {
    T* dst;       // z-major: dst[z * ncols + col]
    template <class V>
    __device__ __forceinline__ void group(uint32_t col, uint32_t z0, uint32_t nz, size_t ncols,
                                          const V (&r)[16]) const {
#pragma unroll
        for (int j = 0; j < 16; ++j)
            if (z0 + j < nz) dst[size_t(z0 + j) * ncols + col] = T(r[j]);
    }
};
template <class T, class Final> struct ZmEmit {
    Final fin;
    uint32_t nx;
    template <class V>
    __device__ __forceinline__ void group(uint32_t col, uint32_t z0, uint32_t nz, size_t, const V (&r)[16]) const {
        const uint32_t x = col % nx, y = col / nx;
        if constexpr (Final::kPrefetch) {
            // every original first, then the emissions: the loads do not wait
            // behind the emitter's stores
            T o[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) o[j] = z0 + j < nz ? fin.fetch(x, y, z0 + j) : T(0);
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if (z0 + j < nz) fin.emit(x, y, z0 + j, T(r[j]), o[j]);
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if (z0 + j < nz) fin(x, y, z0 + j, T(r[j]));
        }
    }
};

// B halves: device arrays of np * kp floats each in the K-major no-swizzle
// core layout (core (n/8, k/4) at ((n/8) * kp/4 + k/4) * 128 B, element
// (n%8, k%4) at (n%8) * 16 + (k%4) * 4 inside it).
template <class T, class Out>
__global__ void __launch_bounds__(kZmThreads, 2)
    zmatrix_kernel(const T* x, const float* bhi, const float* blo, uint32_t nz, uint64_t ncols, Out out,
                   uint32_t* status, uint32_t check_finite) {
    extern __shared__ __align__(1024) unsigned char zm_smem[];
    const ZmPlan P = ZmPlan::make(nz);
    unsigned char* base = zm_smem + ((1024 - (smem_u32(zm_smem) & 1023)) & 1023);
    unsigned char* Ahi = base;
    unsigned char* Alo = Ahi + P.a_bytes;
    unsigned char* Bhi = Alo + P.a_bytes;
    unsigned char* Blo = Bhi + P.b_bytes;
    uint64_t* mma_bar = reinterpret_cast<uint64_t*>(Blo + P.b_bytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint64_t tiles = (ncols + kZmCols - 1) / kZmCols;
    const uint32_t ncols_alloc = P.np <= 32 ? 32 : (P.np <= 64 ? 64 : 128);

    // tensor memory for D (128 lanes x np fp32 columns), barrier, operands B
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols_alloc));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(mma_bar, 1);
        fence_barrier_init();
    }
    for (uint32_t i = tid; i < P.b_bytes / 16; i += kZmThreads) {
        reinterpret_cast<uint4*>(Bhi)[i] = reinterpret_cast<const uint4*>(bhi)[i];
        reinterpret_cast<uint4*>(Blo)[i] = reinterpret_cast<const uint4*>(blo)[i];
    }
    fence_proxy_async();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = zm_idesc(P.np);
    const uint32_t sbo_b = (P.kp / 4) * 128; // 8-row groups of the K-major B operand

    uint32_t phase = 0;
    bool bad = false, range_bad = false, stop = false;
    for (uint64_t tile = blockIdx.x; tile < tiles && !stop; tile += gridDim.x) {
        for (uint32_t k0 = 0; k0 < P.kp; k0 += P.kc) {
            const uint32_t kc = min(P.kc, P.kp - k0); // planes of this chunk (multiple of 8)
            const uint32_t sbo_a = (kc / 4) * 128, kh = kc / 2;
            // split and transpose: thread t takes field column c = t % 128 and the
            // t / 128 half of the chunk's planes; element (c, k) goes to core
            // (c/8, k/4) at ((c/8) * kc/4 + k/4) * 128 B, row c%8
            {
                const int c = tid % kZmCols, half = tid / kZmCols;
                const uint64_t col = tile * kZmCols + c;
                const bool live = col < ncols;
                const T* xcol = x + col;
                unsigned char* hrow = Ahi + (c / 8) * sbo_a + (c % 8) * 16;
                unsigned char* lrow = Alo + (c / 8) * sbo_a + (c % 8) * 16;
                float v[kZmChunk / 2];
#pragma unroll
                for (int j = 0; j < kZmChunk / 2; ++j) {
                    const uint32_t k = k0 + half * kh + j;
                    T w = T(0);
                    if (j < int(kh) && k < nz && live) w = xcol[size_t(k) * ncols];
                    if (check_finite) {
                        bad |= !finite_bits(w);
                        if constexpr (sizeof(T) == 8) range_bad |= finite_bits(w) && fabs(w) > double(FLT_MAX);
                    }
                    v[j] = float(w);
                }
#pragma unroll
                for (int j = 0; j < kZmChunk / 2; j += 4) {
                    if (j < int(kh)) {
                        uint32_t h[4], l[4];
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            h[q] = __float_as_uint(v[j + q]) & 0xffffe000u;
                            l[q] = __float_as_uint(__fsub_rn(v[j + q], __uint_as_float(h[q])));
                        }
                        const uint32_t kq = (half * kh + j) / 4;
                        *reinterpret_cast<uint4*>(hrow + kq * 128) = make_uint4(h[0], h[1], h[2], h[3]);
                        *reinterpret_cast<uint4*>(lrow + kq * 128) = make_uint4(l[0], l[1], l[2], l[3]);
                    }
                }
            }
            fence_proxy_async();
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                // A and B: K-major, no swizzle; cores 128 B apart along K (LBO),
                // 8-row groups kc/4 (A) or kp/4 (B) cores apart (SBO); a K step
                // of 8 is two cores
                const uint32_t a0 = smem_u32(Ahi), a1 = smem_u32(Alo);
                const uint32_t b0 = smem_u32(Bhi) + (k0 / 8) * 256, b1 = smem_u32(Blo) + (k0 / 8) * 256;
                for (uint32_t s = 0; s < kc / 8; ++s) {
                    const uint64_t dah = zm_sdesc(a0 + s * 256, 128, sbo_a, 0);
                    const uint64_t dal = zm_sdesc(a1 + s * 256, 128, sbo_a, 0);
                    const uint64_t dbh = zm_sdesc(b0 + s * 256, 128, sbo_b, 0);
                    const uint64_t dbl = zm_sdesc(b1 + s * 256, 128, sbo_b, 0);
                    zm_mma(tmem, dah, dbh, idesc, (k0 > 0 || s > 0) ? 1u : 0u);
                    zm_mma(tmem, dah, dbl, idesc, 1);
                    zm_mma(tmem, dal, dbh, idesc, 1);
                }
                zm_commit(mma_bar);
            }
            // the chunk's MMAs have read A before the next chunk overwrites it
            if (!__syncthreads_and(warp != 0 || mbar_wait(mma_bar, phase, kWaitBound))) {
                if (tid == 0) atomicOr(status, ST_WAIT_TIMEOUT);
                stop = true;
                break;
            }
            phase ^= 1;
        }
        if (stop) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // epilogue: warp w reads lanes 32 (w % 4) .. (lane = field column) and
        // every other 16-coefficient group, starting at group w / 4
        const uint32_t sub = warp % 4;
        const uint64_t col = tile * kZmCols + 32 * sub + lane;
        for (uint32_t c0 = 16 * (warp / 4); c0 < P.np; c0 += 32) {
            uint32_t r[16];
            tmem_ld16(tmem + (uint32_t(32 * sub) << 16) + c0, r);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float f[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) f[j] = __uint_as_float(r[j]);
            if (col < ncols) out.group(uint32_t(col), c0, nz, ncols, f);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads(); // tensor memory read out: the next tile's MMAs may overwrite it
    }
    if (check_finite && __syncthreads_or(bad) && tid == 0) atomicOr(status, ST_NONFINITE_INPUT);
    if (check_finite && __syncthreads_or(range_bad) && tid == 0) atomicOr(status, ST_MATRIX_RANGE);
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols_alloc));
    }
}


// ---------------------------------------------------------------------------
// TF32x3 for float fields with the planes staged by TMA. The field (or the
// coefficients) is a 2-D tensor of nz planes of ncols floats; a work item is
// (tile of 128 columns, chunk of up to 32 planes), and its box of planes is
// copied into one of two raw buffers two items ahead of its use, so the
// copies run while the threads split, the MMAs run and the epilogue stores.
// The split reads a column of the raw box (consecutive threads on
// consecutive columns), and from there on every step is zmatrix_kernel's:
// the same TF32 halves in the same core layout, the same three products per
// K step into one fp32 tile, the same epilogue, so the output is identical.
// 97 KB of shared memory at nz <= 64 (two CTAs per SM).
constexpr int kZmTmaChunk = 32;

struct ZmTmaPlan {
    uint32_t kp, np, kc;
    uint32_t raw_bytes, a_bytes, b_bytes;
    __host__ __device__ static ZmTmaPlan make(uint32_t nz) {
        ZmTmaPlan p;
        p.kp = (nz + 7) / 8 * 8;
        p.np = (nz + 15) / 16 * 16;
        p.kc = p.kp < uint32_t(kZmTmaChunk) ? p.kp : uint32_t(kZmTmaChunk);
        p.raw_bytes = p.kc * kZmCols * 4;
        p.a_bytes = kZmCols * p.kc * 4;
        p.b_bytes = p.np * p.kp * 4;
        return p;
    }
    // raw boxes, A halves, B halves, four barriers + TMEM slot
    __host__ __device__ uint32_t smem() const { return 1024 + 2 * raw_bytes + 2 * a_bytes + 2 * b_bytes + 64; }
};

template <class Out>
__global__ void __launch_bounds__(kZmThreads, 2)
    zmatrix_tma_kernel(const __grid_constant__ CUtensorMap xmap, const float* bhi, const float* blo, uint32_t nz,
                       uint64_t ncols, Out out, uint32_t* status, uint32_t check_finite) {
    extern __shared__ __align__(1024) unsigned char zt_smem[];
    const ZmTmaPlan P = ZmTmaPlan::make(nz);
    unsigned char* base = zt_smem + ((1024 - (smem_u32(zt_smem) & 1023)) & 1023);
    float* raw = reinterpret_cast<float*>(base);                       // 2 boxes of kc x 128
    unsigned char* Ahi = base + 2 * P.raw_bytes;
    unsigned char* Alo = Ahi + P.a_bytes;
    unsigned char* Bhi = Alo + P.a_bytes;
    unsigned char* Blo = Bhi + P.b_bytes;
    uint64_t* mma_bar = reinterpret_cast<uint64_t*>(Blo + P.b_bytes);
    uint64_t* raw_bar = mma_bar + 1;                                    // two
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 3);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint64_t tiles = (ncols + kZmCols - 1) / kZmCols;
    const uint32_t ncols_alloc = P.np <= 32 ? 32 : (P.np <= 64 ? 64 : 128);
    const uint32_t nch = (P.kp + P.kc - 1) / P.kc;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols_alloc));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // item i of this CTA: tile blockIdx.x + (i / nch) * gridDim.x, chunk i % nch
    auto item_tile = [&](uint64_t i) { return uint64_t(blockIdx.x) + (i / nch) * gridDim.x; };
    auto stage = [&](uint64_t i) { // thread 0: copy item i's planes into raw box i % 2
        const uint32_t b = uint32_t(i & 1);
        mbar_expect_tx(raw_bar + b, P.raw_bytes);
        tma_load_3d(reinterpret_cast<unsigned char*>(raw) + b * P.raw_bytes, &xmap, int(item_tile(i) * kZmCols),
                    int((i % nch) * P.kc), 0, raw_bar + b);
    };
    if (tid == 0) {
        mbar_init(mma_bar, 1);
        mbar_init(raw_bar, 1);
        mbar_init(raw_bar + 1, 1);
        fence_barrier_init();
        if (item_tile(0) < tiles) stage(0);
        if (item_tile(1) < tiles) stage(1);
    }
    for (uint32_t i = tid; i < P.b_bytes / 16; i += kZmThreads) {
        reinterpret_cast<uint4*>(Bhi)[i] = reinterpret_cast<const uint4*>(bhi)[i];
        reinterpret_cast<uint4*>(Blo)[i] = reinterpret_cast<const uint4*>(blo)[i];
    }
    fence_proxy_async();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = zm_idesc(P.np);
    const uint32_t sbo_b = (P.kp / 4) * 128;
    const int c = tid % kZmCols, half = tid / kZmCols;

    uint32_t mphase = 0;
    uint64_t staged = 2;   // next item to stage (thread 0)
    uint64_t consumed = 0; // items whose copy was waited for
    bool bad = false, stop = false;
    for (uint64_t i = 0; item_tile(i) < tiles; ++i) {
        const uint64_t tile = item_tile(i);
        const uint32_t k0 = uint32_t(i % nch) * P.kc;
        const uint32_t kc = min(P.kc, P.kp - k0); // planes of this chunk (multiple of 8)
        const uint32_t sbo_a = (kc / 4) * 128, kh = kc / 2;
        const uint32_t b = uint32_t(i & 1);
        if (!__syncthreads_and(warp != 0 || mbar_wait(raw_bar + b, uint32_t((i >> 1) & 1), kWaitBound))) {
            if (tid == 0) atomicOr(status, ST_WAIT_TIMEOUT);
            stop = true;
            break;
        }
        consumed = i + 1;
        // split and transpose from the raw box: element (c, k) of the box
        // (plane k0 + k) goes to core (c/8, k/4), row c%8, as in zmatrix_kernel
        {
            const float* box = raw + size_t(b) * (P.raw_bytes / 4);
            const uint64_t col = tile * kZmCols + c;
            unsigned char* hrow = Ahi + (c / 8) * sbo_a + (c % 8) * 16;
            unsigned char* lrow = Alo + (c / 8) * sbo_a + (c % 8) * 16;
#pragma unroll
            for (int j = 0; j < kZmTmaChunk / 2; j += 4) {
                if (j < int(kh)) {
                    uint32_t h[4], l[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const uint32_t k = half * kh + j + q;
                        const float w = box[k * kZmCols + c]; // zero past the field (the copy's fill)
                        if (check_finite && col < ncols && k0 + k < nz) bad |= !finite_bits(w);
                        h[q] = __float_as_uint(w) & 0xffffe000u;
                        l[q] = __float_as_uint(__fsub_rn(w, __uint_as_float(h[q])));
                    }
                    const uint32_t kq = (half * kh + j) / 4;
                    *reinterpret_cast<uint4*>(hrow + kq * 128) = make_uint4(h[0], h[1], h[2], h[3]);
                    *reinterpret_cast<uint4*>(lrow + kq * 128) = make_uint4(l[0], l[1], l[2], l[3]);
                }
            }
        }
        fence_proxy_async(); // the raw box's reads before the copy that refills it
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (item_tile(staged) < tiles) stage(staged); // item i + 2 into the box just read
            ++staged;
            const uint32_t a0 = smem_u32(Ahi), a1 = smem_u32(Alo);
            const uint32_t b0 = smem_u32(Bhi) + (k0 / 8) * 256, b1 = smem_u32(Blo) + (k0 / 8) * 256;
            for (uint32_t st = 0; st < kc / 8; ++st) {
                const uint64_t dah = zm_sdesc(a0 + st * 256, 128, sbo_a, 0);
                const uint64_t dal = zm_sdesc(a1 + st * 256, 128, sbo_a, 0);
                const uint64_t dbh = zm_sdesc(b0 + st * 256, 128, sbo_b, 0);
                const uint64_t dbl = zm_sdesc(b1 + st * 256, 128, sbo_b, 0);
                zm_mma(tmem, dah, dbh, idesc, (k0 > 0 || st > 0) ? 1u : 0u);
                zm_mma(tmem, dah, dbl, idesc, 1);
                zm_mma(tmem, dal, dbh, idesc, 1);
            }
            zm_commit(mma_bar);
        }
        if (!__syncthreads_and(warp != 0 || mbar_wait(mma_bar, mphase, kWaitBound))) {
            if (tid == 0) atomicOr(status, ST_WAIT_TIMEOUT);
            stop = true;
            break;
        }
        mphase ^= 1;
        if (k0 + P.kc >= P.kp) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sub = warp % 4;
            const uint64_t ocol = tile * kZmCols + 32 * sub + lane;
            for (uint32_t c0 = 16 * (warp / 4); c0 < P.np; c0 += 32) {
                uint32_t r[16];
                tmem_ld16(tmem + (uint32_t(32 * sub) << 16) + c0, r);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                float f[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) f[j] = __uint_as_float(r[j]);
                if (ocol < ncols) out.group(uint32_t(ocol), c0, nz, ncols, f);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads(); // tensor memory read out: the next tile's MMAs may overwrite it
        }
    }
    if (stop && tid == 0) {
        // copies still in flight (items consumed .. staged - 1 that exist)
        // land before the block leaves, each wait bounded
        for (uint64_t j = consumed; j < staged && item_tile(j) < tiles; ++j)
            mbar_wait(raw_bar + (j & 1), uint32_t((j >> 1) & 1), kWaitBound);
    }
    if (check_finite && __syncthreads_or(bad) && tid == 0) atomicOr(status, ST_NONFINITE_INPUT);
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols_alloc));
    }
}

// ---------------------------------------------------------------------------
// Slice forms, same GEMM D = X^T * Mz^T, same tiling and epilogue layout.
//
// BF16x3 (tcgen05.mma kind::f16, bf16 operands, fp32 accumulation): every
// value is split into three bf16 slices (x = b0 + b1 + b2 + r with
// |r| ~ 2^-24 |x|: b0 = bf16(x), b1 = bf16(x - b0), b2 = bf16(x - b0 - b1),
// each residual exact in fp32) and the six slice products of order <= 2
// accumulate into one fp32 tile. Operands K-major without swizzle: core
// matrices of 8 rows x 16 bytes (8 bf16 along K), cores 128 B apart along K
// (LBO), 8-row groups kc/8 (A) or kp/8 (B) cores apart (SBO); one MMA
// (K = 16) is two cores.
//
// Exact slices (tcgen05.mma kind::i8, signed 8-bit operands, s32
// accumulation; double fields, nz <= 96): every field column c is scaled by
// 2^-(e_c+1) (|x| < 2^e_c over the column) and every matrix row n by
// 2^-(f_n+1), so all values lie in (-1/2, 1/2), then cut into five 7-bit
// integer slices u = sum_s a_s 2^-7(s+1) with |a_s| <= 64. Every product
// order d = s + t accumulates exactly (integers) in its own s32 tile; the
// epilogue recombines the five tiles in double (Horner in 2^-7, exact) and
// scales by 2^(e_c + f_n + 2 - 14). The result is the exact sum of every
// slice product of order <= 4: a truncation error near 2^-34 of (column max
// x row max x K), far below fp32 rounding. One MMA (K = 32) is two cores of
// 16 int8 along K; the int8 operands keep a CTA at 110 KB of shared memory
// (two per SM).

constexpr int kZsExactSlices = 5;
constexpr int kZsExactMaxK = 96; // five accumulators of 96 columns fit the 512 TMEM columns

struct ZsPlan {
    uint32_t S;       // slices per operand
    uint32_t eb;      // bytes per element: 2 (bf16) or 1 (int8)
    uint32_t kp, np;  // K padded to the MMA K (16 or 32), N to a multiple of 16
    uint32_t kc;      // planes per A chunk
    uint32_t a_bytes; // one A slice: 128 x kc elements
    uint32_t b_bytes; // one B slice: np x kp elements
    __host__ __device__ static ZsPlan make(uint32_t nz, bool exact) {
        ZsPlan p;
        p.S = exact ? uint32_t(kZsExactSlices) : 3u;
        p.eb = exact ? 1u : 2u;
        const uint32_t kstep = exact ? 32u : 16u;
        p.kp = (nz + kstep - 1) / kstep * kstep;
        p.np = (nz + 15) / 16 * 16;
        // the exact form stages the whole column (nz <= 96) in one chunk
        p.kc = exact ? p.kp : (p.kp < 64u ? p.kp : 64u);
        p.a_bytes = 128 * p.kc * p.eb;
        p.b_bytes = p.np * p.kp * p.eb;
        return p;
    }
    // A slices, B slices, 2 x 128 column maxima / exponents, barrier, TMEM slot
    __host__ __device__ uint32_t smem() const { return 1024 + S * (a_bytes + b_bytes) + 2 * 128 * 8 + 64; }
};

// Instruction descriptors: kind::f16 with D f32, A and B bf16; kind::i8 with
// D s32, A and B signed 8-bit; both K-major, M = 128, N = np.
__host__ __device__ constexpr uint32_t zs_idesc_bf16(uint32_t np) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((np >> 3) << 17) | ((128u >> 4) << 24);
}
__host__ __device__ constexpr uint32_t zs_idesc_s8(uint32_t np) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((np >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void zs_mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
    const uint32_t mask = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(mask), "r"(mask), "r"(mask), "r"(mask));
}
__device__ __forceinline__ void zs_mma_s8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    const uint32_t mask = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(mask), "r"(mask), "r"(mask), "r"(mask));
}

__device__ __forceinline__ uint16_t bf16_bits(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }
__device__ __forceinline__ float bf16_value(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }

// 2^e as a double (normal range).
__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

// Common set-up of the slice kernels: TMEM allocation, mbarrier, operand B
// copied into shared memory.
__device__ __forceinline__ uint32_t zs_setup(unsigned char* B, const void* bsrc, uint32_t bbytes, uint64_t* mma_bar,
                                             uint32_t* tmem_slot, uint32_t tcols, int tid) {
    if ((tid >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(tcols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(mma_bar, 1);
        fence_barrier_init();
    }
    for (uint32_t i = tid; i < bbytes / 16; i += kZmThreads)
        reinterpret_cast<uint4*>(B)[i] = reinterpret_cast<const uint4*>(bsrc)[i];
    fence_proxy_async();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return *tmem_slot;
}

__device__ __forceinline__ void zs_teardown(uint32_t tmem, uint32_t tcols, bool bad, bool range_bad,
                                            uint32_t check_finite, uint32_t* status, int tid) {
    if (check_finite && __syncthreads_or(bad) && tid == 0) atomicOr(status, ST_NONFINITE_INPUT);
    if (check_finite && __syncthreads_or(range_bad) && tid == 0) atomicOr(status, ST_MATRIX_RANGE);
    __syncthreads();
    if ((tid >> 5) == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols));
    }
}

// BF16x3. bsl: the three B slices of np x kp bf16 each, in the core layout.
template <class T, class Out>
__global__ void __launch_bounds__(kZmThreads, 2)
    zmatrix_bf16_kernel(const T* x, const uint16_t* bsl, uint32_t nz, uint64_t ncols, Out out, uint32_t* status,
                        uint32_t check_finite) {
    constexpr int S = 3;
    extern __shared__ __align__(1024) unsigned char zs_smem[];
    const ZsPlan P = ZsPlan::make(nz, false);
    unsigned char* base = zs_smem + ((1024 - (smem_u32(zs_smem) & 1023)) & 1023);
    unsigned char* A = base;              // S slices of a_bytes
    unsigned char* B = A + S * P.a_bytes; // S slices of b_bytes
    uint64_t* mma_bar = reinterpret_cast<uint64_t*>(B + S * P.b_bytes + 2 * 128 * 8);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint64_t tiles = (ncols + kZmCols - 1) / kZmCols;
    const uint32_t tcols = P.np <= 32 ? 32u : (P.np <= 64 ? 64u : 128u);
    const uint32_t tmem = zs_setup(B, bsl, S * P.b_bytes, mma_bar, tmem_slot, tcols, tid);
    const uint32_t idesc = zs_idesc_bf16(P.np);
    const uint32_t sbo_b = (P.kp / 8) * 128;

    uint32_t phase = 0;
    bool bad = false, range_bad = false, stop = false;
    for (uint64_t tile = blockIdx.x; tile < tiles && !stop; tile += gridDim.x) {
        const int c = tid % kZmCols, half = tid / kZmCols;
        const uint64_t col = tile * kZmCols + c;
        const bool live = col < ncols;
        const T* xcol = x + col;
        for (uint32_t k0 = 0; k0 < P.kp; k0 += P.kc) {
            const uint32_t kc = min(P.kc, P.kp - k0);
            const uint32_t sbo_a = (kc / 8) * 128, kh = kc / 2;
            // every plane this thread slices is loaded first (all loads in
            // flight at once): planes half * kh .. half * kh + kh - 1 of the chunk
            constexpr int MAXH = kZmChunk / 2;
            T v[MAXH];
#pragma unroll
            for (int j = 0; j < MAXH; ++j) {
                const uint32_t k = k0 + half * kh + j;
                v[j] = (uint32_t(j) < kh && k < nz && live) ? xcol[size_t(k) * ncols] : T(0);
            }
            // slice and transpose: element (c, kk) of slice s goes to core
            // (c/8, kk/8) of that slice, row c % 8, 2-byte column kk % 8
            unsigned char* row0 = A + (c / 8) * sbo_a + (c % 8) * 16;
#pragma unroll
            for (int j = 0; j < MAXH; j += 8) {
                if (uint32_t(j) >= kh) break;
                uint32_t pk[S][4];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const T w = v[j + q];
                    if (check_finite) {
                        bad |= !finite_bits(w);
                        if constexpr (sizeof(T) == 8) range_bad |= finite_bits(w) && fabs(w) > double(FLT_MAX);
                    }
                    const float xf = float(w);
                    uint16_t sl[S];
                    sl[0] = bf16_bits(xf);
                    const float r1 = __fsub_rn(xf, bf16_value(sl[0]));
                    sl[1] = bf16_bits(r1);
                    sl[2] = bf16_bits(__fsub_rn(r1, bf16_value(sl[1])));
#pragma unroll
                    for (int s2 = 0; s2 < S; ++s2) {
                        if (q & 1) pk[s2][q >> 1] |= uint32_t(sl[s2]) << 16;
                        else pk[s2][q >> 1] = sl[s2];
                    }
                }
                const uint32_t kq = (half * kh + j) / 8;
#pragma unroll
                for (int s2 = 0; s2 < S; ++s2)
                    *reinterpret_cast<uint4*>(row0 + s2 * P.a_bytes + kq * 128) =
                        make_uint4(pk[s2][0], pk[s2][1], pk[s2][2], pk[s2][3]);
            }
            fence_proxy_async();
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a0 = smem_u32(A), b0 = smem_u32(B) + (k0 / 8) * 128;
                for (uint32_t st = 0; st < kc / 16; ++st) {
                    // the six slice products of order <= 2, one accumulator
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
#pragma unroll
                        for (int s2 = 0; s2 <= d; ++s2) {
                            const uint64_t da = zm_sdesc(a0 + s2 * P.a_bytes + st * 256, 128, sbo_a, 0);
                            const uint64_t db = zm_sdesc(b0 + (d - s2) * P.b_bytes + st * 256, 128, sbo_b, 0);
                            const bool first = k0 == 0 && st == 0 && d == 0;
                            zs_mma_bf16(tmem, da, db, idesc, first ? 0u : 1u);
                        }
                    }
                }
                zm_commit(mma_bar);
            }
            if (!__syncthreads_and(warp != 0 || mbar_wait(mma_bar, phase, kWaitBound))) {
                if (tid == 0) atomicOr(status, ST_WAIT_TIMEOUT);
                stop = true;
                break;
            }
            phase ^= 1;
        }
        if (stop) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t sub = warp % 4;
        const uint64_t ocol = tile * kZmCols + 32 * sub + lane;
        for (uint32_t c0 = 16 * (warp / 4); c0 < P.np; c0 += 32) {
            uint32_t r[16];
            tmem_ld16(tmem + (uint32_t(32 * sub) << 16) + c0, r);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float f[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) f[j] = __uint_as_float(r[j]);
            if (ocol < ncols) out.group(uint32_t(ocol), c0, nz, ncols, f);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads(); // tensor memory read out: the next tile's MMAs may overwrite it
    }
    zs_teardown(tmem, tcols, bad, range_bad, check_finite, status, tid);
}

// Exact slices. bsl: the five B slices of np x kp int8 each, in the core
// layout (core (n/8, k/16) at ((n/8) * kp/16 + k/16) * 128 B, element
// (n%8, k%16) at (n%8) * 16 + k%16); bscale[n] = 2^(f_n + 1 - 14).
template <class T, class Out>
__global__ void __launch_bounds__(kZmThreads, 2)
    zmatrix_exact_kernel(const T* x, const int8_t* bsl, const double* bscale, uint32_t nz, uint64_t ncols, Out out,
                         uint32_t* status, uint32_t check_finite) {
    constexpr int S = kZsExactSlices;
    extern __shared__ __align__(1024) unsigned char zs_smem[];
    const ZsPlan P = ZsPlan::make(nz, true);
    unsigned char* base = zs_smem + ((1024 - (smem_u32(zs_smem) & 1023)) & 1023);
    unsigned char* A = base;              // S slices of a_bytes
    unsigned char* B = A + S * P.a_bytes; // S slices of b_bytes
    double* cmax = reinterpret_cast<double*>(B + S * P.b_bytes); // [2][128] partial maxima
    int* cexp = reinterpret_cast<int*>(cmax);                     // [128] column exponents, after the maxima
    uint64_t* mma_bar = reinterpret_cast<uint64_t*>(cmax + 2 * 128);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint64_t tiles = (ncols + kZmCols - 1) / kZmCols;
    const uint32_t tmem = zs_setup(B, bsl, S * P.b_bytes, mma_bar, tmem_slot, 512u, tid);
    const uint32_t idesc = zs_idesc_s8(P.np);
    const uint32_t kc = P.kp, kh = kc / 2;
    const uint32_t sbo_a = (kc / 16) * 128, sbo_b = (P.kp / 16) * 128;

    uint32_t phase = 0;
    bool bad = false, range_bad = false;
    for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int c = tid % kZmCols, half = tid / kZmCols;
        const uint64_t col = tile * kZmCols + c;
        const bool live = col < ncols;
        const T* xcol = x + col;
        // column maximum over both threads' planes (half * kh .. + kh - 1)
        double m = 0.0;
#pragma unroll 8
        for (uint32_t j = 0; j < kh; ++j) {
            const uint32_t k = half * kh + j;
            const double w = (k < nz && live) ? double(xcol[size_t(k) * ncols]) : 0.0;
            if (check_finite) bad |= !finite_bits(w);
            m = fmax(m, fabs(w));
        }
        cmax[half * 128 + c] = m;
        __syncthreads();
        const double amax = fmax(cmax[c], cmax[128 + c]);
        // |x| < 2^e over the column; e clamped so that the scalings stay
        // normal doubles (columns below 2^-1000 become zero, beyond 2^1000
        // are refused)
        int e = amax > 0.0 ? int((__double_as_longlong(amax) >> 52) & 0x7ff) - 1022 : -1000;
        if (amax >= 0x1p1000) range_bad = true;
        e = e < -1000 ? -1000 : (e > 1000 ? 1000 : e);
        const double scale = pow2(-(e + 1));
        __syncthreads();
        if (half == 0) cexp[c] = e;
        // slice and transpose: element (c, kk) of slice s goes to core
        // (c/8, kk/16) of that slice, row c % 8, byte kk % 16
        unsigned char* row0 = A + (c / 8) * sbo_a + (c % 8) * 16;
        for (uint32_t j = 0; j < kh; j += 16) {
            uint32_t pk[S][4];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const uint32_t k = half * kh + j + q;
                const double w = (k < nz && live) ? double(xcol[size_t(k) * ncols]) : 0.0;
                double u = w * scale;
#pragma unroll
                for (int s2 = 0; s2 < S; ++s2) {
                    const double a = rint(u * 128.0);
                    u = u * 128.0 - a;
                    const uint32_t b = uint32_t(int32_t(a)) & 0xffu;
                    if (q & 3) pk[s2][q >> 2] |= b << (8 * (q & 3));
                    else pk[s2][q >> 2] = b;
                }
            }
            const uint32_t kq = (half * kh + j) / 16;
#pragma unroll
            for (int s2 = 0; s2 < S; ++s2)
                *reinterpret_cast<uint4*>(row0 + s2 * P.a_bytes + kq * 128) =
                    make_uint4(pk[s2][0], pk[s2][1], pk[s2][2], pk[s2][3]);
        }
        fence_proxy_async();
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
            for (uint32_t st = 0; st < kc / 32; ++st) {
                // products of order d = s + t, each order in its own accumulator
#pragma unroll
                for (int d = 0; d < S; ++d) {
#pragma unroll
                    for (int s2 = 0; s2 <= d; ++s2) {
                        const uint64_t da = zm_sdesc(a0 + s2 * P.a_bytes + st * 256, 128, sbo_a, 0);
                        const uint64_t db = zm_sdesc(b0 + (d - s2) * P.b_bytes + st * 256, 128, sbo_b, 0);
                        zs_mma_s8(tmem + uint32_t(d) * P.np, da, db, idesc, (st == 0 && s2 == 0) ? 0u : 1u);
                    }
                }
            }
            zm_commit(mma_bar);
        }
        if (!__syncthreads_and(warp != 0 || mbar_wait(mma_bar, phase, kWaitBound))) {
            if (tid == 0) atomicOr(status, ST_WAIT_TIMEOUT);
            break;
        }
        phase ^= 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t sub = warp % 4;
        const uint32_t lc = 32 * sub + lane;
        const uint64_t ocol = tile * kZmCols + lc;
        const double cs = pow2(cexp[lc] + 1);
        for (uint32_t c0 = 16 * (warp / 4); c0 < P.np; c0 += 32) {
            double v[16];
#pragma unroll
            for (int d = S - 1; d >= 0; --d) {
                uint32_t r[16];
                tmem_ld16(tmem + (uint32_t(32 * sub) << 16) + uint32_t(d) * P.np + c0, r);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    v[j] = d == S - 1 ? double(int32_t(r[j])) : fma(v[j], 0x1p-7, double(int32_t(r[j])));
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = v[j] * cs * (c0 + j < P.np ? bscale[c0 + j] : 0.0);
            if (ocol < ncols) out.group(uint32_t(ocol), c0, nz, ncols, v);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads(); // tensor memory read out: the next tile's MMAs may overwrite it
    }
    zs_teardown(tmem, 512u, bad, range_bad, check_finite, status, tid);
}

} // namespace wb

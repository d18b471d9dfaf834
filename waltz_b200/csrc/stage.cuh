// Whole-stage kernels of the plane schedule: every level of the Z stage, or
// every level of the XY stage, in one launch, for fields whose lines (Z) or
// planes (XY) fit in shared memory.
//
// The per-level kernels stage a tile plus a halo per level and go through
// HBM between levels; these keep a whole column set (Z) or a whole z-plane
// (XY) in shared memory and run all levels there, reading the field once and
// writing each coefficient once. The arithmetic is the per-level kernels'
// own: the same halo windows of the same lifting steps, so the bits are the
// same.
//  * forward windows are position independent (any even origin gives the same
//    bits); W = 16 here;
//  * inverse Z windows are the canonical folded ones (W = 16 for float, 8 for
//    double, origins at multiples of W), inverse Y windows W = 8 (folded),
//    inverse X is not folded (W = 16), exactly as in the per-level kernels
//    (reference: cpu/src/transform.cpp:149-179, include/transformers/
//    all_halo.cuh:143-224 for the plane schedule's stage order).
#pragma once
#include "transform.cuh"

namespace wb {

constexpr int kStageMaxLevels = 5;
constexpr size_t kStageSmemCap = 200u * 1024u;

// Level extents of one stage: Z lengths, or XY box sizes.
struct StageLevels {
    uint32_t x[kStageMaxLevels], y[kStageMaxLevels], z[kStageMaxLevels];
    uint32_t count;
};

// Column tile of the Z stage: 64 columns, rows of 128 bytes along x.
template <class T> struct ZCols {
    static constexpr int CX = 128 / int(sizeof(T));
    static constexpr int C = 64;
    static constexpr int CY = C / CX;
};
constexpr int kZStageThreads = 256;
constexpr int kXYStageThreads = 512;
static_assert(kZStageThreads % 64 == 0, "every thread keeps one column");

template <class T> inline size_t zstage_smem(uint32_t nz) { return 2 * size_t(ZCols<T>::C) * nz * sizeof(T); }
__host__ __device__ inline uint32_t xy_pitch(uint32_t nx) { return nx | 1u; } // odd pitch: row-parallel passes hit distinct banks
template <class T> inline size_t xystage_smem(uint32_t nx, uint32_t ny) {
    return 2 * size_t(xy_pitch(nx)) * ny * sizeof(T);
}

// Window of P even/odd pairs starting at spatial position s-4 of a line of
// length m, read through `at(p)` (reflected position p -> element). Interior
// windows skip the reflection.
template <class T, int P, class Get>
__device__ __forceinline__ void load_window(int64_t s, uint32_t m, T (&e)[P], T (&o)[P], Get&& at) {
    if (s >= 4 && s + 2 * P - 4 <= int64_t(m)) {
#pragma unroll
        for (int j = 0; j < P; ++j) {
            e[j] = at(uint32_t(s - 4 + 2 * j));
            o[j] = at(uint32_t(s - 3 + 2 * j));
        }
    } else {
#pragma unroll
        for (int j = 0; j < P; ++j) {
            e[j] = at(mirror(s - 4 + 2 * j, m));
            o[j] = at(mirror(s - 3 + 2 * j, m));
        }
    }
}

// ------------------------------------------------------------------ Z stage
// Forward: a CTA owns 64 columns (x-fastest) over the whole z extent. Level l
// lifts lines of length z[l]; high bands go to `dst` at their split
// positions, low bands stay in shared memory for the next level; the last
// level writes both. With `status`, the input is checked for finiteness.
template <class T> struct ZStageFwdOp {
    static constexpr int kThreads = kZStageThreads, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        const T* in;
        size_t sy, sz;
        uint32_t nx, ny, nz;
        StageLevels lv;
        T* dst;
        uint32_t* status;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t);
};

template <class T>
__device__ __forceinline__ void ZStageFwdOp<T>::run(const Params Pm, uint32_t block, uint32_t) {
    const T* in = Pm.in;
    const size_t sy = Pm.sy, sz = Pm.sz;
    const uint32_t nx = Pm.nx, ny = Pm.ny, nz = Pm.nz;
    const StageLevels& lv = Pm.lv;
    T* const dst = Pm.dst;
    uint32_t* const status = Pm.status;
    constexpr int CX = ZCols<T>::CX, C = ZCols<T>::C;
    constexpr int W = 16, P = W / 2 + 4;
    extern __shared__ __align__(16) unsigned char zstage_raw[];
    T* buf[2] = {reinterpret_cast<T*>(zstage_raw), reinterpret_cast<T*>(zstage_raw) + size_t(C) * nz};
    const uint32_t tiles_x = (nx + CX - 1) / CX;
    const int c = threadIdx.x % C;
    const uint32_t x = (block % tiles_x) * CX + c % CX, y = (block / tiles_x) * ZCols<T>::CY + c / CX;
    const bool live = x < nx && y < ny;
    const size_t col = size_t(y) * sy + x;
    bool bad = false;
    for (uint32_t z = threadIdx.x / C; z < nz; z += kZStageThreads / C) {
        const T v = live ? in[size_t(z) * sz + col] : T(0);
        buf[0][size_t(z) * C + c] = v;
        bad |= !finite_bits(v);
    }
    if (__syncthreads_or(bad) && status && threadIdx.x == 0) atomicOr(status, ST_NONFINITE_INPUT);
    for (uint32_t l = 0; l < lv.count; ++l) {
        const uint32_t m = lv.z[l], h = half_len(m);
        const bool last = l + 1 == lv.count;
        const T* src = buf[l & 1];
        T* low = buf[(l + 1) & 1];
        const uint32_t wins = (m + W - 1) / W;
        for (uint32_t w = threadIdx.x / C; w < wins; w += kZStageThreads / C) {
            const uint32_t s = w * W;
            T e[P], o[P];
            load_window<T, P>(int64_t(s), m, e, o, [&](uint32_t p) { return src[size_t(p) * C + c]; });
            lift_forward<T, P>(e, o);
#pragma unroll
            for (int j = 2; j < P - 2; ++j) {
                const uint32_t u = s + 2 * (j - 2);
                if (u < m) {
                    if (!last) low[size_t(u >> 1) * C + c] = e[j];
                    else if (live) dst[size_t(u >> 1) * sz + col] = e[j];
                }
                if (u + 1 < m && live) dst[size_t(h + (u >> 1)) * sz + col] = o[j];
            }
        }
        __syncthreads();
    }
}

// Inverse: the column set's coefficients are loaded once into both buffers
// (each level's high band already sits at its place in the split layout);
// level l reads one buffer and writes its spatial output over the low part of
// the other, which is the next finer level's low band. The finest level hands
// every sample to `out`.
template <class T, class Out> struct ZStageInvOp {
    static constexpr int kThreads = kZStageThreads, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        const T* coef;
        size_t sy, sz;
        uint32_t nx, ny, nz;
        StageLevels lv;
        Out out;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t);
};

template <class T, class Out>
__device__ __forceinline__ void ZStageInvOp<T, Out>::run(const Params Pm, uint32_t block, uint32_t) {
    const T* coef = Pm.coef;
    const size_t sy = Pm.sy, sz = Pm.sz;
    const uint32_t nx = Pm.nx, ny = Pm.ny, nz = Pm.nz;
    const StageLevels& lv = Pm.lv;
    const Out out = Pm.out;
    constexpr int CX = ZCols<T>::CX, C = ZCols<T>::C;
    constexpr int W = inverse_zwin<T>(), P = W / 2 + 4;
    extern __shared__ __align__(16) unsigned char zstage_raw[];
    T* buf[2] = {reinterpret_cast<T*>(zstage_raw), reinterpret_cast<T*>(zstage_raw) + size_t(C) * nz};
    const uint32_t tiles_x = (nx + CX - 1) / CX;
    const int c = threadIdx.x % C;
    const uint32_t x = (block % tiles_x) * CX + c % CX, y = (block / tiles_x) * ZCols<T>::CY + c / CX;
    const bool live = x < nx && y < ny;
    const size_t col = size_t(y) * sy + x;
    for (uint32_t z = threadIdx.x / C; z < nz; z += kZStageThreads / C) {
        const T v = live ? coef[size_t(z) * sz + col] : T(0);
        buf[0][size_t(z) * C + c] = v;
        buf[1][size_t(z) * C + c] = v;
    }
    __syncthreads();
    int cur = 0;
    for (int l = int(lv.count) - 1; l >= 0; --l) {
        const uint32_t m = lv.z[l];
        const T* src = buf[cur];
        T* nxt = buf[cur ^ 1];
        const uint32_t wins = (m + W - 1) / W;
        for (uint32_t w = threadIdx.x / C; w < wins; w += kZStageThreads / C) {
            const uint32_t s = w * W;
            // finest level with a prefetching emitter: the originals of the
            // window's outputs are requested before the lifting
            T pe[P], po[P];
            if constexpr (Out::kPrefetch) {
                if (l == 0 && live) {
#pragma unroll
                    for (int j = 2; j < P - 2; ++j) {
                        const uint32_t u = s + 2 * (j - 2);
                        pe[j] = u < m ? out.fetch(x, y, u) : T(0);
                        po[j] = u + 1 < m ? out.fetch(x, y, u + 1) : T(0);
                    }
                }
            }
            T e[P], o[P];
            load_window<T, P>(int64_t(s), m, e, o,
                              [&](uint32_t p) { return src[size_t(split_of(p, m)) * C + c]; });
            lift_inverse<T, P, true>(e, o);
#pragma unroll
            for (int j = 2; j < P - 2; ++j) {
                const uint32_t u = s + 2 * (j - 2);
                if (l > 0) {
                    if (u < m) nxt[size_t(u) * C + c] = e[j];
                    if (u + 1 < m) nxt[size_t(u + 1) * C + c] = o[j];
                } else if (live) {
                    if constexpr (Out::kPrefetch) {
                        if (u < m) out.emit(x, y, u, e[j], pe[j]);
                        if (u + 1 < m) out.emit(x, y, u + 1, o[j], po[j]);
                    } else {
                        if (u < m) out(x, y, u, e[j]);
                        if (u + 1 < m) out(x, y, u + 1, o[j]);
                    }
                }
            }
        }
        __syncthreads();
        cur ^= 1;
    }
}

// ----------------------------------------------------------------- XY stage
// Forward: one CTA per z-plane. Per level: Y lifting (P -> Q, spatial), X
// lifting (Q -> P in the level's split layout), then the high bands (all of
// the box at the last level) are copied out row by row; the low corner of P
// is the next level's input. With `status`, the input is checked.
template <class T> struct XYStageFwdOp {
    static constexpr int kThreads = kXYStageThreads, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        const T* in;
        size_t sy, sz;
        uint32_t nx, ny;
        StageLevels lv;
        T* dst;
        size_t dsy, dsz;
        uint32_t* status;
    };
    static __device__ __forceinline__ void run(const Params Pm, uint32_t block, uint32_t);
};

template <class T>
__device__ __forceinline__ void XYStageFwdOp<T>::run(const Params Pm, uint32_t block, uint32_t) {
    const T* in = Pm.in;
    const size_t sy = Pm.sy, sz = Pm.sz, dsy = Pm.dsy, dsz = Pm.dsz;
    const uint32_t nx = Pm.nx, ny = Pm.ny;
    const StageLevels& lv = Pm.lv;
    T* const dst = Pm.dst;
    uint32_t* const status = Pm.status;
    constexpr int W = 16, P = W / 2 + 4;
    extern __shared__ __align__(16) unsigned char xystage_raw[];
    const uint32_t PX = xy_pitch(nx);
    T* Pb = reinterpret_cast<T*>(xystage_raw);
    T* Qb = Pb + size_t(PX) * ny;
    const uint32_t z = block;
    const T* plane = in + size_t(z) * sz;
    bool bad = false;
    for (uint32_t i = threadIdx.x; i < nx * ny; i += kXYStageThreads) {
        const uint32_t y = i / nx, x = i - y * nx;
        const T v = plane[size_t(y) * sy + x];
        Pb[size_t(y) * PX + x] = v;
        bad |= !finite_bits(v);
    }
    if (__syncthreads_or(bad) && status && threadIdx.x == 0) atomicOr(status, ST_NONFINITE_INPUT);
    T* out = dst + size_t(z) * dsz;
    for (uint32_t l = 0; l < lv.count; ++l) {
        const uint32_t mx = lv.x[l], my = lv.y[l], hx = half_len(mx), hy = half_len(my);
        const bool last = l + 1 == lv.count;
        // Y: columns of P -> Q
        {
            const uint32_t wins = (my + W - 1) / W;
            for (uint32_t it = threadIdx.x; it < mx * wins; it += kXYStageThreads) {
                const uint32_t cx = it % mx, s = (it / mx) * W;
                T e[P], o[P];
                load_window<T, P>(int64_t(s), my, e, o, [&](uint32_t p) { return Pb[size_t(p) * PX + cx]; });
                lift_forward<T, P>(e, o);
#pragma unroll
                for (int j = 2; j < P - 2; ++j) {
                    const uint32_t u = s + 2 * (j - 2);
                    if (u < my) Qb[size_t(u) * PX + cx] = e[j];
                    if (u + 1 < my) Qb[size_t(u + 1) * PX + cx] = o[j];
                }
            }
        }
        __syncthreads();
        // X: rows of Q -> P at split positions
        {
            const uint32_t wins = (mx + W - 1) / W;
            for (uint32_t it = threadIdx.x; it < my * wins; it += kXYStageThreads) {
                const uint32_t r = it % my, s = (it / my) * W;
                const T* row = Qb + size_t(r) * PX;
                T* prow = Pb + size_t(split_of(r, my)) * PX;
                T e[P], o[P];
                load_window<T, P>(int64_t(s), mx, e, o, [&](uint32_t p) { return row[p]; });
                lift_forward<T, P>(e, o);
#pragma unroll
                for (int j = 2; j < P - 2; ++j) {
                    const uint32_t u = s + 2 * (j - 2);
                    if (u < mx) prow[u >> 1] = e[j];
                    if (u + 1 < mx) prow[hx + (u >> 1)] = o[j];
                }
            }
        }
        __syncthreads();
        // copy out (P is only read here; the next level's Y pass reads P's low
        // corner and writes Q, which nothing reads any more)
        for (uint32_t i = threadIdx.x; i < mx * my; i += kXYStageThreads) {
            const uint32_t cy = i / mx, cx = i - cy * mx;
            if (!last && cx < hx && cy < hy) continue;
            out[size_t(cy) * dsy + cx] = Pb[size_t(cy) * PX + cx];
        }
    }
}

// Inverse: the plane's coefficients are loaded into P once. Per level
// (coarsest first): X lifting of the box's coefficient rows (P -> Q), then Y
// lifting of Q's columns read through the split layout, written spatially
// over P's box (the next finer level's low corner), or to `out` at level 0.
template <class T, class Out> struct XYStageInvOp {
    static constexpr int kThreads = kXYStageThreads, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        const T* coef;
        size_t sy, sz;
        uint32_t nx, ny;
        StageLevels lv;
        Out out;
    };
    static __device__ __forceinline__ void run(const Params Pm, uint32_t block, uint32_t);
};

template <class T, class Out>
__device__ __forceinline__ void XYStageInvOp<T, Out>::run(const Params Pm, uint32_t block, uint32_t) {
    const T* coef = Pm.coef;
    const size_t sy = Pm.sy, sz = Pm.sz;
    const uint32_t nx = Pm.nx, ny = Pm.ny;
    const StageLevels& lv = Pm.lv;
    const Out out = Pm.out;
    constexpr int WX = 16, PXW = WX / 2 + 4;
    constexpr int WY = 8, PYW = WY / 2 + 4;
    extern __shared__ __align__(16) unsigned char xystage_raw[];
    const uint32_t PX = xy_pitch(nx);
    T* Pb = reinterpret_cast<T*>(xystage_raw);
    T* Qb = Pb + size_t(PX) * ny;
    const uint32_t z = block;
    const T* plane = coef + size_t(z) * sz;
    for (uint32_t i = threadIdx.x; i < nx * ny; i += kXYStageThreads) {
        const uint32_t y = i / nx, x = i - y * nx;
        Pb[size_t(y) * PX + x] = plane[size_t(y) * sy + x];
    }
    __syncthreads();
    for (int l = int(lv.count) - 1; l >= 0; --l) {
        const uint32_t mx = lv.x[l], my = lv.y[l];
        // X: coefficient rows of P -> Q (spatial x)
        {
            const uint32_t wins = (mx + WX - 1) / WX;
            for (uint32_t it = threadIdx.x; it < my * wins; it += kXYStageThreads) {
                const uint32_t r = it % my, s = (it / my) * WX;
                const T* row = Pb + size_t(r) * PX;
                T e[PXW], o[PXW];
                load_window<T, PXW>(int64_t(s), mx, e, o, [&](uint32_t p) { return row[split_of(p, mx)]; });
                lift_inverse<T, PXW, false>(e, o);
                T* q = Qb + size_t(r) * PX;
#pragma unroll
                for (int j = 2; j < PXW - 2; ++j) {
                    const uint32_t u = s + 2 * (j - 2);
                    if (u < mx) q[u] = e[j];
                    if (u + 1 < mx) q[u + 1] = o[j];
                }
            }
        }
        __syncthreads();
        // Y: columns of Q through the split layout -> P (spatial) or out
        {
            const uint32_t wins = (my + WY - 1) / WY;
            for (uint32_t it = threadIdx.x; it < mx * wins; it += kXYStageThreads) {
                const uint32_t cx = it % mx, s = (it / mx) * WY;
                T pe[PYW], po[PYW];
                if constexpr (Out::kPrefetch) {
                    if (l == 0) {
#pragma unroll
                        for (int j = 2; j < PYW - 2; ++j) {
                            const uint32_t u = s + 2 * (j - 2);
                            pe[j] = u < my ? out.fetch(cx, u, z) : T(0);
                            po[j] = u + 1 < my ? out.fetch(cx, u + 1, z) : T(0);
                        }
                    }
                }
                T e[PYW], o[PYW];
                load_window<T, PYW>(int64_t(s), my, e, o,
                                    [&](uint32_t p) { return Qb[size_t(split_of(p, my)) * PX + cx]; });
                lift_inverse<T, PYW, true>(e, o);
#pragma unroll
                for (int j = 2; j < PYW - 2; ++j) {
                    const uint32_t u = s + 2 * (j - 2);
                    if (l > 0) {
                        if (u < my) Pb[size_t(u) * PX + cx] = e[j];
                        if (u + 1 < my) Pb[size_t(u + 1) * PX + cx] = o[j];
                    } else if constexpr (Out::kPrefetch) {
                        if (u < my) out.emit(cx, u, z, e[j], pe[j]);
                        if (u + 1 < my) out.emit(cx, u + 1, z, o[j], po[j]);
                    } else {
                        if (u < my) out(cx, u, z, e[j]);
                        if (u + 1 < my) out(cx, u + 1, z, o[j]);
                    }
                }
            }
        }
        __syncthreads();
    }
}

} // namespace wb

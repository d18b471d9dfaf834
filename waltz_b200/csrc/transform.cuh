// Multi-level CDF 9/7 lifting on the GPU: one fused kernel per level.
//
// A CTA owns an output tile U = (UX, UY, UZ) of one level's box. It stages
// the tile plus a 4-sample halo per lifted axis in shared memory, lifts the
// axes one after another (forward Y, X, Z; inverse Z, X, Y), shrinking the
// staged region after every pass, and hands each finished sample to an
// emitter functor. Every lifted line is processed in windows of W outputs
// that read W+8 samples, exactly like the reference's halo windows
// (cpu/src/transform.cpp:149-179, include/transformers/halo3d.cuh:66-169):
//  * forward windows are tile independent (any even origin gives the same
//    bits), so W is chosen for speed;
//  * inverse Y and Z windows fold their endpoint normalisations, so their
//    results depend on the window: W_Y = 8 and W_Z = 16 (f32) / 8 (f64)
//    with origins at multiples of W, the reference's canonical windows;
//  * inverse X does not fold and is window independent.
#pragma once
#include "common.cuh"

namespace wb {

enum Axes : int { AX = 1, AY = 2, AZ = 4 };

// Forward source: a compact or strided box, reflected at its edges. With
// `status` set, every staged sample is also checked for finiteness (the
// finest level stages every input sample at least once). Samples are staged
// row by row: `row(y, z)` resolves a row once, `get(row, x)` reads one sample.
template <class T> struct FwdSrc {
    const T* p;
    size_t sy, sz; // element strides
    uint32_t* status = nullptr;
    struct Row {
        const T* p;
    };
    __device__ __forceinline__ Row row(uint32_t y, uint32_t z) const { return {p + size_t(z) * sz + size_t(y) * sy}; }
    __device__ __forceinline__ T get(const Row& r, uint32_t x) const { return r.p[x]; }
};

template <class Src> __device__ __forceinline__ uint32_t* finite_status(const Src&) { return nullptr; }
template <class T> __device__ __forceinline__ uint32_t* finite_status(const FwdSrc<T>& s) { return s.status; }

// Inverse source: coefficient box whose low corner (lo dims) may come from a
// separately reconstructed compact array, the rest from `base`.
template <class T> struct InvSrc {
    const T* base;
    size_t sy, sz;
    const T* low; // nullable
    Dims lo;
    struct Row {
        const T* b;
        const T* l; // the row's low-corner part, or null
    };
    __device__ __forceinline__ Row row(uint32_t y, uint32_t z) const {
        const T* l = (low && y < lo.y && z < lo.z) ? low + (size_t(z) * lo.y + y) * lo.x : nullptr;
        return {base + size_t(z) * sz + size_t(y) * sy, l};
    }
    __device__ __forceinline__ T get(const Row& r, uint32_t x) const { return (r.l && x < lo.x) ? r.l[x] : r.b[x]; }
};

// Forward output: high bands to `dst` at split positions; the all-even low
// corner to `low` (compact, dims lo) when given, else to dst as well.
template <class T> struct FwdOut {
    T* dst;
    size_t sy, sz;
    T* low;
    Dims lo;
    Dims a;
    int mask;
    __device__ __forceinline__ void operator()(uint32_t x, uint32_t y, uint32_t z, T v) const {
        const bool ex = !(mask & AX) || !(x & 1), ey = !(mask & AY) || !(y & 1), ez = !(mask & AZ) || !(z & 1);
        const uint32_t cx = (mask & AX) ? split_of(x, a.x) : x;
        const uint32_t cy = (mask & AY) ? split_of(y, a.y) : y;
        const uint32_t cz = (mask & AZ) ? split_of(z, a.z) : z;
        if (low && ex && ey && ez) low[(size_t(cz) * lo.y + cy) * lo.x + cx] = v;
        else dst[size_t(cz) * sz + size_t(cy) * sy + cx] = v;
    }
    // All-axes form with the column's split (cx, cy) resolved by the caller.
    __device__ __forceinline__ void put(uint32_t cx, uint32_t cy, bool even_xy, uint32_t z, T v) const {
        const uint32_t cz = split_of(z, a.z);
        if (low && even_xy && !(z & 1)) low[(size_t(cz) * lo.y + cy) * lo.x + cx] = v;
        else dst[size_t(cz) * sz + size_t(cy) * sy + cx] = v;
    }
};

// Inverse output into a compact or strided array.
template <class T> struct StoreOut {
    static constexpr bool kPrefetch = false;
    T* dst;
    size_t sy, sz;
    __device__ __forceinline__ void operator()(uint32_t x, uint32_t y, uint32_t z, T v) const {
        dst[size_t(z) * sz + size_t(y) * sy + x] = v;
    }
};

// Emitters whose samples sit at dst + z * sz + y * sy + x take pointers
// computed once per row or column; the others take each sample through
// their own operator().
template <class Out> struct RowStore {
    static constexpr bool value = false;
};
template <class T> struct RowStore<StoreOut<T>> {
    static constexpr bool value = true;
};

template <int Mask, int U, int Axis> struct Ext {
    static constexpr int value = (Mask & Axis) ? U + 8 : U;
};

// One lifting pass along `Axis` over a staged region.
// in: extents (IX, IY, IZ) with the lifted axis extended by 8 halo samples;
// out: same with the lifted axis reduced to its tile length U.
// Items are (line, window) pairs with consecutive threads on consecutive
// lines, so the other-axis stride keeps shared-memory banks distinct.
template <class T, bool Inverse, int Axis, int W, int U, int IX, int IY, int IZ, int PX, class Sink>
__device__ __forceinline__ void lift_pass(const T* in, Sink&& sink) {
    constexpr int P = W / 2 + 4;
    constexpr int WIN = U / W;
    static_assert(U % W == 0, "tile must hold whole windows");
    constexpr int LA = Axis == AX ? IY : IX;          // first line axis extent
    constexpr int LB = Axis == AZ ? IY : IZ;          // second line axis extent
    constexpr int LINES = LA * LB;
    constexpr int STEP = Axis == AX ? 1 : (Axis == AY ? PX : PX * IY);
    constexpr bool Folded = Inverse && Axis != AX;
    for (int item = threadIdx.x; item < LINES * WIN; item += blockDim.x) {
        const int line = item % LINES, win = item / LINES;
        const int la = line % LA, lb = line / LA;
        int bx, by, bz;
        if (Axis == AX) { bx = 0; by = la; bz = lb; }
        else if (Axis == AY) { bx = la; by = 0; bz = lb; }
        else { bx = la; by = lb; bz = 0; }
        const T* src = in + (size_t(bz) * IY + by) * PX + bx + size_t(win) * W * STEP;
        T e[P], o[P];
#pragma unroll
        for (int j = 0; j < P; ++j) {
            e[j] = src[(2 * j) * STEP];
            o[j] = src[(2 * j + 1) * STEP];
        }
        if constexpr (Inverse) lift_inverse<T, P, Folded>(e, o);
        else lift_forward<T, P>(e, o);
#pragma unroll
        for (int j = 2; j < P - 2; ++j) {
            const int u = win * W + 2 * (j - 2);
            sink(bx, by, bz, u, e[j]);
            sink(bx, by, bz, u + 1, o[j]);
        }
    }
}

template <class T, bool Inverse, int Mask, int UX, int UY, int UZ> struct LevelShape {
    static constexpr int FX = Ext<Mask, UX, AX>::value;
    static constexpr int FY = Ext<Mask, UY, AY>::value;
    static constexpr int FZ = Ext<Mask, UZ, AZ>::value;
    static constexpr int FOOT = FX * FY * FZ;
    static constexpr int FPX = FX | 1; // odd pitches keep X-pass banks distinct
};

template <class T> constexpr int inverse_zwin() { return sizeof(T) == 4 ? 16 : 8; }

// Shared-memory bytes of one level kernel instance.
template <class T, bool Inverse, int Mask, int UX, int UY, int UZ>
constexpr size_t level_smem() {
    using S = LevelShape<T, Inverse, Mask, UX, UY, UZ>;
    // buffer A holds the footprint; buffer B the region after the first pass
    const size_t a = size_t(S::FPX) * S::FY * S::FZ;
    size_t b = 0;
    if (Mask == (AX | AY | AZ)) b = Inverse ? size_t(S::FPX) * S::FY * UZ : size_t(S::FPX) * UY * S::FZ;
    else if (Mask == (AX | AY)) b = Inverse ? a : size_t(S::FPX) * UY * S::FZ;
    return (a + b) * sizeof(T);
}

// Level op (1-D grid of grid.x * grid.y * grid.z tiles). Src: FwdSrc/InvSrc (positions are spatial in box a and are
// reflected / coefficient-mapped on load). Out: functor (x,y,z,value).
template <class T, bool Inverse, int Mask, int UX, int UY, int UZ, class Src, class Out> struct LevelOp {
    static constexpr int kThreads = 256, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        Src src;
        Dims a, grid;
        Out out;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t);
};

template <class T, bool Inverse, int Mask, int UX, int UY, int UZ, class Src, class Out>
__device__ __forceinline__ void LevelOp<T, Inverse, Mask, UX, UY, UZ, Src, Out>::run(const Params P, uint32_t block,
                                                                                      uint32_t) {
    const Src src = P.src;
    const Dims a = P.a, grid = P.grid;
    const Out out = P.out;
    using S = LevelShape<T, Inverse, Mask, UX, UY, UZ>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* A = reinterpret_cast<T*>(smem_raw);
    T* B = A + size_t(S::FPX) * S::FY * S::FZ;
    const uint32_t bx = block % grid.x, by = (block / grid.x) % grid.y, bz = block / (grid.x * grid.y);
    const uint32_t ox = bx * UX, oy = by * UY, oz = bz * UZ;
    const int hx = (Mask & AX) ? 4 : 0, hy = (Mask & AY) ? 4 : 0, hz = (Mask & AZ) ? 4 : 0;

    // ---- stage the footprint: warp w takes rows w, w+8, ...; a lane covers
    // x = lane and lane + 32 of every row. Source positions are reflected
    // (forward) or coefficient-mapped (inverse) once per lane and per row, and
    // each lane keeps kBatch rows of loads in flight before storing them.
    static_assert(S::FX <= 64, "footprint rows wider than two warps");
    {
        auto map = [&](int64_t p, uint32_t n, bool lifted) -> uint32_t {
            return (Inverse && lifted) ? coeff_at(p, n) : mirror(p, n);
        };
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        constexpr int NW = 256 / 32;
        const bool has0 = lane < S::FX, has1 = lane + 32 < S::FX;
        const uint32_t x0 = map(int64_t(ox) + lane - hx, a.x, Mask & AX);
        const uint32_t x1 = map(int64_t(ox) + lane + 32 - hx, a.x, Mask & AX);
        constexpr int ROWS = S::FY * S::FZ;
        constexpr int kBatch = 8;
        bool bad = false;
        for (int r0 = warp; r0 < ROWS; r0 += NW * kBatch) {
            T v0[kBatch], v1[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int r = r0 + u * NW;
                v0[u] = T(0);
                v1[u] = T(0);
                if (r < ROWS) {
                    const int fy = r % S::FY, fz = r / S::FY;
                    const auto row = src.row(map(int64_t(oy) + fy - hy, a.y, Mask & AY),
                                             map(int64_t(oz) + fz - hz, a.z, Mask & AZ));
                    if (has0) v0[u] = src.get(row, x0);
                    if (has1) v1[u] = src.get(row, x1);
                }
            }
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int r = r0 + u * NW;
                if (r < ROWS) {
                    const int fy = r % S::FY, fz = r / S::FY;
                    T* dst = A + (size_t(fz) * S::FY + fy) * S::FPX;
                    if (has0) dst[lane] = v0[u];
                    if (has1) dst[lane + 32] = v1[u];
                    bad |= !finite_bits(v0[u]) || !finite_bits(v1[u]);
                }
            }
        }
        if (uint32_t* st = finite_status(src)) {
            if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(st, ST_NONFINITE_INPUT);
        }
    }
    __syncthreads();

    constexpr int WZ = Inverse ? inverse_zwin<T>() : (UZ % 16 == 0 ? 16 : 8);
    constexpr int WY = Inverse ? 8 : (UY % 16 == 0 ? 16 : 8);
    constexpr int WX = UX % 16 == 0 ? 16 : 8;

    // Final emission of a tile-relative position.
    auto emit = [&](int ux, int uy, int uz, T v) {
        const uint32_t px = ox + ux, py = oy + uy, pz = oz + uz;
        if (px < a.x && py < a.y && pz < a.z) out(px, py, pz, v);
    };

    if constexpr (!Inverse) {
        // forward order: Y, X, Z over the active axes
        if constexpr (Mask == (AX | AY | AZ)) {
            // Y: A(FX,FY,FZ) -> B(FX,UY,FZ)
            lift_pass<T, false, AY, WY, UY, S::FX, S::FY, S::FZ, S::FPX>(A, [&](int bx, int, int bz, int u, T v) {
                B[(size_t(bz) * UY + u) * S::FPX + bx] = v;
            });
            __syncthreads();
            // X: B(FX,UY,FZ) -> A(UX,UY,FZ)
            lift_pass<T, false, AX, WX, UX, S::FX, UY, S::FZ, S::FPX>(B, [&](int, int by, int bz, int u, T v) {
                A[(size_t(bz) * UY + by) * S::FPX + u] = v;
            });
            __syncthreads();
            // Z: A(UX,UY,FZ) -> emit
            lift_pass<T, false, AZ, WZ, UZ, UX, UY, S::FZ, S::FPX>(A, [&](int bx, int by, int, int u, T v) {
                emit(bx, by, u, v);
            });
        } else if constexpr (Mask == (AX | AY)) {
            lift_pass<T, false, AY, WY, UY, S::FX, S::FY, S::FZ, S::FPX>(A, [&](int bx, int, int bz, int u, T v) {
                B[(size_t(bz) * UY + u) * S::FPX + bx] = v;
            });
            __syncthreads();
            lift_pass<T, false, AX, WX, UX, S::FX, UY, S::FZ, S::FPX>(B, [&](int, int by, int bz, int u, T v) {
                emit(u, by, bz, v);
            });
        } else {
            static_assert(Mask == AZ, "unsupported axis set");
            lift_pass<T, false, AZ, WZ, UZ, S::FX, S::FY, S::FZ, S::FPX>(A, [&](int bx, int by, int, int u, T v) {
                emit(bx, by, u, v);
            });
        }
    } else {
        // inverse order: Z, X, Y over the active axes
        if constexpr (Mask == (AX | AY | AZ)) {
            // Z: A(FX,FY,FZ) -> B(FX,FY,UZ)
            lift_pass<T, true, AZ, WZ, UZ, S::FX, S::FY, S::FZ, S::FPX>(A, [&](int bx, int by, int, int u, T v) {
                B[(size_t(u) * S::FY + by) * S::FPX + bx] = v;
            });
            __syncthreads();
            // X: B(FX,FY,UZ) -> A(UX,FY,UZ)
            lift_pass<T, true, AX, WX, UX, S::FX, S::FY, UZ, S::FPX>(B, [&](int, int by, int bz, int u, T v) {
                A[(size_t(bz) * S::FY + by) * S::FPX + u] = v;
            });
            __syncthreads();
            // Y: A(UX,FY,UZ) -> emit
            lift_pass<T, true, AY, WY, UY, UX, S::FY, UZ, S::FPX>(A, [&](int bx, int, int bz, int u, T v) {
                emit(bx, u, bz, v);
            });
        } else if constexpr (Mask == (AX | AY)) {
            lift_pass<T, true, AX, WX, UX, S::FX, S::FY, S::FZ, S::FPX>(A, [&](int, int by, int bz, int u, T v) {
                B[(size_t(bz) * S::FY + by) * S::FPX + u] = v;
            });
            __syncthreads();
            lift_pass<T, true, AY, WY, UY, UX, S::FY, S::FZ, S::FPX>(B, [&](int bx, int, int bz, int u, T v) {
                emit(bx, u, bz, v);
            });
        } else {
            static_assert(Mask == AZ, "unsupported axis set");
            lift_pass<T, true, AZ, WZ, UZ, S::FX, S::FY, S::FZ, S::FPX>(A, [&](int bx, int by, int, int u, T v) {
                emit(bx, by, u, v);
            });
        }
    }
}

} // namespace wb

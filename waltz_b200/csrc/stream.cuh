// Forward dyadic level as a z-march (all three axes in one kernel), and the
// same march for an XY level of the plane schedule (Z = false: Y and X per
// plane, no z pipeline and no z halo).
//
// The forward analysis is window independent (every output depends only on
// its reflected neighbourhood, cpu/src/transform.cpp:136-146), so a level can
// be computed in any order that keeps the per-axis order Y, X, Z of every
// sample. A CTA owns a UX x UY column tile and marches along z: Q input planes
// at a time are staged with their 4-sample XY halo, lifted along Y then X in
// shared memory, and fed to a register pipeline that lifts every column along
// Z as the planes arrive. The pipeline holds five values per column and emits
// one even/odd output pair per input pair; feeding starts 4 planes before the
// CTA's first output plane, so the z halo costs 8 planes per z range instead
// of 8 planes per tile of 16.
//
// Z pipeline for pair j (e_j, o_j raw), all steps as in lift_forward:
//   o1[j-1] = fma(A, e[j-1] + e[j], o[j-1])
//   e2[j-1] = fma(B, o1[j-2] + o1[j-1], e[j-1])
//   o3[j-2] = fma(G, e2[j-2] + e2[j-1], o1[j-2])
//   e4[j-2] = fma(D, o3[j-3] + o3[j-2], e2[j-2])
//   out: z = 2(j-2) -> e4[j-2] * K, z = 2(j-2)+1 -> o3[j-2] * (-1/K)
// Outputs are exact from the third pair after the first fed pair on.
//
// Staging: with a tensor map the planes arrive as per-plane TMA boxes
// (FX x FY x 1 at the reflected z), the copy of the next Q planes overlapping
// the X and Z passes of the current ones; cells of edge tiles that fall
// outside the array are then reflected in shared memory. Without a map
// (unaligned rows) the planes are staged with batched ordinary loads.
#pragma once
#include "common.cuh"
#include "tma.cuh"
#include "transform.cuh"

namespace wb {

template <class T> struct StreamTile;
template <> struct StreamTile<float> {
    static constexpr int UX = 32, UY = 16, Q = 8;
};
template <> struct StreamTile<double> {
    static constexpr int UX = 16, UY = 16, Q = 8;
};

template <class T, int UX, int UY, int Q, int NT = 256> struct StreamShape {
    static constexpr int FX = UX + 8, FY = UY + 8;
    static constexpr int YP = UX + 9 - (UX + 8) % 2; // odd pitch of the lifted rows
    static constexpr int IN = Q * FY * FX;          // staged planes
    static constexpr int MID = Q * UY * YP;          // Y-lifted planes
    static constexpr size_t smem = size_t(IN + MID) * sizeof(T) + 128 + 16; // + alignment + barrier
    static constexpr int COLS = UX * UY;
    static constexpr int CPT = (COLS + NT - 1) / NT; // columns per thread
};

template <class T> struct ZPipe {
    T e, o, o1, e2, o3;
};

// Largest |bit pattern| of the staged input (finiteness check: a non-finite
// value has every exponent bit set).
__device__ __forceinline__ uint32_t abs_bits(float v) { return __float_as_uint(v) & 0x7fffffffu; }
__device__ __forceinline__ unsigned long long abs_bits(double v) {
    return (unsigned long long)(__double_as_longlong(v)) & 0x7fffffffffffffffull;
}
__device__ __forceinline__ bool nonfinite_max(uint32_t m) { return m >= 0x7f800000u; }
__device__ __forceinline__ bool nonfinite_max(unsigned long long m) { return m >= 0x7ff0000000000000ull; }

// Tma: stage planes with per-plane tensor-map boxes; otherwise with batched
// ordinary loads. `status` receives ST_WAIT_TIMEOUT if a copy never
// completes within the wait bound (the block then stops as a whole).
// NT threads per CTA: 256 (four CTAs per SM) for the large levels; 512 (two
// CTAs per SM, every Y item of a batch of planes in one round) measured
// faster on the coarser levels, slower on the finest.
template <class T, int UX, int UY, int Q, bool Tma, bool Z = true, int NT = 256> struct FwdStreamOp {
    // 256 threads: four CTAs per SM (64 registers), measured faster than
    // three with more registers, for both staging forms
    static constexpr int kThreads = NT, kMinBlocks = NT == 512 ? 2 : 4;
    static constexpr bool kGridConstant = true;
    struct Params {
        CUtensorMap map;
        FwdSrc<T> src;
        Dims a;
        uint32_t tiles_x, tiles_y, zrange;
        FwdOut<T> out;
        uint32_t* status;
    };
    static __device__ __forceinline__ void run(const Params& P, uint32_t block, uint32_t);
    static __device__ __forceinline__ void acquire_maps(const Params& P) {
        if (Tma) tensormap_acquire(&P.map);
    }
};

template <class T, int UX, int UY, int Q, bool Tma, bool Z, int NT>
__device__ __forceinline__ void FwdStreamOp<T, UX, UY, Q, Tma, Z, NT>::run(const Params& P, uint32_t block, uint32_t) {
    const FwdSrc<T> src = P.src;
    const Dims a = P.a;
    const uint32_t tiles_x = P.tiles_x, tiles_y = P.tiles_y, zrange = P.zrange;
    const FwdOut<T> out = P.out;
    uint32_t* const status = P.status;
    const CUtensorMap* map = &P.map;
    using S = StreamShape<T, UX, UY, Q, NT>;
    using L = Lift<T>;
    using Bits = decltype(abs_bits(T(0)));
    extern __shared__ __align__(128) unsigned char stream_smem[];
    T* In = reinterpret_cast<T*>(stream_smem + ((128 - (smem_u32(stream_smem) & 127)) & 127)); // [Q][FY][FX]
    T* Mid = In + S::IN;                                                                  // [Q][UY][YP]
    uint64_t* bar = reinterpret_cast<uint64_t*>(Mid + S::MID);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t bx = block % tiles_x, by = (block / tiles_x) % tiles_y;
    const uint32_t bzr = block / (tiles_x * tiles_y);
    const uint32_t ox = bx * UX, oy = by * UY;
    const uint32_t z0 = bzr * zrange, z1 = min(a.z, z0 + zrange);
    if (z0 >= z1) return;
    // input planes [zin0, zin1): with Z, pairs from z0 - 4 until the pair
    // that completes output z1 - 1; an XY level reads its output planes only
    const int64_t zin0 = Z ? int64_t(z0) - 4 : int64_t(z0);
    const int64_t zin1 = Z ? 2 * (int64_t((z1 - 1) / 2) + 2) + 2 : int64_t(z1);
    const bool check = src.status != nullptr;
    const bool edge = ox < 4 || ox + UX + 4 > a.x || oy < 4 || oy + UY + 4 > a.y;
    const int fx_lo = ox < 4 ? int(4 - ox) : 0, fx_hi = min(S::FX, int(a.x - ox) + 4);
    const int fy_lo = oy < 4 ? int(4 - oy) : 0, fy_hi = min(S::FY, int(a.y - oy) + 4);

    // per-thread output columns: x/y parts of the split addresses
    size_t hi_off[S::CPT], lo_off[S::CPT];
    bool even_xy[S::CPT];
    ZPipe<T> pipe[S::CPT];
#pragma unroll
    for (int c = 0; c < S::CPT; ++c) {
        const int k = tid + c * NT;
        const uint32_t x = ox + k % UX, y = oy + k / UX;
        const uint32_t cx = split_of(x, a.x), cy = split_of(y, a.y);
        hi_off[c] = size_t(cy) * out.sy + cx;
        lo_off[c] = size_t(cy) * out.lo.x + cx;
        even_xy[c] = out.low && !(x & 1) && !(y & 1);
        pipe[c] = ZPipe<T>{T(0), T(0), T(0), T(0), T(0)};
    }
    const uint32_t zhalf = half_len(a.z);
    const size_t lo_plane = size_t(out.lo.x) * out.lo.y;
    Bits seen = 0;

    auto issue = [&](int64_t zb) { // one thread: arm the barrier and copy Q planes
        fence_proxy_async();
        mbar_expect_tx(bar, uint32_t(Q * S::FY * S::FX * sizeof(T)));
#pragma unroll 1
        for (int q = 0; q < Q; ++q)
            tma_load_3d(In + q * S::FY * S::FX, map, int(ox) - 4, int(oy) - 4, int(mirror(zb + q, a.z)), bar);
    };
    uint32_t phase = 0;
    if constexpr (Tma) {
        if (tid == 0) {
            mbar_init(bar, 1);
            fence_barrier_init();
        }
        __syncthreads();
        if (tid == 0) issue(zin0);
    }

    for (int64_t zb = zin0; zb < zin1; zb += Q) {
        if constexpr (Tma) {
            // warp 0 polls the barrier; the other warps park at the block
            // barrier instead of spinning on issue slots
            const bool ok = __syncthreads_and(warp != 0 || mbar_wait(bar, phase, kWaitBound));
            if (!ok) {
                if (tid == 0) atomicOr(status, ST_WAIT_TIMEOUT);
                return;
            }
            phase ^= 1;
            if (edge) {
                // cells outside the array only (the in-range box of a plane
                // is [f*_lo, f*_hi)): cells of in-range rows left or right of
                // it, then whole out-of-range rows, as one flat list; each is
                // reflected from inside the box, or loaded when its reflection
                // lies outside the box
                const int nx_out = fx_lo + (S::FX - fx_hi), ny_in = fy_hi - fy_lo, ny_out = S::FY - ny_in;
                const int na = Q * ny_in * nx_out, nb = Q * ny_out * S::FX;
                for (int i = tid; i < na + nb; i += NT) {
                    int fx, fy, q;
                    if (i < na) {
                        const int k = i % nx_out, row = i / nx_out;
                        fy = fy_lo + row % ny_in;
                        q = row / ny_in;
                        fx = k < fx_lo ? k : fx_hi + (k - fx_lo);
                    } else {
                        const int j = i - na, rr = j / S::FX, ks = rr % ny_out;
                        fx = j % S::FX;
                        q = rr / ny_out;
                        fy = ks < fy_lo ? ks : fy_hi + (ks - fy_lo);
                    }
                    const int64_t x = int64_t(ox) + fx - 4, y = int64_t(oy) + fy - 4;
                    const uint32_t mx = mirror(x, a.x), my = mirror(y, a.y);
                    const int64_t bxm = int64_t(mx) - (int64_t(ox) - 4), bym = int64_t(my) - (int64_t(oy) - 4);
                    T v;
                    if (bxm >= 0 && bxm < S::FX && bym >= 0 && bym < S::FY)
                        v = In[(q * S::FY + int(bym)) * S::FX + int(bxm)];
                    else
                        v = src.get(src.row(my, mirror(zb + q, a.z)), mx);
                    In[(q * S::FY + fy) * S::FX + fx] = v;
                }
                fence_proxy_async(); // these writes precede the next copy into In
                __syncthreads();
            }
        } else {
            // ---- stage Q planes x FY rows of FX samples (reflected)
            constexpr int ROWS = Q * S::FY;
            constexpr int kBatch = 6;
            const uint32_t x0 = mirror(int64_t(ox) + lane - 4, a.x), x1 = mirror(int64_t(ox) + lane + 28, a.x);
            const bool has0 = lane < S::FX, has1 = lane + 32 < S::FX;
            for (int r0 = warp; r0 < ROWS; r0 += (NT / 32) * kBatch) {
                T v0[kBatch], v1[kBatch];
#pragma unroll
                for (int u = 0; u < kBatch; ++u) {
                    const int r = r0 + u * (NT / 32);
                    v0[u] = T(0);
                    v1[u] = T(0);
                    if (r < ROWS) {
                        const int q = r / S::FY, fy = r % S::FY;
                        const auto row = src.row(mirror(int64_t(oy) + fy - 4, a.y), mirror(zb + q, a.z));
                        if (has0) v0[u] = src.get(row, x0);
                        if (has1) v1[u] = src.get(row, x1);
                    }
                }
#pragma unroll
                for (int u = 0; u < kBatch; ++u) {
                    const int r = r0 + u * (NT / 32);
                    if (r < ROWS) {
                        T* dst = In + r * S::FX;
                        if (has0) dst[lane] = v0[u];
                        if (has1) dst[lane + 32] = v1[u];
                    }
                }
            }
            __syncthreads();
        }
        // ---- Y: one window of UY outputs per (plane, column); every staged
        // sample is read here exactly once, so the finiteness check rides along
        {
            constexpr int P = UY / 2 + 4;
            for (int item = tid; item < Q * S::FX; item += NT) {
                const int q = item / S::FX, fx = item % S::FX;
                const T* s = In + q * S::FY * S::FX + fx;
                T e[P], o[P];
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    e[j] = s[(2 * j) * S::FX];
                    o[j] = s[(2 * j + 1) * S::FX];
                }
                if (check) {
#pragma unroll
                    for (int j = 0; j < P; ++j) seen = max(seen, max(abs_bits(e[j]), abs_bits(o[j])));
                }
                lift_forward<T, P>(e, o);
                T* d = Mid + q * UY * S::YP + fx;
#pragma unroll
                for (int j = 2; j < P - 2; ++j) {
                    d[(2 * (j - 2)) * S::YP] = e[j];
                    d[(2 * (j - 2) + 1) * S::YP] = o[j];
                }
            }
        }
        __syncthreads();
        if constexpr (Tma) {
            if (tid == 0 && zb + Q < zin1) issue(zb + Q); // In is free: overlap the next copy
        }
        // ---- X: windows of 16 outputs per (plane, row), in place in Mid
        {
            constexpr int WX = 16, P = WX / 2 + 4, WIN = UX / WX;
            constexpr int ITEMS = Q * UY * WIN;
            static_assert(ITEMS <= NT, "one X window per thread");
            const int item = tid;
            T e[P], o[P];
            T* rowp = nullptr;
            if (item < ITEMS) {
                const int row = item % (Q * UY), win = item / (Q * UY);
                rowp = Mid + row * S::YP + win * WX;
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    e[j] = rowp[2 * j];
                    o[j] = rowp[2 * j + 1];
                }
                lift_forward<T, P>(e, o);
            }
            __syncthreads();
            if (item < ITEMS) {
#pragma unroll
                for (int j = 2; j < P - 2; ++j) {
                    rowp[2 * (j - 2)] = e[j];
                    rowp[2 * (j - 2) + 1] = o[j];
                }
            }
        }
        __syncthreads();
        if constexpr (!Z) {
            // ---- an XY level: every lifted plane is an output plane
#pragma unroll
            for (int c = 0; c < S::CPT; ++c) {
                const int k = tid + c * NT;
                if (k >= S::COLS) break;
                const int x = k % UX, y = k / UX;
                if (ox + x >= a.x || oy + y >= a.y) continue;
                const T* s = Mid + y * S::YP + x;
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int64_t zo = zb + q;
                    if (zo >= int64_t(z1)) break;
                    const T v = s[q * UY * S::YP];
                    if (even_xy[c]) out.low[size_t(zo) * lo_plane + lo_off[c]] = v;
                    else out.dst[size_t(zo) * out.sz + hi_off[c]] = v;
                }
            }
        } else {
            // ---- Z: feed the Q lifted planes pair by pair into the column pipes
#pragma unroll
            for (int c = 0; c < S::CPT; ++c) {
                const int k = tid + c * NT;
                if (k >= S::COLS) break;
                const int x = k % UX, y = k / UX;
                const bool inside = ox + x < a.x && oy + y < a.y;
                const T* s = Mid + y * S::YP + x;
                ZPipe<T>& p = pipe[c];
#pragma unroll
                for (int q = 0; q < Q; q += 2) {
                    const T en = s[q * UY * S::YP], on = s[(q + 1) * UY * S::YP];
                    const T o1 = L::fma(K97<T>::a, L::add(p.e, en), p.o);
                    const T e2 = L::fma(K97<T>::b, L::add(p.o1, o1), p.e);
                    const T o3 = L::fma(K97<T>::g, L::add(p.e2, e2), p.o1);
                    const T e4 = L::fma(K97<T>::d, L::add(p.o3, o3), p.e2);
                    const int64_t zo = zb + q - 4; // even output plane of this pair
                    if (inside && zo >= int64_t(z0) && zo < int64_t(z1)) {
                        const size_t cz = size_t(zo) >> 1;
                        const T ev = L::mul(e4, K97<T>::k);
                        if (even_xy[c]) out.low[cz * lo_plane + lo_off[c]] = ev;
                        else out.dst[cz * out.sz + hi_off[c]] = ev;
                        if (zo + 1 < int64_t(z1)) out.dst[(zhalf + cz) * out.sz + hi_off[c]] = L::mul(o3, -K97<T>::ik);
                    }
                    p.o3 = o3;
                    p.e2 = e2;
                    p.o1 = o1;
                    p.e = en;
                    p.o = on;
                }
            }
        }
        // the next iteration's barrier vote orders these Mid reads before the
        // next Y pass writes Mid
    }
    if (check) {
        if (__syncthreads_or(nonfinite_max(seen)) && threadIdx.x == 0) atomicOr(src.status, ST_NONFINITE_INPUT);
    }
}

} // namespace wb

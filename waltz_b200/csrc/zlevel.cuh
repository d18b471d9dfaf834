// One Z level of the plane schedule as a per-column march in registers.
//
// A thread owns one (x, y) column of the level and a run of its Z windows; a
// warp's 32 lanes take 32 consecutive x of one row, so every load and store
// of a z row is one 128-byte line and nothing is staged in shared memory.
// Window w covers outputs [W*w, W*w + W) and reads the P = W/2 + 4 pairs at
// spatial positions W*w - 4 + 2j (even) and + 1 (odd), reflected at the
// column's ends exactly as the tile kernels reflect them. Consecutive windows
// share their last / first 4 pairs: those are kept raw in registers, so a
// later window loads only its W/2 new pairs.
//  * forward: windows of 16 (the analysis is window independent);
//  * inverse: the canonical folded windows (16 outputs for float, 8 for
//    double, origins at multiples of W; cpu/src/transform.cpp:110-147), so
//    every output takes the arithmetic of the tile kernels' Z pass.
// Forward sources are checked for finiteness when they carry a status word
// (the finest level reads every input sample at least once).
#pragma once
#include "transform.cuh"

namespace wb {

template <class T, bool Inverse> struct ZMarchShape {
    static constexpr int W = Inverse ? inverse_zwin<T>() : 16; // outputs per window
    static constexpr int P = W / 2 + 4;                        // pairs per window
    static constexpr int NEW = W / 2;                          // pairs each later window loads
    static constexpr int KEEP = P - NEW;                       // pairs shared with the next window
};

template <class T, bool Inverse, class Src, class Out> struct ZMarchOp {
    static constexpr int kThreads = 256, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        Src src;
        Dims a;
        Out out;
        uint32_t seg;  // windows per thread
        uint32_t tx;   // groups of 32 columns along x
    };
    static __device__ __forceinline__ void run(const Params& P, uint32_t block, uint32_t);
};

// Column accessors: at(z) reads the sample (forward) or the split-band
// coefficient (inverse: even positions from the low half, odd ones from the
// high half) of spatial position z after reflection; `m` is the level's z
// length.
// pairs(p0, from, e, o) fills pairs from .. PP-1 of the window whose pair 0
// starts at spatial position p0: windows inside the column read with one
// pointer per half and no reflection, edge windows through at().
template <class T> struct ZColFwd {
    const T* p;   // column base
    size_t s;     // z stride
    uint32_t m;
    __device__ __forceinline__ T at(int64_t z) const { return p[size_t(mirror(z, m)) * s]; }
    template <int PP> __device__ __forceinline__ void pairs(int64_t p0, int from, T (&e)[PP], T (&o)[PP]) const {
        if (p0 >= 0 && p0 + 2 * PP <= int64_t(m)) {
            const T* b = p + size_t(p0) * s;
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                if (j < from) continue;
                e[j] = b[size_t(2 * j) * s];
                o[j] = b[size_t(2 * j + 1) * s];
            }
        } else {
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                if (j < from) continue;
                e[j] = at(p0 + 2 * j);
                o[j] = at(p0 + 2 * j + 1);
            }
        }
    }
};
template <class T> struct ZColInv {
    const T* lo;  // low coefficients: index i at lo[i * ls]
    size_t ls;
    const T* hi;  // high coefficients: index i at hi[i * s]
    size_t s;
    uint32_t m;
    __device__ __forceinline__ T at(int64_t z) const {
        const uint32_t r = mirror(z, m);
        return (r & 1) ? hi[size_t(r >> 1) * s] : lo[size_t(r >> 1) * ls];
    }
    template <int PP> __device__ __forceinline__ void pairs(int64_t p0, int from, T (&e)[PP], T (&o)[PP]) const {
        if (p0 >= 0 && p0 + 2 * PP <= int64_t(m)) {
            // p0 is even: pair j's even sample is low coefficient p0/2 + j,
            // its odd one high coefficient p0/2 + j
            const T* lb = lo + size_t(p0 >> 1) * ls;
            const T* hb = hi + size_t(p0 >> 1) * s;
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                if (j < from) continue;
                e[j] = lb[size_t(j) * ls];
                o[j] = hb[size_t(j) * s];
            }
        } else {
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                if (j < from) continue;
                e[j] = at(p0 + 2 * j);
                o[j] = at(p0 + 2 * j + 1);
            }
        }
    }
};

template <class T, bool Inverse, class Src, class Out>
__device__ __forceinline__ void ZMarchOp<T, Inverse, Src, Out>::run(const Params& Pm, uint32_t block, uint32_t) {
    using Sh = ZMarchShape<T, Inverse>;
    constexpr int W = Sh::W, PP = Sh::P, KEEP = Sh::KEEP;
    const Dims a = Pm.a;
    const Out out = Pm.out;
    const uint32_t m = a.z, wins = (m + W - 1) / W, nseg = (wins + Pm.seg - 1) / Pm.seg;
    const uint64_t warp = uint64_t(block) * (kThreads / 32) + threadIdx.x / 32;
    const uint32_t lane = threadIdx.x & 31;
    if (warp >= uint64_t(Pm.tx) * a.y * nseg) return;
    const uint32_t xg = uint32_t(warp % Pm.tx), rest = uint32_t(warp / Pm.tx);
    const uint32_t y = rest % a.y, sg = rest / a.y;
    const uint32_t x = xg * 32 + lane;
    const bool live = x < a.x;
    const uint32_t xs = live ? x : a.x - 1; // lanes past the row read a live column and store nothing
    const uint32_t w0 = sg * Pm.seg, w1 = min(w0 + Pm.seg, wins);

    auto column = [&]() {
        if constexpr (Inverse) {
            const Src& s = Pm.src;
            const size_t off = size_t(y) * s.sy + xs;
            ZColInv<T> c;
            // the compact low band holds the z-even half of the columns it
            // covers: every column of a plane-schedule Z level, the x/y-low
            // corner of a dyadic level
            if (s.low && xs < s.lo.x && y < s.lo.y) {
                c.lo = s.low + size_t(y) * s.lo.x + xs;
                c.ls = size_t(s.lo.x) * s.lo.y;
            } else {
                c.lo = s.base + off;
                c.ls = s.sz;
            }
            c.hi = s.base + size_t(half_len(m)) * s.sz + off;
            c.s = s.sz;
            c.m = m;
            return c;
        } else {
            const Src& s = Pm.src;
            return ZColFwd<T>{s.p + size_t(y) * s.sy + xs, s.sz, m};
        }
    };
    const auto col = column();
    bool bad = false;
    T ke[KEEP], ko[KEEP]; // raw pairs the next window shares
    for (uint32_t w = w0; w < w1; ++w) {
        const int64_t p0 = int64_t(w) * W - 4; // spatial position of pair 0's even sample
        T e[PP], o[PP];
        if (w == w0) {
            col.template pairs<PP>(p0, 0, e, o);
        } else {
#pragma unroll
            for (int j = 0; j < KEEP; ++j) {
                e[j] = ke[j];
                o[j] = ko[j];
            }
            col.template pairs<PP>(p0, KEEP, e, o);
        }
#pragma unroll
        for (int j = 0; j < KEEP; ++j) {
            ke[j] = e[PP - KEEP + j];
            ko[j] = o[PP - KEEP + j];
        }
        if constexpr (!Inverse) {
            if (Pm.src.status) {
#pragma unroll
                for (int j = KEEP; j < PP; ++j) bad |= !finite_bits(e[j]) || !finite_bits(o[j]);
                if (w == w0) {
#pragma unroll
                    for (int j = 0; j < KEEP; ++j) bad |= !finite_bits(e[j]) || !finite_bits(o[j]);
                }
            }
        }
        const uint32_t z0 = w * W;
        if constexpr (Inverse) {
            T pre[W];
            if constexpr (Out::kPrefetch) {
#pragma unroll
                for (int k = 0; k < W; ++k) pre[k] = (live && z0 + k < m) ? out.fetch(x, y, z0 + k) : T(0);
            }
            lift_inverse<T, PP, true>(e, o);
            if (live) {
#pragma unroll
                for (int j = 2; j < PP - 2; ++j) {
                    const uint32_t z = z0 + 2 * (j - 2);
                    if constexpr (Out::kPrefetch) {
                        if (z < m) out.emit(x, y, z, e[j], pre[2 * (j - 2)]);
                        if (z + 1 < m) out.emit(x, y, z + 1, o[j], pre[2 * (j - 2) + 1]);
                    } else if constexpr (RowStore<Out>::value) {
                        T* const c = out.dst + size_t(z) * out.sz + size_t(y) * out.sy + x;
                        if (z < m) c[0] = e[j];
                        if (z + 1 < m) c[out.sz] = o[j];
                    } else {
                        if (z < m) out(x, y, z, e[j]);
                        if (z + 1 < m) out(x, y, z + 1, o[j]);
                    }
                }
            }
        } else {
            lift_forward<T, PP>(e, o);
            if (live) {
                // a Z level's split positions (the output's mask is AZ):
                // even z -> z / 2, in the compact low band for the columns
                // it covers (all of a plane-schedule level, the x/y-low
                // corner of a dyadic level); odd z -> hz + z / 2
                T* const cd = out.dst + size_t(y) * out.sy + x;
                T* const cl = (out.low && x < out.lo.x && y < out.lo.y) ? out.low + size_t(y) * out.lo.x + x : nullptr;
                const size_t ls = size_t(out.lo.x) * out.lo.y;
                const uint32_t hz = half_len(m);
#pragma unroll
                for (int j = 2; j < PP - 2; ++j) {
                    const uint32_t z = z0 + 2 * (j - 2);
                    if (z < m) {
                        if (cl) cl[size_t(z >> 1) * ls] = e[j];
                        else cd[size_t(z >> 1) * out.sz] = e[j];
                    }
                    if (z + 1 < m) cd[size_t(hz + (z >> 1)) * out.sz] = o[j];
                }
            }
        }
    }
    if constexpr (!Inverse) {
        if (bad && Pm.src.status) atomicOr(Pm.src.status, ST_NONFINITE_INPUT);
    }
}

} // namespace wb

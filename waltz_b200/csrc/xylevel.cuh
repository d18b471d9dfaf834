// One XY level of the plane schedule as a warp march in registers.
//
// A warp owns a strip of 64 consecutive x (56 outputs and a 4-sample halo
// per side) on one z plane, and marches down y through a run of Y windows;
// a lane keeps its two columns' windows in registers, exactly as the Z march
// (zlevel.cuh) does along z. Lane l holds the pair of spatial x = x0 + 2l
// (even) and x0 + 2l + 1 (odd), x0 even: in the split-band layout that pair
// is low-half and high-half coefficient x0/2 + l, so a warp reads a
// coefficient row as two contiguous 128-byte runs. The X lifting of a row
// runs across the lanes: every lifting step updates one sample of each pair
// from the other sample of its own pair and one of the neighbouring lane's,
// one shuffle per step. After the four steps pairs 2..29 hold exact results
// (each output depends only on its 4-sample neighbourhood, the reason the
// forward analysis and the inverse X synthesis are window independent);
// lanes 0-1 and 30-31 are the halo.
//  * forward (order Y, X): a window's rows are lifted along Y in registers
//    (windows of 8, any size and origin give the same bits; 8 keeps the
//    registers to about 80, three CTAs per SM), then each output row along X
//    across the lanes;
//  * inverse (order X, Y): every coefficient row a window loads is first
//    lifted along X across the lanes, then the window along Y in the
//    canonical folded windows of 8 (origins at multiples of 8,
//    cpu/src/transform.cpp:110-147).
// Each lane reads its columns of every row it needs once per window (the 4
// pairs of rows shared with the next window stay in registers); nothing is
// staged in shared memory.
#pragma once
#include "transform.cuh"

namespace wb {

template <class T, bool Inverse> struct XYMarchShape {
    static constexpr int W = 8;                // Y outputs per window
    static constexpr int P = W / 2 + 4;        // pairs of rows per window
    static constexpr int KEEP = 4;             // pairs of rows shared with the next window
    static constexpr int U = 56;               // x outputs per warp (lanes 2..29, two each)
};

// Lane-wise lifting of one row held as one (even, odd) pair per lane (lane l
// = pair x0/2 + l). The step order, operands and operand order are those of
// lift_forward / lift_inverse<..., false> (common.cuh): an odd update adds
// the pair's own even sample and the next lane's, an even update the
// previous lane's odd sample and the pair's own.
template <class T> __device__ __forceinline__ void pair_odd(T& o, T e, T c) {
    const T next = __shfl_down_sync(0xffffffffu, e, 1);
    o = Lift<T>::fma(c, Lift<T>::add(e, next), o);
}
template <class T> __device__ __forceinline__ void pair_even(T& e, T o, T c) {
    const T prev = __shfl_up_sync(0xffffffffu, o, 1);
    e = Lift<T>::fma(c, Lift<T>::add(prev, o), e);
}
template <class T> __device__ __forceinline__ void pair_forward(T& e, T& o) {
    using L = Lift<T>;
    pair_odd(o, e, K97<T>::a);
    pair_even(e, o, K97<T>::b);
    pair_odd(o, e, K97<T>::g);
    pair_even(e, o, K97<T>::d);
    e = L::mul(e, K97<T>::k);
    o = L::mul(o, -K97<T>::ik);
}
template <class T> __device__ __forceinline__ void pair_inverse(T& e, T& o) {
    using L = Lift<T>;
    e = L::mul(e, K97<T>::ik);
    o = L::mul(o, -K97<T>::k);
    pair_even(e, o, -K97<T>::d);
    pair_odd(o, e, -K97<T>::g);
    pair_even(e, o, -K97<T>::b);
    pair_odd(o, e, -K97<T>::a);
}

template <class T, bool Inverse, class Src, class Out> struct XYMarchOp {
    static constexpr int kThreads = 256, kMinBlocks = 0; // no occupancy floor: about 80 registers, three CTAs per SM
    struct Params {
        Src src;
        Dims a;   // level dims (x, y lifted; z planes)
        Out out;
        uint32_t seg; // Y windows per warp
        uint32_t tx;  // strips of 56 x
    };
    static __device__ __forceinline__ void run(const Params& P, uint32_t block, uint32_t);
};

template <class T, bool Inverse, class Src, class Out>
__device__ __forceinline__ void XYMarchOp<T, Inverse, Src, Out>::run(const Params& Pm, uint32_t block, uint32_t) {
    using Sh = XYMarchShape<T, Inverse>;
    constexpr int W = Sh::W, PP = Sh::P, KEEP = Sh::KEEP;
    const Dims a = Pm.a;
    const Out out = Pm.out;
    const Src src = Pm.src;
    const uint32_t wins = (a.y + W - 1) / W, nseg = (wins + Pm.seg - 1) / Pm.seg;
    const uint64_t warp = uint64_t(block) * (kThreads / 32) + threadIdx.x / 32;
    const int lane = int(threadIdx.x & 31);
    if (warp >= uint64_t(Pm.tx) * nseg * a.z) return; // whole warps only: every lane shuffles
    const uint32_t xs = uint32_t(warp % Pm.tx);
    const uint64_t rest = warp / Pm.tx;
    const uint32_t sg = uint32_t(rest % nseg), z = uint32_t(rest / nseg);
    const int64_t xe = int64_t(xs) * Sh::U - 4 + 2 * lane; // this lane's even x; the odd one is xe + 1
    const bool live = lane >= 2 && lane < 2 + Sh::U / 2;
    const bool live_e = live && xe < int64_t(a.x), live_o = live && xe + 1 < int64_t(a.x);
    const uint32_t hx = half_len(a.x), hy = half_len(a.y);
    // columns read for this lane: split-band positions (inverse) or spatial
    // ones (forward), reflected at the row's ends; inside the row the pair is
    // low / high coefficient xe / 2 (inverse) or samples xe, xe + 1 (forward).
    // Reflection keeps parity, so the even column is always a low-half
    // coefficient and the odd one a high-half one.
    const bool inside = xe >= 0 && xe + 1 < int64_t(a.x);
    const uint32_t me = inside ? uint32_t(xe) : mirror(xe, a.x), mo = inside ? uint32_t(xe + 1) : mirror(xe + 1, a.x);
    const uint32_t ce = Inverse ? split_of(me, a.x) : me, co = Inverse ? split_of(mo, a.x) : mo;
    const uint32_t w0 = sg * Pm.seg, w1 = min(w0 + Pm.seg, wins);

    // the plane's rows: inverse, coefficient row cy of the base array (and of
    // the compact low band for cy < hy, the even rows); forward, sample row y
    const T* plane;
    const T* lplane = nullptr;
    size_t rs, lrs = 0; // row strides
    if constexpr (Inverse) {
        plane = src.base + size_t(z) * src.sz;
        rs = src.sy;
        if (src.low) {
            lplane = src.low + size_t(z) * src.lo.y * src.lo.x;
            lrs = src.lo.x;
        }
    } else {
        plane = src.p + size_t(z) * src.sz;
        rs = src.sy;
    }
    // the two columns of spatial row p, reflected into the level
    auto row = [&](int64_t p, T& ve, T& vo) {
        const uint32_t my = mirror(p, a.y);
        if constexpr (Inverse) {
            const uint32_t cy = split_of(my, a.y);
            const T* b = plane + size_t(cy) * rs;
            ve = (lplane && cy < hy) ? lplane[size_t(cy) * lrs + ce] : b[ce];
            vo = b[co];
        } else {
            const T* b = plane + size_t(my) * rs;
            ve = b[ce];
            vo = b[co];
        }
    };
    bool bad = false;
    T ke[KEEP][2], ko[KEEP][2]; // pairs of rows the next window shares (inverse: already lifted along X)
    for (uint32_t w = w0; w < w1; ++w) {
        const int64_t p0 = int64_t(w) * W - 4; // spatial row of pair 0's even row
        T e[PP][2], o[PP][2];                  // [row pair][even / odd column]
        const int from = w == w0 ? 0 : KEEP;
        if (from) {
#pragma unroll
            for (int j = 0; j < KEEP; ++j) {
                e[j][0] = ke[j][0], e[j][1] = ke[j][1];
                o[j][0] = ko[j][0], o[j][1] = ko[j][1];
            }
        }
        if (p0 >= 0 && p0 + 2 * PP <= int64_t(a.y)) {
            // a window inside the level: no reflection; inverse, pair j's even
            // row is coefficient row p0/2 + j and its odd row hy + p0/2 + j
            if constexpr (Inverse) {
                const uint32_t r0 = uint32_t(p0) >> 1;
                const T* be = plane + size_t(r0) * rs;
                const T* bo = plane + size_t(hy + r0) * rs;
                const T* le = lplane ? lplane + size_t(r0) * lrs : nullptr;
#pragma unroll
                for (int j = 0; j < PP; ++j) {
                    if (j < from) continue;
                    e[j][0] = le ? le[size_t(j) * lrs + ce] : be[size_t(j) * rs + ce];
                    e[j][1] = be[size_t(j) * rs + co];
                    o[j][0] = bo[size_t(j) * rs + ce];
                    o[j][1] = bo[size_t(j) * rs + co];
                }
            } else {
                const T* b = plane + size_t(p0) * rs;
#pragma unroll
                for (int j = 0; j < PP; ++j) {
                    if (j < from) continue;
                    e[j][0] = b[size_t(2 * j) * rs + ce];
                    e[j][1] = b[size_t(2 * j) * rs + co];
                    o[j][0] = b[size_t(2 * j + 1) * rs + ce];
                    o[j][1] = b[size_t(2 * j + 1) * rs + co];
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                if (j < from) continue;
                row(p0 + 2 * j, e[j][0], e[j][1]);
                row(p0 + 2 * j + 1, o[j][0], o[j][1]);
            }
        }
        if constexpr (Inverse) {
            // X first: every newly loaded coefficient row across the lanes
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                if (j < from) continue;
                pair_inverse(e[j][0], e[j][1]);
                pair_inverse(o[j][0], o[j][1]);
            }
        } else if (src.status) {
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                if (j < from) continue;
                bad |= !finite_bits(e[j][0]) || !finite_bits(e[j][1]) || !finite_bits(o[j][0]) ||
                       !finite_bits(o[j][1]);
            }
        }
#pragma unroll
        for (int j = 0; j < KEEP; ++j) {
            ke[j][0] = e[PP - KEEP + j][0], ke[j][1] = e[PP - KEEP + j][1];
            ko[j][0] = o[PP - KEEP + j][0], ko[j][1] = o[PP - KEEP + j][1];
        }
        const uint32_t y0 = w * W;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            // one column of the pair along Y, in registers
            T ye[PP], yo[PP];
#pragma unroll
            for (int j = 0; j < PP; ++j) ye[j] = e[j][c], yo[j] = o[j][c];
            if constexpr (Inverse) lift_inverse<T, PP, true>(ye, yo);
            else lift_forward<T, PP>(ye, yo);
#pragma unroll
            for (int j = 0; j < PP; ++j) e[j][c] = ye[j], o[j][c] = yo[j];
        }
        const uint32_t x = uint32_t(xe);
#pragma unroll
        for (int j = 2; j < PP - 2; ++j) {
            const uint32_t y = y0 + 2 * (j - 2); // even; the pair's odd row is y + 1
            if constexpr (!Inverse) {
                pair_forward(e[j][0], e[j][1]); // X, across the lanes
                pair_forward(o[j][0], o[j][1]);
                // an XY level's split positions: x even -> xe / 2, odd ->
                // hx + xe / 2; y even -> y / 2 (the all-even corner to the
                // compact low band when there is one), odd -> hy + y / 2
                const size_t ye_row = size_t(z) * out.sz + size_t(y >> 1) * out.sy;
                const size_t yo_row = size_t(z) * out.sz + size_t(hy + (y >> 1)) * out.sy;
                const uint32_t cxe = x >> 1, cxo = hx + (x >> 1);
                if (y < a.y) {
                    if (live_e) {
                        if (out.low) out.low[(size_t(z) * out.lo.y + (y >> 1)) * out.lo.x + cxe] = e[j][0];
                        else out.dst[ye_row + cxe] = e[j][0];
                    }
                    if (live_o) out.dst[ye_row + cxo] = e[j][1];
                }
                if (y + 1 < a.y) {
                    if (live_e) out.dst[yo_row + cxe] = o[j][0];
                    if (live_o) out.dst[yo_row + cxo] = o[j][1];
                }
            } else if constexpr (RowStore<Out>::value) {
                T* re = out.dst + size_t(z) * out.sz + size_t(y) * out.sy + x;
                T* ro = re + out.sy;
                if (y < a.y) {
                    if (live_e) re[0] = e[j][0];
                    if (live_o) re[1] = e[j][1];
                }
                if (y + 1 < a.y) {
                    if (live_e) ro[0] = o[j][0];
                    if (live_o) ro[1] = o[j][1];
                }
            } else {
                if (y < a.y) {
                    if (live_e) out(x, y, z, e[j][0]);
                    if (live_o) out(x + 1, y, z, e[j][1]);
                }
                if (y + 1 < a.y) {
                    if (live_e) out(x, y + 1, z, o[j][0]);
                    if (live_o) out(x + 1, y + 1, z, o[j][1]);
                }
            }
        }
    }
    if constexpr (!Inverse) {
        if (src.status && __any_sync(0xffffffffu, bad) && lane == 0) atomicOr(src.status, ST_NONFINITE_INPUT);
    }
}

} // namespace wb

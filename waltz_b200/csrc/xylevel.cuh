// One XY level of the plane schedule as a warp march in registers.
//
// A warp owns a strip of 32 consecutive x (24 outputs and a 4-sample halo
// per side) on one z plane, and marches down y through a run of Y windows;
// a lane keeps its column's window in registers, exactly as the Z march
// (zlevel.cuh) does along z, and the X lifting of a row runs across the
// warp's lanes with shuffles: lane l holds spatial x = x0 + l (x0 even), so
// even lanes hold the even samples and odd lanes the odd ones, and every
// lifting step reads the two neighbours with one shuffle each way. After the
// four steps lanes 4..27 hold exact results (each output depends only on its
// 4-sample neighbourhood, the reason the forward analysis and the inverse X
// synthesis are window independent); lanes 0-3 and 28-31 are the halo.
//  * forward (order Y, X): a window's rows are lifted along Y in registers
//    (windows of 16, any origin gives the same bits), then each output row
//    along X across the lanes;
//  * inverse (order X, Y): every coefficient row a window loads is first
//    lifted along X across the lanes, then the window along Y in the
//    canonical folded windows of 8 (origins at multiples of 8,
//    cpu/src/transform.cpp:110-147).
// Each lane reads its column of every row it needs once per window (the 4
// pairs shared with the next window stay in registers); a warp's loads and
// stores of a row are contiguous, nothing is staged in shared memory.
#pragma once
#include "transform.cuh"

namespace wb {

template <class T, bool Inverse> struct XYMarchShape {
    static constexpr int W = Inverse ? 8 : 16; // Y outputs per window
    static constexpr int P = W / 2 + 4;        // pairs per window
    static constexpr int KEEP = 4;             // pairs shared with the next window
    static constexpr int U = 24;               // x outputs per warp
};

// Lane-wise lifting of one row held one sample per lane (lane l = spatial
// x0 + l, x0 even). The step order, operands and operand order are those of
// lift_forward / lift_inverse<..., false> (common.cuh).
template <class T> __device__ __forceinline__ T lane_step(T v, T c, bool mine) {
    const T left = __shfl_up_sync(0xffffffffu, v, 1), right = __shfl_down_sync(0xffffffffu, v, 1);
    return mine ? Lift<T>::fma(c, Lift<T>::add(left, right), v) : v;
}
template <class T> __device__ __forceinline__ T lane_forward(T v, bool odd) {
    using L = Lift<T>;
    v = lane_step(v, K97<T>::a, odd);
    v = lane_step(v, K97<T>::b, !odd);
    v = lane_step(v, K97<T>::g, odd);
    v = lane_step(v, K97<T>::d, !odd);
    return odd ? L::mul(v, -K97<T>::ik) : L::mul(v, K97<T>::k);
}
template <class T> __device__ __forceinline__ T lane_inverse(T v, bool odd) {
    using L = Lift<T>;
    v = odd ? L::mul(v, -K97<T>::k) : L::mul(v, K97<T>::ik);
    v = lane_step(v, -K97<T>::d, !odd);
    v = lane_step(v, -K97<T>::g, odd);
    v = lane_step(v, -K97<T>::b, !odd);
    v = lane_step(v, -K97<T>::a, odd);
    return v;
}

template <class T, bool Inverse, class Src, class Out> struct XYMarchOp {
    static constexpr int kThreads = 256, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        Src src;
        Dims a;   // level dims (x, y lifted; z planes)
        Out out;
        uint32_t seg; // Y windows per warp
        uint32_t tx;  // strips of 24 x
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
    const int64_t x = int64_t(xs) * Sh::U - 4 + lane; // x0 = 24 xs - 4 is even: odd lanes hold odd x
    const bool odd = (lane & 1) != 0;
    const bool live = lane >= 4 && lane < 4 + Sh::U && x < int64_t(a.x);
    const uint32_t mx = mirror(x, a.x);
    const uint32_t w0 = sg * Pm.seg, w1 = min(w0 + Pm.seg, wins);

    // sample (forward) or coefficient (inverse) of this lane's column at
    // spatial row p, reflected into the level
    auto row = [&](int64_t p) -> T {
        const uint32_t my = mirror(p, a.y);
        if constexpr (Inverse) {
            const uint32_t cx = split_of(mx, a.x), cy = split_of(my, a.y);
            if (src.low && cx < src.lo.x && cy < src.lo.y)
                return src.low[(size_t(z) * src.lo.y + cy) * src.lo.x + cx];
            return src.base[size_t(z) * src.sz + size_t(cy) * src.sy + cx];
        } else {
            return src.p[size_t(z) * src.sz + size_t(my) * src.sy + mx];
        }
    };
    bool bad = false;
    T ke[KEEP], ko[KEEP]; // pairs the next window shares (inverse: already lifted along X)
    for (uint32_t w = w0; w < w1; ++w) {
        const int64_t p0 = int64_t(w) * W - 4; // spatial row of pair 0's even row
        T e[PP], o[PP];
        const int from = w == w0 ? 0 : KEEP;
        if (from) {
#pragma unroll
            for (int j = 0; j < KEEP; ++j) {
                e[j] = ke[j];
                o[j] = ko[j];
            }
        }
#pragma unroll
        for (int j = 0; j < PP; ++j) {
            if (j < from) continue;
            e[j] = row(p0 + 2 * j);
            o[j] = row(p0 + 2 * j + 1);
        }
        if constexpr (Inverse) {
            // X first: every newly loaded coefficient row across the lanes
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                if (j < from) continue;
                e[j] = lane_inverse(e[j], odd);
                o[j] = lane_inverse(o[j], odd);
            }
        } else if (src.status) {
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                if (j < from) continue;
                bad |= !finite_bits(e[j]) || !finite_bits(o[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < KEEP; ++j) {
            ke[j] = e[PP - KEEP + j];
            ko[j] = o[PP - KEEP + j];
        }
        const uint32_t y0 = w * W;
        if constexpr (Inverse) {
            T pre[W];
            if constexpr (Out::kPrefetch) {
#pragma unroll
                for (int k = 0; k < W; ++k)
                    pre[k] = (live && y0 + k < a.y) ? out.fetch(uint32_t(x), y0 + k, z) : T(0);
            }
            lift_inverse<T, PP, true>(e, o);
            if (live) {
#pragma unroll
                for (int j = 2; j < PP - 2; ++j) {
                    const uint32_t y = y0 + 2 * (j - 2);
                    if constexpr (Out::kPrefetch) {
                        if (y < a.y) out.emit(uint32_t(x), y, z, e[j], pre[2 * (j - 2)]);
                        if (y + 1 < a.y) out.emit(uint32_t(x), y + 1, z, o[j], pre[2 * (j - 2) + 1]);
                    } else {
                        if (y < a.y) out(uint32_t(x), y, z, e[j]);
                        if (y + 1 < a.y) out(uint32_t(x), y + 1, z, o[j]);
                    }
                }
            }
        } else {
            lift_forward<T, PP>(e, o); // Y, in registers
#pragma unroll
            for (int j = 2; j < PP - 2; ++j) {
                const uint32_t y = y0 + 2 * (j - 2);
                const T ve = lane_forward(e[j], odd), vo = lane_forward(o[j], odd); // X, across the lanes
                if (live && y < a.y) out(uint32_t(x), y, z, ve);
                if (live && y + 1 < a.y) out(uint32_t(x), y + 1, z, vo);
            }
        }
    }
    if constexpr (!Inverse) {
        if (src.status && __any_sync(0xffffffffu, bad) && lane == 0) atomicOr(src.status, ST_NONFINITE_INPUT);
    }
}

} // namespace wb

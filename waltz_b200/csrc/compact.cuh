// Compact repair records (the reference's opt-in WPW1 section,
// src/small_pwe.cuh:21-152 and include/utils/Blob.hpp:93-102): the repair
// errors of an archive stored as int8 multiples of a step where that is safe,
// in groups of 32 records.
//
// Section layout (little endian), replacing the native T[np] errors:
//   header  u32 magic "WPW1" (0x31575057), u32 groups = ceil(np/32),
//           u64 payload bytes, f64 step                            (24 bytes)
//   directory, per group: u32 offset into the payload (bit 31: the group is
//           stored natively), u32 mask of the records kept natively
//   payload, per group at its 8-byte aligned offset: native: count errors;
//           compact: count int8 codes (0 where native), padded to the
//           error size, then the natively kept errors in record order;
//           zero-padded to 8 bytes.
// A record is coded when code = nearbyint(e / step) fits int8 and the
// decoder's correction T(code * step) provably leaves the sample within
// `step` of the original (outward-rounded enclosure of the encoder's
// reconstruction, as the reference checks). A group is compact when that is
// smaller than storing it natively; the section is compact when smaller
// than the native errors. Payload offsets follow the group order (an
// exclusive scan), so the bytes are deterministic.
//
// Encoding runs after the ordered native sections are written: WpwSizeOp
// sizes every group, WpwScanOp places them and decides, WpwWriteOp builds
// the section and a copy of the q-outlier sections in scratch, WpwMoveOp
// moves that tail into the archive. Every kernel takes the record count from
// the layout words on the device, so the launches can be captured.
#pragma once
#include "common.cuh"
#include "scan.cuh"

#include <cmath>

namespace wb {

constexpr uint32_t kWpwMagic = 0x31575057u;
constexpr uint32_t kWpwHeader = 24, kWpwEntry = 8;
constexpr int kWpwThreads = 256; // 8 warps, one group of 32 records each

// Outward enclosure of (reconstruction - correction) - original, where the
// reconstruction r satisfies T(r - original) = e: r lies within one unit of
// e's last place of original + e. True when the enclosure is finite and
// inside [-budget, budget].
template <class T>
__device__ __forceinline__ bool wpw_safe(T original, T e, T correction, double budget) {
    if (!finite_bits(e) || !finite_bits(correction) || !finite_bits(original)) return false;
    double lo, hi;
    if constexpr (sizeof(T) == 4) {
        float l = __fadd_rd(original, nextafterf(e, -INFINITY));
        float h = __fadd_ru(original, nextafterf(e, INFINITY));
        l = __fsub_rd(l, correction);
        h = __fsub_ru(h, correction);
        lo = double(l) - double(original); // exact: float differences fit a double
        hi = double(h) - double(original);
    } else {
        double l = __dadd_rd(original, nextafter(e, -INFINITY));
        double h = __dadd_ru(original, nextafter(e, INFINITY));
        l = __dsub_rd(l, correction);
        h = __dsub_ru(h, correction);
        lo = __dsub_rd(l, original);
        hi = __dsub_ru(h, original);
    }
    return isfinite(lo) && isfinite(hi) && lo >= -budget && hi <= budget;
}

// One record's code (valid when the function returns true).
template <class T>
__device__ __forceinline__ bool wpw_code(T original, T e, double step, int& code) {
    const double r = nearbyint(double(e) / step);
    if (!(isfinite(r) && r >= -127.0 && r <= 127.0)) return false;
    code = int(r);
    return wpw_safe<T>(original, e, T(double(code) * step), step);
}

// Loads from the archive, whose base need not be aligned: typed loads when
// it is 8-byte aligned (every section starts on an 8-byte offset), bytes
// otherwise.
template <class V> __device__ __forceinline__ V wpw_load(const uint8_t* p, bool aligned) {
    if (aligned) return *reinterpret_cast<const V*>(p);
    V v;
    memcpy(&v, p, sizeof(V));
    return v;
}

__device__ __forceinline__ uint32_t wpw_group_bytes(uint32_t count, uint32_t native_mask, uint32_t width,
                                                    bool& compact) {
    const uint32_t raw_start = (count + width - 1) / width * width;
    const uint32_t small = raw_start + __popc(native_mask) * width, native = count * width;
    compact = small < native;
    return uint32_t(pad8(compact ? small : native));
}

// Layout words of the archive being written (see ScanLayoutOp): pi, pv, qi,
// qv, end, np, nq, overflow, status. The state words of the compaction:
// 0 compact?, 1 section bytes, 2 old qi, 3 old qv, 4 nq, 5 tail bytes
// (compact section + q-outlier sections, padded), 6 groups, 7 payload bytes.
template <class T> struct WpwSizeOp {
    static constexpr int kThreads = kWpwThreads, kMinBlocks = 0;
    struct Params {
        const uint64_t* layout;
        const uint8_t* archive;
        const T* original;
        double step;
        uint32_t* gbytes; // per group
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t blocks) {
        if (P.layout[7]) return;
        const uint32_t np = uint32_t(P.layout[5]), groups = (np + 31) / 32;
        const uint8_t* idx = P.archive + P.layout[0];
        const uint8_t* err = P.archive + P.layout[1];
        const bool al = (reinterpret_cast<uintptr_t>(P.archive) & 7u) == 0;
        const uint32_t lane = threadIdx.x & 31u;
        for (uint32_t g = block * (kThreads / 32) + threadIdx.x / 32; g < groups; g += blocks * (kThreads / 32)) {
            const uint32_t i = g * 32 + lane, count = min(32u, np - g * 32);
            bool coded = false;
            if (lane < count) {
                int code;
                coded = wpw_code<T>(P.original[wpw_load<uint32_t>(idx + 4 * size_t(i), al)],
                                    wpw_load<T>(err + sizeof(T) * size_t(i), al), P.step, code);
            }
            const uint32_t native = __ballot_sync(0xffffffffu, lane < count && !coded);
            bool compact;
            const uint32_t bytes = wpw_group_bytes(count, native, sizeof(T), compact);
            if (lane == 0) P.gbytes[g] = bytes;
        }
    }
};

// One CTA: group offsets (exclusive scan in place), the decision, the new
// layout and header fields.
struct WpwScanOp {
    static constexpr int kThreads = 1024, kMinBlocks = 0;
    struct Params {
        uint64_t* layout;
        uint8_t* archive;
        uint32_t* gbytes;
        uint64_t* state;
        uint32_t width;
        double step;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t, uint32_t) {
        __shared__ uint32_t tmp[40];
        const bool overflow = P.layout[7] != 0;
        const uint32_t np = overflow ? 0u : uint32_t(P.layout[5]), groups = (np + 31) / 32;
        const uint32_t per = (groups + kThreads - 1) / kThreads;
        const uint32_t g0 = min(groups, threadIdx.x * per), g1 = min(groups, g0 + per);
        uint64_t run = 0;
        for (uint32_t g = g0; g < g1; ++g) run += P.gbytes[g];
        // group sizes are at most 32 * 8 + 8 bytes: 32-bit partial sums
        uint32_t total;
        uint32_t at = block_excl_scan<kThreads>(uint32_t(run), tmp, total);
        for (uint32_t g = g0; g < g1; ++g) {
            const uint32_t v = P.gbytes[g];
            P.gbytes[g] = at;
            at += v;
        }
        if (threadIdx.x != 0) return;
        const uint64_t section = uint64_t(kWpwHeader) + uint64_t(kWpwEntry) * groups + total;
        const bool compact = np > 0 && section < uint64_t(np) * P.width;
        const uint64_t nq = P.layout[6];
        P.state[0] = compact;
        P.state[1] = section;
        P.state[2] = P.layout[2];
        P.state[3] = P.layout[3];
        P.state[4] = nq;
        P.state[5] = pad8(section) + 2 * pad8(nq * 4);
        P.state[6] = groups;
        P.state[7] = total;
        if (!compact) return;
        // the q-outlier sections move down behind the shorter repair section
        const uint64_t pv = P.layout[1];
        const uint64_t qi = pv + pad8(section), qv = qi + pad8(nq * 4), end = qv + pad8(nq * 4);
        P.layout[2] = qi;
        P.layout[3] = qv;
        P.layout[4] = end;
        P.archive[0] |= 2; // repair encoding: compact
        for (int k = 0; k < 4; ++k) P.archive[4 + k] = uint8_t(uint32_t(section) >> (8 * k));
    }
};

template <class T> struct WpwWriteOp {
    static constexpr int kThreads = kWpwThreads, kMinBlocks = 0;
    struct Params {
        const uint64_t* layout;
        const uint8_t* archive;
        const T* original;
        double step;
        const uint32_t* goff; // per group payload offset
        const uint64_t* state;
        uint8_t* wbuf;        // the tail: compact section, then the q-outlier sections
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t blocks) {
        if (!P.state[0]) return;
        const uint32_t np = uint32_t(P.layout[5]), groups = uint32_t(P.state[6]);
        const uint8_t* idx = P.archive + P.layout[0];
        const uint8_t* err = P.archive + P.layout[1];
        const bool al = (reinterpret_cast<uintptr_t>(P.archive) & 7u) == 0;
        uint8_t* dir = P.wbuf + kWpwHeader;
        uint8_t* payload = dir + size_t(kWpwEntry) * groups;
        const uint32_t lane = threadIdx.x & 31u;
        if (block == 0 && threadIdx.x == 0) {
            const uint64_t pb = P.state[7];
            uint64_t sb;
            memcpy(&sb, &P.step, 8);
            reinterpret_cast<uint32_t*>(P.wbuf)[0] = kWpwMagic;
            reinterpret_cast<uint32_t*>(P.wbuf)[1] = groups;
            reinterpret_cast<uint64_t*>(P.wbuf)[1] = pb;
            reinterpret_cast<uint64_t*>(P.wbuf)[2] = sb;
        }
        for (uint32_t g = block * (kThreads / 32) + threadIdx.x / 32; g < groups; g += blocks * (kThreads / 32)) {
            const uint32_t i = g * 32 + lane, count = min(32u, np - g * 32);
            bool coded = false;
            int code = 0;
            T e = T(0);
            if (lane < count) {
                e = wpw_load<T>(err + sizeof(T) * size_t(i), al);
                coded = wpw_code<T>(P.original[wpw_load<uint32_t>(idx + 4 * size_t(i), al)], e, P.step, code);
            }
            const uint32_t native = __ballot_sync(0xffffffffu, lane < count && !coded);
            bool compact;
            const uint32_t bytes = wpw_group_bytes(count, native, sizeof(T), compact);
            const uint32_t off = P.goff[g];
            uint8_t* out = payload + off;
            if (lane == 0) {
                reinterpret_cast<uint32_t*>(dir)[2 * g] = off | (compact ? 0u : 0x80000000u);
                reinterpret_cast<uint32_t*>(dir)[2 * g + 1] = compact ? native : 0u;
            }
            const uint32_t raw_start = (count + uint32_t(sizeof(T)) - 1) / uint32_t(sizeof(T)) * uint32_t(sizeof(T));
            uint32_t used;
            if (!compact) {
                if (lane < count) reinterpret_cast<T*>(out)[lane] = e;
                used = count * uint32_t(sizeof(T));
            } else {
                if (lane < count) {
                    out[lane] = uint8_t(int8_t(coded ? code : 0));
                    if (!coded)
                        reinterpret_cast<T*>(out + raw_start)[__popc(native & ((1u << lane) - 1u))] = e;
                }
                if (lane >= count && lane < raw_start) out[lane] = 0; // padding after the codes
                used = raw_start + __popc(native) * uint32_t(sizeof(T));
            }
            for (uint32_t b = used + lane; b < bytes; b += 32) out[b] = 0;
        }
        // the section's tail padding, then the q-outlier sections behind it
        const uint64_t section = P.state[1], sec8 = pad8(section);
        const uint64_t nq = P.state[4], qbytes = pad8(nq * 4);
        const uint64_t tid = uint64_t(block) * kThreads + threadIdx.x, stride = uint64_t(blocks) * kThreads;
        for (uint64_t b = section + tid; b < sec8; b += stride) P.wbuf[b] = 0;
        const uint8_t* qsrc[2] = {P.archive + P.state[2], P.archive + P.state[3]};
        for (int s = 0; s < 2; ++s) {
            uint32_t* dst = reinterpret_cast<uint32_t*>(P.wbuf + sec8 + s * qbytes);
            for (uint64_t w = tid; w < qbytes / 4; w += stride) dst[w] = wpw_load<uint32_t>(qsrc[s] + 4 * w, al);
        }
    }
};

struct WpwMoveOp {
    static constexpr int kThreads = 256, kMinBlocks = 0;
    struct Params {
        const uint64_t* layout;
        const uint64_t* state;
        const uint8_t* wbuf;
        uint8_t* archive;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t blocks) {
        if (!P.state[0]) return;
        const uint64_t words = P.state[5] / 8; // tail bytes are a multiple of 8
        uint8_t* dst = P.archive + P.layout[1];
        const uint64_t* src = reinterpret_cast<const uint64_t*>(P.wbuf);
        const bool al = (reinterpret_cast<uintptr_t>(P.archive) & 7u) == 0;
        for (uint64_t w = uint64_t(block) * kThreads + threadIdx.x; w < words; w += uint64_t(blocks) * kThreads) {
            if (al) reinterpret_cast<uint64_t*>(dst)[w] = src[w];
            else memcpy(dst + 8 * w, &src[w], 8);
        }
    }
};

// Decoder side: the correction of record i of a compact section (sec = the
// section's first byte, `bytes` its length, np records). Returns false for a
// malformed section (header, directory entry or span).
template <class T>
__device__ __forceinline__ bool wpw_correction(const uint8_t* sec, uint64_t bytes, uint32_t np, uint32_t i, T& corr) {
    const uint32_t groups = (np + 31) / 32;
    const uint64_t prefix = uint64_t(kWpwHeader) + uint64_t(kWpwEntry) * groups;
    uint32_t magic, hg;
    uint64_t pb, sb;
    memcpy(&magic, sec, 4);
    memcpy(&hg, sec + 4, 4);
    memcpy(&pb, sec + 8, 8);
    memcpy(&sb, sec + 16, 8);
    double step;
    memcpy(&step, &sb, 8);
    if (magic != kWpwMagic || hg != groups || prefix > bytes || pb != bytes - prefix || !(step > 0.0) ||
        !isfinite(step))
        return false;
    const uint32_t g = i / 32, lane = i % 32, count = min(32u, np - g * 32);
    uint32_t off, mask;
    memcpy(&off, sec + kWpwHeader + size_t(kWpwEntry) * g, 4);
    memcpy(&mask, sec + kWpwHeader + size_t(kWpwEntry) * g + 4, 4);
    if (count < 32 && (mask >> count)) return false;
    const uint32_t raw_start = (count + uint32_t(sizeof(T)) - 1) / uint32_t(sizeof(T)) * uint32_t(sizeof(T));
    const uint64_t gb = (off >> 31) ? uint64_t(count) * sizeof(T) : raw_start + uint64_t(__popc(mask)) * sizeof(T);
    const uint64_t start = off & 0x7fffffffu;
    if ((start & 7) || start > pb || gb > pb - start) return false;
    const uint8_t* p = sec + prefix + start;
    if (off >> 31) {
        memcpy(&corr, p + size_t(lane) * sizeof(T), sizeof(T));
    } else if ((mask >> lane) & 1u) {
        memcpy(&corr, p + raw_start + size_t(__popc(mask & ((1u << lane) - 1u))) * sizeof(T), sizeof(T));
    } else {
        corr = T(double(int8_t(p[lane])) * step);
    }
    return true;
}

} // namespace wb

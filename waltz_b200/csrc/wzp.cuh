// WZP magnitude/sign codec on the GPU.
//
// Stream format (byte-exact with cpu/src/wzp_cpu.cpp:769-867):
//   [u32 LE group offset x groups][u24 LE metadata x chunks][payload]
// 8192 magnitudes per chunk, 16 chunks per directory group. A nonzero chunk
// stores its magnitude bytes (bit-plane transpose + zero/repetition
// elimination, or verbatim when that is not at least 3 bytes smaller) and
// then its compacted sign bits, one per nonzero magnitude, LSB first.
//
// Encoder: one CTA per chunk, chunks taken from a ticket counter so that
// every chunk's predecessors are already resident; the payload offset is
// found by decoupled lookback over per-chunk states and the chunk writes
// straight into the archive. Every wait is bounded: a wait that hits its cap
// records ST_LOOKBACK_TIMEOUT and the kernel still terminates.
// Decoder: one CTA per chunk, fused with dequantisation and the inverse
// Morton scatter into the row-major coefficient array.
#pragma once
#include "common.cuh"
#include "quantize.cuh"
#include "scan.cuh"

namespace wb {

constexpr int kWzpThreads = 512;

__device__ __forceinline__ void store_u24(uint8_t* p, uint32_t v) {
    p[0] = uint8_t(v);
    p[1] = uint8_t(v >> 8);
    p[2] = uint8_t(v >> 16);
}
__device__ __forceinline__ uint32_t load_u24(const uint8_t* p) {
    return uint32_t(p[0]) | (uint32_t(p[1]) << 8) | (uint32_t(p[2]) << 16);
}
__device__ __forceinline__ uint32_t load_u32(const uint8_t* p) {
    return load_u24(p) | (uint32_t(p[3]) << 24);
}
__device__ __forceinline__ void store_u32(uint8_t* p, uint32_t v) {
    store_u24(p, v);
    p[3] = uint8_t(v >> 24);
}

// chunk lookback state: bits 62-63 flag, low 62 bits value
constexpr uint64_t kAggregate = 1ull << 62;
constexpr uint64_t kInclusive = 2ull << 62;
constexpr uint64_t kValueMask = (1ull << 62) - 1;

// Bytes of the plane / payload buffer: the 2 * 8192 plane bytes, which the
// zero and repetition elimination overwrite in place with at most
// 16384 + 2048 + 256 + 32 + 4 payload bytes, plus slack for word-wide copies.
constexpr uint32_t kEncBytes = 2 * kChunk + 2048 + 256 + 32 + 4 + 28;

// Bit planes in shared memory: the stream's natural layout puts plane p's
// u16 word b at p * blocks + b, so the 16 lanes that hold the 16 planes of one
// 32-sample group would all hit one bank. Both directions therefore keep the
// planes of a full chunk (512 blocks) at a padded pitch of kEncPitch u32
// words: lane p's word of group g lands in bank (4p + g) mod 32 (two lanes per
// bank instead of sixteen), and a thread's 32 consecutive natural bytes
// (8 words of one plane) stay 16-byte aligned and contiguous at natural word
// 8t plus 4 * (t / 32), so the zero elimination reads them, and the decoder's
// byte spreading writes them, in place. A partial chunk (a field's last)
// keeps the natural layout; the decoder repacks it to plane p at u32 word
// p * kPlanePitch + group by a conflict-free pass (consecutive threads on
// consecutive natural words).
constexpr uint32_t kPlanePitch = kChunk / 32 + 1; // u32 words per padded plane, partial chunks
constexpr uint32_t kEncPitch = kChunk / 32 + 4;   // u32 words per padded plane, full chunks
static_assert(16 * kEncPitch * 4 <= kEncBytes, "padded encoder planes fit the plane buffer");

// natural -> padded (dir = true) or padded -> natural, in place in `buf`
// (room for 16 * kPlanePitch words); the caller syncs before and after.
__device__ __forceinline__ void planes_repack(uint8_t* buf, uint32_t blocks, bool to_padded, int tid) {
    constexpr int PER = (16 * kChunk / 16 / 2 + kWzpThreads - 1) / kWzpThreads; // u32 words per thread
    uint32_t* w = reinterpret_cast<uint32_t*>(buf);
    if (blocks == 0) return; // no whole block: no planes (uniform across the block)
    if ((blocks & 1u) == 0) {
        const uint32_t per_plane = blocks / 2, words = 16 * per_plane;
        uint32_t v[PER];
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const uint32_t q = tid + k * kWzpThreads;
            const uint32_t p = q / per_plane, g = q - p * per_plane;
            if (q < words) v[k] = to_padded ? w[q] : w[p * kPlanePitch + g];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const uint32_t q = tid + k * kWzpThreads;
            const uint32_t p = q / per_plane, g = q - p * per_plane;
            if (q < words) (to_padded ? w[p * kPlanePitch + g] : w[q]) = v[k];
        }
    } else {
        // an odd number of 16-sample blocks (a field's last chunk): u16 steps
        uint16_t* h = reinterpret_cast<uint16_t*>(buf);
        const uint32_t halves = 16 * blocks;
        uint16_t v[2 * PER];
#pragma unroll
        for (int k = 0; k < 2 * PER; ++k) {
            const uint32_t q = tid + k * kWzpThreads;
            const uint32_t p = q / blocks, b = q - p * blocks;
            if (q < halves) v[k] = to_padded ? h[q] : h[2 * p * kPlanePitch + b];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 2 * PER; ++k) {
            const uint32_t q = tid + k * kWzpThreads;
            const uint32_t p = q / blocks, b = q - p * blocks;
            if (q < halves) (to_padded ? h[2 * p * kPlanePitch + b] : h[q]) = v[k];
        }
    }
}

struct WzpEncodeSmem {
    uint16_t m[kChunk + 8];            // magnitudes (+ slack for word-wide copies)
    union {
        uint8_t planes[kEncBytes];     // bit planes, then the eliminated payload in place
        uint8_t sneg[kChunk];          // negative-code flags while a source quantises
    };
    uint8_t lv[2048 + 256 + 32 + 4 + 4]; // nonzero bitmap and its reductions
    uint32_t sgn[kChunk / 32 + 1];     // compacted sign bits (+ slack)
    uint32_t gcount[kChunk / 32];      // nonzero magnitudes per 32-group
    uint32_t gsign[kChunk / 32];       // per 32-group: sign bits of its nonzero magnitudes, compacted
    uint32_t nsign[kChunk / 32];       // natural sign words of the chunk
    uint32_t bbase[32];                // row-major bases of the chunk's bricks (quantising source)
    uint32_t sel[16];                  // byte_perm selectors: compact the bytes of a 4-bit mask
    uint32_t tmp[40];
    uint32_t chunk, excl;
};

struct WzpEncodeArgs {
    uint32_t n;
    uint8_t* out;       // start of the WZP stream
    size_t capacity;    // bytes available from `out`
    uint32_t* ticket;   // zeroed before launch
    uint64_t* state;    // per chunk, zeroed before launch
    uint64_t* sizes;    // per chunk byte count (output)
    uint32_t* status;
    uint32_t spin_cap;  // lookback wait bound (polls of ~0.2 us)
    uint32_t skip_publish; // test hook: this chunk never publishes (0xffffffff = none)
};

// 32x32 bit transpose across a warp (five butterfly exchanges): on return
// lane i holds in bit j what lane j held in bit i. The half-word and byte
// exchanges are byte permutes; the nibble, pair and bit exchanges are shifts
// under the stage's mask.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, int lane) {
    uint32_t y = __shfl_xor_sync(0xffffffffu, x, 16);
    x = __byte_perm(x, y, (lane & 16) ? 0x3276u : 0x5410u);
    y = __shfl_xor_sync(0xffffffffu, x, 8);
    x = __byte_perm(x, y, (lane & 8) ? 0x3715u : 0x6240u);
#pragma unroll
    for (int j = 4; j >= 1; j >>= 1) {
        const uint32_t m = j == 4 ? 0x0f0f0f0fu : j == 2 ? 0x33333333u : 0x55555555u;
        y = __shfl_xor_sync(0xffffffffu, x, j);
        x = (lane & j) ? ((x & ~m) | ((y >> j) & m)) : ((x & m) | ((y << j) & ~m));
    }
    return x;
}

// 4-bit mask of the nonzero bytes of w (bit k = byte k).
__device__ __forceinline__ uint32_t nonzero_nibble(uint32_t w) { return (__vsetne4(w, 0u) * 0x01020408u) >> 24; }
// 4-bit mask of the bytes of w that differ from the byte before them
// (`prev` is the byte preceding w).
__device__ __forceinline__ uint32_t changed_nibble(uint32_t w, uint32_t prev) {
    return (__vsetne4(w, (w << 8) | (prev & 0xffu)) * 0x01020408u) >> 24;
}
// Appends the bytes of w selected by the 4-bit mask to dst + o; returns how many.
__device__ __forceinline__ uint32_t put_selected(uint8_t* dst, uint32_t o, uint32_t w, uint32_t mask,
                                                 const uint32_t* sel) {
    const uint32_t c = __popc(mask), cw = __byte_perm(w, 0u, sel[mask]);
    if (c > 0) dst[o] = uint8_t(cw);
    if (c > 1) dst[o + 1] = uint8_t(cw >> 8);
    if (c > 2) dst[o + 2] = uint8_t(cw >> 16);
    if (c > 3) dst[o + 3] = uint8_t(cw >> 24);
    return c;
}

// Copies len bytes from 4-byte aligned shared memory to any global address:
// aligned 32-bit stores for whole destination words, byte stores at the two
// ends. src must stay readable 4 bytes past len.
__device__ __forceinline__ void copy_to_global(uint8_t* dst, const uint8_t* src, uint32_t len, int tid, int nthreads) {
    const uint32_t mis = uint32_t(reinterpret_cast<uintptr_t>(dst) & 3u);
    uint32_t* base = reinterpret_cast<uint32_t*>(dst - mis);
    const uint32_t* sw = reinterpret_cast<const uint32_t*>(src);
    const uint32_t total = mis + len, words = (total + 3) / 4;
    for (uint32_t j = tid; j < words; j += nthreads) {
        const int64_t r0 = int64_t(4 * j) - mis; // source offset of the word's first byte
        if (r0 >= 0 && r0 + 4 <= int64_t(len)) {
            base[j] = mis ? __funnelshift_r(sw[j - 1], sw[j], 8 * (4 - mis)) : sw[j];
        } else {
            for (int t = 0; t < 4; ++t) {
                const int64_t r = r0 + t;
                if (r >= 0 && r < int64_t(len)) dst[r] = src[r];
            }
        }
    }
}

// Four consecutive samples through 16-byte accesses (p 16-byte aligned).
__device__ __forceinline__ void load4(const float* p, float (&v)[4]) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
}
__device__ __forceinline__ void load4(const double* p, double (&v)[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
}
__device__ __forceinline__ void store4(float* p, const float (&v)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void store4(double* p, const double (&v)[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}


// ---------------------------------------------------------------------------
// 16-sample blocks. The stream's bit planes are per 16 consecutive Morton
// slots (a "block"): plane p of block b is a u16 whose bit 15-j is bit 15-p
// of the block's magnitude j. In a whole 16 x 16 x bz brick (bz a power of
// two) a block is an aligned 4 x 2 x 2 box when bz = 16 and an aligned
// 4 x 4 x 1 box when bz <= 8 (the recursive octant order of morton_rank), so
// one thread can own a block: load it as four 16-byte rows, hold its 16
// magnitudes in registers and move between magnitudes and planes with one
// 16 x 16 bit transpose.

// 16 x 16 bit transpose, rows packed in pairs (w[i] = row 2i | row 2i+1 << 16,
// bit 15 of a row = column 0): on return row p holds column p. Its own
// inverse. Four block-swap stages (Hacker's Delight 7-3); the stages of
// width 8, 4 and 2 act on both halves of a word pair at once, the stage of
// width 1 inside each word.
__device__ __forceinline__ void bit_transpose16(uint32_t (&w)[8]) {
#pragma unroll
    for (int j = 8; j >= 2; j >>= 1) {
        const uint32_t m = j == 8 ? 0x00ff00ffu : j == 4 ? 0x0f0f0f0fu : 0x33333333u;
        const int h = j / 2; // word distance of rows k and k + j
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            if (i & h) continue;
            const uint32_t t = (w[i] ^ (w[i + h] >> j)) & m;
            w[i] ^= t;
            w[i + h] ^= t << j;
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t t = (w[i] ^ (w[i] >> 17)) & 0x5555u;
        w[i] ^= t ^ (t << 17);
    }
}

// Element layout of a block: row r (0..3) of the block's four 16-byte rows
// holds magnitudes e0(r), e0(r)+1 (x = 0, 1) and e0(r)+d, e0(r)+d+1 (x = 2, 3);
// its offset from the block origin is dz * plane + dy * nx.
// Tall: bz = 16, 4 x 2 x 2 (rows dy + 2 dz); else 4 x 4 x 1 (rows dy). A
// compile-time shape keeps the packed magnitudes in registers.
template <bool Tall> struct BlockShape {
    static __device__ __forceinline__ constexpr int e0(int r) { return Tall ? 2 * r : ((r & 1) << 1) | ((r >> 1) << 3); }
    static constexpr int d = Tall ? 8 : 4;
    static __device__ __forceinline__ uint32_t row_offset(int r, uint32_t nx, uint32_t plane) {
        return Tall ? uint32_t(r >> 1) * plane + uint32_t(r & 1) * nx : uint32_t(r) * nx;
    }
};

// Origin (x, y, z) inside a 16 x 16 x 2^zb brick of the block holding Morton
// ranks 16k .. 16k+15: the rank's bits come in levels from the bottom, 4 - zb
// levels of (x, y) bits, then zb levels of (x, y, z) bits; the block index
// drops the lowest four bits.
__device__ __forceinline__ void block_origin(uint32_t k, uint32_t zb, uint32_t& x, uint32_t& y, uint32_t& z) {
    uint32_t r = k << 4, bit = 0;
    x = y = z = 0;
    uint32_t zl = 0;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        const bool withz = uint32_t(l) >= 4 - zb;
        x |= ((r >> bit) & 1u) << l;
        y |= ((r >> (bit + 1)) & 1u) << l;
        bit += 2;
        if (withz) {
            z |= ((r >> bit) & 1u) << zl;
            ++zl;
            ++bit;
        }
    }
}

// Bits of x selected by mask, packed towards bit 0 in order (16-bit
// compress, Hacker's Delight 7-4).
__device__ __forceinline__ uint32_t compress16(uint32_t x, uint32_t m) {
    x &= m;
    uint32_t mk = (~m << 1) & 0xffffu;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        uint32_t mp = mk ^ (mk << 1);
        mp ^= mp << 2;
        mp ^= mp << 4;
        mp ^= mp << 8;
        mp &= 0xffffu;
        const uint32_t mv = mp & m;
        m = (m ^ mv) | (mv >> (1 << i));
        const uint32_t t = x & mv;
        x = (x ^ t) | (t >> (1 << i));
        mk &= ~mp;
    }
    return x;
}

// The low popc(m) bits of x spread to the set positions of m, in order
// (16-bit expand, the inverse of compress16).
__device__ __forceinline__ uint32_t expand16(uint32_t x, uint32_t m) {
    uint32_t a[4];
    const uint32_t m0 = m;
    uint32_t mk = (~m << 1) & 0xffffu;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        uint32_t mp = mk ^ (mk << 1);
        mp ^= mp << 2;
        mp ^= mp << 4;
        mp ^= mp << 8;
        mp &= 0xffffu;
        const uint32_t mv = mp & m;
        a[i] = mv;
        m = (m ^ mv) | (mv >> (1 << i));
        mk &= ~mp;
    }
#pragma unroll
    for (int i = 3; i >= 0; --i) {
        const uint32_t mv = a[i], t = x << (1 << i);
        x = (x & ~mv) | (t & mv);
    }
    return x & m0;
}

// Magnitude sources of the encoder. Each fills S.m[0, 8192) (zeros past
// the chunk's end) and S.nsign (the chunk's natural sign words).

// Morton-packed u16 magnitudes and a natural sign bitmap in global memory.
struct MagArrays {
    static constexpr bool kBlockPlanes = false;
    const uint16_t* mag;
    const uint32_t* sign;
    __device__ __forceinline__ void load(WzpEncodeSmem& S, uint32_t first, uint32_t count, int tid) const {
        if (count == kChunk) {
            const uint4* src = reinterpret_cast<const uint4*>(mag + first);
            for (int i = tid; i < int(kChunk / 8); i += kWzpThreads) reinterpret_cast<uint4*>(S.m)[i] = src[i];
        } else {
            for (int i = tid; i < int(kChunk); i += kWzpThreads) S.m[i] = i < int(count) ? mag[first + i] : 0;
        }
        for (uint32_t g = tid; g < kChunk / 32; g += kWzpThreads)
            S.nsign[g] = g * 32 < count ? sign[(first >> 5) + g] : 0u;
    }
};

// The coefficients themselves, quantised by the encoder (quantize_kernel
// fused in): the chunk is a run of whole 16 x 16 x bz bricks (2^lb samples
// each, the field made of whole bricks only); every brick is read and
// rewritten (dequantised) row by row, its magnitudes and negative flags placed
// at their Morton ranks, and q-outliers recorded as in quantize_kernel.
template <class T> struct QuantBricks {
    static constexpr bool kBlockPlanes = true;
    T* coeff;
    uint32_t nx, ny, bz, lb;
    const uint16_t* rank; // full-brick slot: brick-local row-major index -> rank
    T q, inv;
    uint32_t* qbits;
    uint32_t* qval;
    uint32_t* status;

    // Quantises block t of the chunk starting at `first` (its dequantised
    // values written back): packed magnitudes w (pairs of Morton slots),
    // nonzero and negative masks (bit j = slot j of the block).
    template <bool Tall>
    __device__ __forceinline__ void quantise_block(uint32_t first, uint32_t t, uint32_t (&w)[8], uint32_t& zm,
                                                   uint32_t& nm) const {
        using Sh = BlockShape<Tall>;
        const uint32_t plane = nx * ny;
        const uint32_t b = (first >> lb) + ((t << 4) >> lb), k = t & ((1u << (lb - 4)) - 1u);
        const uint32_t nbx = nx / 16, nby = ny / 16;
        const uint32_t bxi = b % nbx, tb = b / nbx, byi = tb % nby, slab = tb / nby;
        uint32_t lx, ly, lz;
        block_origin(k, lb - 8, lx, ly, lz);
        const uint32_t at0 = (slab * bz + lz) * plane + (byi * 16 + ly) * nx + bxi * 16 + lx;
        uint32_t bad = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t at = at0 + Sh::row_offset(r, nx, plane);
            constexpr int dd = Sh::d;
            const int e0 = Sh::e0(r), e1 = e0 + dd;
            T v[4];
            load4(coeff + at, v);
            uint32_t mg[4];
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                int32_t m;
                bool neg;
                v[x] = quantize_one<T>(v[x], inv, q, m, neg, bad);
                const int e = (x < 2 ? e0 : e1) + (x & 1);
                mg[x] = uint32_t(m > 65535 ? 65535 : m);
                zm |= uint32_t(m != 0) << e;
                nm |= uint32_t(neg && m) << e;
                if (m > 65535) {
                    atomicOr(&qbits[(at + x) >> 5], 1u << ((at + x) & 31));
                    qval[at + x] = uint32_t(m);
                }
            }
            store4(coeff + at, v);
            // e0 and e1 are even: each pair fills one packed word
            w[e0 >> 1] = mg[0] | (mg[1] << 16);
            w[e1 >> 1] = mg[2] | (mg[3] << 16);
        }
        if (bad) atomicOr(status, ST_QUANT_DOMAIN);
    }

    // One thread per 16-sample block (thread t: Morton slots 16t .. 16t+15 of
    // the chunk): quantise the block's four rows (dequantised values written
    // back), then write its magnitudes to S.m, its 16 bit planes to S.planes
    // (full chunks at the padded pitch, a partial chunk in the natural
    // layout), and per 32-group the nonzero count and the compacted sign bits
    // of its nonzero magnitudes (the even thread of each pair). Blocks past
    // the chunk's end are zero.
    __device__ __forceinline__ void block_planes(WzpEncodeSmem& S, uint32_t first, uint32_t count, int tid) const {
        const uint32_t blocks = count >> 4, t = uint32_t(tid);
        uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        uint32_t zm = 0, nm = 0;
        if (t < blocks) {
            if (bz == 16) quantise_block<true>(first, t, w, zm, nm);
            else quantise_block<false>(first, t, w, zm, nm);
        }
        uint4* dm = reinterpret_cast<uint4*>(S.m + 16 * t);

        dm[0] = make_uint4(w[0], w[1], w[2], w[3]);
        dm[1] = make_uint4(w[4], w[5], w[6], w[7]);
        // group statistics: this block's count and compacted signs, merged
        // with the odd neighbour's by the even thread of the pair
        const uint32_t cnt = __popc(zm), cs = compress16(nm, zm);
        const uint32_t cnt1 = __shfl_xor_sync(0xffffffffu, cnt, 1), cs1 = __shfl_xor_sync(0xffffffffu, cs, 1);
        if (!(t & 1) && t < kChunk / 16) {
            S.gcount[t >> 1] = cnt + cnt1;
            S.gsign[t >> 1] = cs | (cs1 << cnt);
        }
        if (t < blocks) {
            if ((w[0] | w[1] | w[2] | w[3] | w[4] | w[5] | w[6] | w[7]) != 0) bit_transpose16(w);
            uint16_t* pl = reinterpret_cast<uint16_t*>(S.planes);
            const bool full = blocks == kChunk / 16;
            const uint32_t stride = full ? 2 * kEncPitch : blocks;
#pragma unroll
            for (int p = 0; p < 16; ++p) pl[p * stride + t] = uint16_t(p & 1 ? w[p >> 1] >> 16 : w[p >> 1]);
        }
    }
    __device__ __forceinline__ void load(WzpEncodeSmem& S, uint32_t first, uint32_t count, int tid) const {
        const uint32_t bsz = 1u << lb, nb = count >> lb, plane = nx * ny;
        if (tid < int(nb)) {
            const uint32_t b = (first >> lb) + tid, nbx = nx / 16, nby = ny / 16;
            const uint32_t bxi = b % nbx, t = b / nbx, byi = t % nby, slab = t / nby;
            S.bbase[tid] = slab * bz * plane + byi * 16 * nx + bxi * 16;
        }
        for (uint32_t e = nb * bsz + tid; e < kChunk; e += kWzpThreads) {
            S.m[e] = 0;
            S.sneg[e] = 0;
        }
        __syncthreads();
        uint32_t bad = 0;
        auto place = [&](uint32_t at, uint32_t slot, int32_t m, bool neg) {
            S.m[slot] = uint16_t(m > 65535 ? 65535 : m);
            S.sneg[slot] = neg && m;
            if (m > 65535) {
                atomicOr(&qbits[at >> 5], 1u << (at & 31));
                qval[at] = uint32_t(m);
            }
        };
        if (((reinterpret_cast<uintptr_t>(coeff) & 15u) | (reinterpret_cast<uintptr_t>(rank) & 7u)) == 0) {
            // four consecutive samples of a brick row per step (16 | nx, so a
            // row's quarter is 16-byte aligned): one vector load and store of
            // the coefficients, one 8-byte load of their four ranks
            for (uint32_t e = 4 * uint32_t(tid); e < nb * bsz; e += 4 * kWzpThreads) {
                const uint32_t j = e >> lb, i = e & (bsz - 1u);
                const uint32_t at = S.bbase[j] + (i >> 8) * plane + ((i >> 4) & 15u) * nx + (i & 15u);
                T v[4];
                load4(coeff + at, v);
                const uint2 rk = *reinterpret_cast<const uint2*>(rank + i);
                const uint32_t base = j << lb;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    int32_t m;
                    bool neg;
                    v[k] = quantize_one<T>(v[k], inv, q, m, neg, bad);
                    const uint32_t r = ((k < 2 ? rk.x : rk.y) >> (16 * (k & 1))) & 0xffffu;
                    place(at + k, base + r, m, neg);
                }
                store4(coeff + at, v);
            }
        } else {
            for (uint32_t e = tid; e < nb * bsz; e += kWzpThreads) {
                const uint32_t j = e >> lb, i = e & (bsz - 1u);
                const uint32_t at = S.bbase[j] + (i >> 8) * plane + ((i >> 4) & 15u) * nx + (i & 15u);
                int32_t m;
                bool neg;
                coeff[at] = quantize_one<T>(coeff[at], inv, q, m, neg, bad);
                place(at, (j << lb) + rank[i], m, neg);
            }
        }
        if (bad) atomicOr(status, ST_QUANT_DOMAIN);
        __syncthreads();
        for (uint32_t g = tid; g < kChunk / 32; g += kWzpThreads) {
            const uint32_t* f = reinterpret_cast<const uint32_t*>(S.sneg + 32 * g);
            uint32_t bits = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) bits |= (((f[k] & 0x01010101u) * 0x01020408u) >> 24) << (4 * k);
            S.nsign[g] = bits;
        }
    }
};

template <class Src> struct WzpEncodeOp {
    static constexpr int kThreads = kWzpThreads, kMinBlocks = 4; // 32 registers: four CTAs per SM
    struct Params {
        WzpEncodeArgs A;
        Src src;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t, uint32_t);
};

template <class Src>
__device__ __forceinline__ void WzpEncodeOp<Src>::run(const Params P, uint32_t, uint32_t) {
    const WzpEncodeArgs& A = P.A;
    const Src& src = P.src;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WzpEncodeSmem& S = *reinterpret_cast<WzpEncodeSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kWzpThreads / 32;
    const uint32_t chunks = wzp_chunks(A.n), groups = wzp_groups(A.n);
    if (tid == 0) S.chunk = atomicAdd(A.ticket, 1u);
    if (tid < 16) {
        uint32_t sel = 0x4444u, k = 0;
        for (int b = 0; b < 4; ++b)
            if ((tid >> b) & 1) {
                sel = (sel & ~(0xfu << (4 * k))) | (uint32_t(b) << (4 * k));
                ++k;
            }
        S.sel[tid] = sel;
    }
    __syncthreads();
    const uint32_t c = S.chunk;
    if (c >= chunks) return;
    const uint32_t first = c * kChunk;
    const uint32_t count = min(kChunk, A.n - first);
    const uint32_t blocks = count / 16;

    if constexpr (Src::kBlockPlanes) {
        // ---- one thread per 16-sample block: magnitudes, bit planes and
        // group statistics in one pass
        src.block_planes(S, first, count, tid);
        for (int i = tid; i < int(kChunk / 32) + 1; i += kWzpThreads) S.sgn[i] = 0;
        __syncthreads();
    } else {
    // ---- magnitudes and natural sign words of the chunk
    src.load(S, first, count, tid);
    for (int i = tid; i < int(kChunk / 32) + 1; i += kWzpThreads) S.sgn[i] = 0;
    __syncthreads();

    // ---- per 32-group nonzero counts and sign bits, and the bit planes, two
    // groups per warp step: one 32x32 transpose turns the pair's 16-bit
    // magnitudes (group g in the high half of each lane's word, g+1 in the
    // low half) into plane p of g in lane p and of g+1 in lane 16+p
    const uint32_t in_planes = blocks * 16;
    for (int k = warp; k < int(kChunk / 64); k += NW) {
        const int g0 = 2 * k, e0 = g0 * 32 + lane;
        const uint32_t v = S.m[e0], u = S.m[e0 + 32];
        const uint32_t nz0 = __ballot_sync(0xffffffffu, v != 0), nz1 = __ballot_sync(0xffffffffu, u != 0);
        // each group's nonzero magnitudes' sign bits packed in order (merged
        // at the group's rank below)
        const uint32_t below = (1u << lane) - 1u;
        const uint32_t s0 = __reduce_or_sync(
            0xffffffffu, (v != 0 && ((S.nsign[g0] >> lane) & 1u)) ? 1u << __popc(nz0 & below) : 0u);
        const uint32_t s1 = __reduce_or_sync(
            0xffffffffu, (u != 0 && ((S.nsign[g0 + 1] >> lane) & 1u)) ? 1u << __popc(nz1 & below) : 0u);
        if (lane < 2) {
            S.gcount[g0 + lane] = __popc(lane ? nz1 : nz0);
            S.gsign[g0 + lane] = lane ? s1 : s0;
        }
        if (uint32_t(g0 * 32) < in_planes) {
            const uint32_t va = uint32_t(e0) < in_planes ? v : 0u, ua = uint32_t(e0 + 32) < in_planes ? u : 0u;
            const int top = 32 - __clz(__reduce_or_sync(0xffffffffu, va | ua)); // planes 16-top .. 15 may be set
            uint32_t mine = 0;
            if (top > 2) {
                mine = __brev(warp_transpose32(__brev((va << 16) | ua), lane));
            } else {
                // one or two planes: a ballot each (bit 31-e = magnitude e's bit)
#pragma unroll
                for (int p = 14; p < 16; ++p) {
                    if (15 - p < top) {
                        const uint32_t r0 = __brev(__ballot_sync(0xffffffffu, (va >> (15 - p)) & 1u));
                        const uint32_t r1 = __brev(__ballot_sync(0xffffffffu, (ua >> (15 - p)) & 1u));
                        if (lane == p) mine = r0;
                        if (lane == 16 + p) mine = r1;
                    }
                }
            }
            // lane l holds plane l % 16 of group g0 + l / 16 (blocks 2g, 2g+1 in
            // its high and low halves); full chunks: one word at the padded
            // pitch; a partial chunk keeps the natural layout, u16 words at
            // p * blocks + b
            const uint32_t g = uint32_t(g0) + (uint32_t(lane) >> 4), pl_ = uint32_t(lane) & 15u;
            if (blocks == kChunk / 16) {
                reinterpret_cast<uint32_t*>(S.planes)[pl_ * kEncPitch + g] = __funnelshift_l(mine, mine, 16);
            } else {
                uint16_t* pl = reinterpret_cast<uint16_t*>(S.planes);
                if (2 * g < blocks) pl[pl_ * blocks + 2 * g] = uint16_t(mine >> 16);
                if (2 * g + 1 < blocks) pl[pl_ * blocks + 2 * g + 1] = uint16_t(mine & 0xffffu);
            }
        }
    }
    // verbatim tail after the planes
    for (uint32_t i = blocks * 16 + tid; i < count; i += kWzpThreads)
        reinterpret_cast<uint16_t*>(S.planes)[i] = S.m[i];
    __syncthreads();
    }

    // ---- signs: each group's packed sign bits go to its rank offset (at most
    // two words)
    uint32_t nnz;
    {
        const uint32_t gc = tid < int(kChunk / 32) ? S.gcount[tid] : 0;
        const uint32_t r = block_excl_scan<kWzpThreads>(gc, S.tmp, nnz);
        if (tid < int(kChunk / 32)) {
            const uint32_t packed = S.gsign[tid];
            if (packed) {
                const uint32_t sh = r & 31;
                atomicOr(&S.sgn[r >> 5], packed << sh);
                if (sh && (packed >> (32 - sh))) atomicOr(&S.sgn[(r >> 5) + 1], packed >> (32 - sh));
            }
        }
    }
    __syncthreads();

    // ---- zero elimination of the plane bytes: thread t owns bytes 32t..32t+31
    const uint32_t raw_bytes = 2 * count;
    uint32_t nzb, c1 = 0, c2 = 0, c3 = 0;
    {
        const uint32_t b0 = tid * 32;
        uint32_t w[8];
        const uint32_t pad = blocks == kChunk / 16 ? 4 * (kEncPitch - kChunk / 32) * (uint32_t(tid) >> 5) : 0u;
        const uint4* q = reinterpret_cast<const uint4*>(S.planes + b0 + pad);
        const uint4 q0 = q[0], q1 = q[1];
        w[0] = q0.x; w[1] = q0.y; w[2] = q0.z; w[3] = q0.w;
        w[4] = q1.x; w[5] = q1.y; w[6] = q1.z; w[7] = q1.w;
        uint32_t bits = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) bits |= nonzero_nibble(w[k]) << (4 * k);
        if (b0 + 32 > raw_bytes) bits &= b0 >= raw_bytes ? 0u : ((1u << (raw_bytes - b0)) - 1u);
        uint32_t o = block_excl_scan<kWzpThreads>(__popc(bits), S.tmp, nzb);
#pragma unroll
        for (int k = 0; k < 8; ++k) o += put_selected(S.planes, o, w[k], (bits >> (4 * k)) & 15u, S.sel);
        reinterpret_cast<uint32_t*>(S.lv)[tid] = bits; // bitmap bytes 4t..4t+3
    }
    __syncthreads();
    // ---- repetition elimination: 2048 -> 256 -> 32 -> 4 bytes; a byte is
    // kept iff it differs from the byte before it (before the first: 0)
    {
        // level 1: thread t < 256 owns bitmap bytes 8t..8t+7
        uint32_t flags = 0, w0 = 0, w1 = 0;
        if (tid < 256) {
            const uint32_t* lw = reinterpret_cast<const uint32_t*>(S.lv);
            w0 = lw[2 * tid];
            w1 = lw[2 * tid + 1];
            const uint32_t prev = tid ? (lw[2 * tid - 1] >> 24) : 0u;
            flags = changed_nibble(w0, prev) | (changed_nibble(w1, w0 >> 24) << 4);
        }
        uint32_t o = nzb + block_excl_scan<kWzpThreads>(__popc(flags), S.tmp, c1);
        if (tid < 256) {
            o += put_selected(S.planes, o, w0, flags & 15u, S.sel);
            put_selected(S.planes, o, w1, flags >> 4, S.sel);
            S.lv[2048 + tid] = uint8_t(flags);
        }
        __syncthreads();
        // levels 2 and 3 by warp 0
        if (warp == 0) {
            const uint32_t* l1 = reinterpret_cast<const uint32_t*>(S.lv + 2048);
            const uint32_t v0 = l1[2 * lane], v1 = l1[2 * lane + 1];
            const uint32_t pv = lane ? (l1[2 * lane - 1] >> 24) : 0u;
            const uint32_t f2 = changed_nibble(v0, pv) | (changed_nibble(v1, v0 >> 24) << 4);
            const uint32_t n2 = __popc(f2);
            const uint32_t inc = warp_incl_scan(n2);
            c2 = __shfl_sync(0xffffffffu, inc, 31);
            uint32_t o2 = nzb + c1 + inc - n2;
            o2 += put_selected(S.planes, o2, v0, f2 & 15u, S.sel);
            put_selected(S.planes, o2, v1, f2 >> 4, S.sel);
            S.lv[2048 + 256 + lane] = uint8_t(f2);
            __syncwarp();
            const uint32_t* l2 = reinterpret_cast<const uint32_t*>(S.lv + 2048 + 256);
            uint32_t f3 = 0, u0 = 0, u1 = 0;
            if (lane < 4) {
                u0 = l2[2 * lane];
                u1 = l2[2 * lane + 1];
                const uint32_t pu = lane ? (l2[2 * lane - 1] >> 24) : 0u;
                f3 = changed_nibble(u0, pu) | (changed_nibble(u1, u0 >> 24) << 4);
            }
            const uint32_t n3 = __popc(f3);
            const uint32_t inc3 = warp_incl_scan(n3);
            c3 = __shfl_sync(0xffffffffu, inc3, 31);
            if (lane < 4) {
                uint32_t o3 = nzb + c1 + c2 + inc3 - n3;
                o3 += put_selected(S.planes, o3, u0, f3 & 15u, S.sel);
                put_selected(S.planes, o3, u1, f3 >> 4, S.sel);
                S.planes[nzb + c1 + c2 + c3 + lane] = uint8_t(f3);
            }
            if (lane == 0) {
                S.tmp[34] = c2;
                S.tmp[35] = c3;
            }
        }
        __syncthreads();
        c2 = S.tmp[34];
        c3 = S.tmp[35];
    }
    const uint32_t rze = nzb ? nzb + c1 + c2 + c3 + 4 : 0;
    const bool raw = rze + 2 >= raw_bytes;
    const uint32_t mbytes = raw ? raw_bytes : rze;
    const uint32_t sbytes = (nnz + 7) / 8;
    const uint64_t chunk_bytes = nnz ? uint64_t(mbytes) + sbytes : 0;

    // ---- decoupled lookback by warp 0: 32 predecessor states per step; the
    // closest inclusive prefix ends the walk. Every wait is bounded.
    if (warp == 0) {
        const bool publish = c != A.skip_publish;
        if (lane == 0 && publish)
            atomicExch(reinterpret_cast<unsigned long long*>(&A.state[c]),
                       (unsigned long long)((c == 0 ? kInclusive : kAggregate) | chunk_bytes));
        uint64_t excl = 0;
        bool timed_out = false;
        int64_t top = int64_t(c) - 1; // predecessor examined by lane 0
        uint32_t spins = 0;
        while (top >= 0) {
            const int64_t j = top - lane;
            const uint64_t st = j >= 0 ? *reinterpret_cast<volatile uint64_t*>(&A.state[j]) : uint64_t(2ull << 62);
            const uint32_t pub = __ballot_sync(0xffffffffu, (st >> 62) != 0);
            const uint32_t inc = __ballot_sync(0xffffffffu, (st >> 62) == 2);
            const int last = inc ? __ffs(inc) - 1 : 31; // lanes 0..last are needed
            const uint32_t need = last == 31 ? 0xffffffffu : ((2u << last) - 1u);
            if ((pub & need) != need) {
                if (++spins >= A.spin_cap) {
                    timed_out = true;
                    break;
                }
                __nanosleep(200);
                continue;
            }
            uint64_t v = lane <= last ? (st & kValueMask) : 0;
#pragma unroll
            for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
            excl += v;
            if (inc) break;
            top -= 32;
        }
        if (lane == 0) {
            if (timed_out) atomicOr(A.status, ST_LOOKBACK_TIMEOUT);
            if (c > 0 && publish)
                atomicExch(reinterpret_cast<unsigned long long*>(&A.state[c]),
                           (unsigned long long)(kInclusive | (excl + chunk_bytes)));
            A.sizes[c] = chunk_bytes;
            S.excl = uint32_t(excl);
            const size_t header = size_t(groups) * 4 + size_t(chunks) * 3;
            if (header + excl + chunk_bytes > A.capacity || excl + chunk_bytes > 0xffffffffull) {
                atomicOr(A.status, ST_CAPACITY);
                S.excl = 0xffffffffu;
            }
            const uint32_t meta = nnz ? ((raw ? kRawCode : mbytes) | ((sbytes == 1024 ? 0u : sbytes) << 14)) : 0u;
            store_u24(A.out + size_t(groups) * 4 + size_t(c) * 3, meta);
        }
    }
    __syncthreads();
    if (!nnz || S.excl == 0xffffffffu) return;
    // ---- payload: magnitude bytes (eliminated, or the raw magnitudes), then
    // the sign bytes, each copied with word-wide stores
    uint8_t* dst = A.out + size_t(groups) * 4 + size_t(chunks) * 3 + S.excl;
    copy_to_global(dst, raw ? reinterpret_cast<const uint8_t*>(S.m) : S.planes, mbytes, tid, kWzpThreads);
    copy_to_global(dst + mbytes, reinterpret_cast<const uint8_t*>(S.sgn), sbytes, tid, kWzpThreads);
}

// Group directory: payload offset of the first byte of every nonempty group.
struct WzpDirectoryOp {
    static constexpr int kThreads = 256, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        uint8_t* out;
        uint32_t n;
        const uint64_t *state, *sizes;
        uint64_t* total;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t);
};

__device__ __forceinline__ void WzpDirectoryOp::run(const Params P, uint32_t block, uint32_t) {
    uint8_t* const out = P.out;
    const uint32_t n = P.n;
    const uint64_t *state = P.state, *sizes = P.sizes;
    uint64_t* const total = P.total;
    const uint32_t chunks = wzp_chunks(n), groups = wzp_groups(n);
    const uint32_t g = block * kThreads + threadIdx.x;
    if (g >= groups) return;
    const uint32_t f = g * kGroup, l = min(f + kGroup, chunks) - 1;
    const uint64_t start = (state[f] & kValueMask) - sizes[f];
    const uint64_t end = state[l] & kValueMask;
    store_u32(out + size_t(g) * 4, end > start ? uint32_t(start) : 0u);
    if (g == groups - 1) *total = size_t(groups) * 4 + size_t(chunks) * 3 + end;
}

// ------------------------------------------------------------------ decode

// Brick geometry of the Morton-packed stream (bricks of 16 x 16 x bz, raster
// order z, y, x; edge bricks shrink): packed index -> row-major index.
struct BrickMap {
    uint32_t nx, ny, nz, bz;
    const uint16_t* local; // 8 slots x 256*bz: rank -> packed brick-local (x | y << 4 | z << 8)
    const uint16_t* rank;  // 8 slots x 256*bz: brick-local row-major index -> rank (slot 0: whole
                           // bricks), or null (the decoder then scatters through `local`)
    // Fast map: every brick whole (16 | nx, 16 | ny, bz | nz) and 256*bz a power
    // of two (lb = its log2), so a chunk is a run of whole bricks.
    bool fast;
    uint32_t lb;
    __device__ __forceinline__ uint32_t brick_base(uint32_t b) const {
        const uint32_t nbx = nx / 16, nby = ny / 16;
        const uint32_t bxi = b % nbx, t = b / nbx, byi = t % nby, slab = t / nby;
        return slab * bz * (nx * ny) + byi * 16 * nx + bxi * 16;
    }
    __device__ __forceinline__ uint32_t in_full_brick(uint32_t base, uint32_t rk) const {
        const uint32_t loc = __ldg(local + rk);
        return base + (loc >> 8) * (nx * ny) + ((loc >> 4) & 15u) * nx + (loc & 15u);
    }
    // Every index fits 32 bits: archives hold at most 2^32 - 1 sample bytes.
    __device__ __forceinline__ uint32_t rowmajor(uint32_t k) const {
        const uint32_t plane = nx * ny;
        const uint32_t slab_sz = plane * bz;
        const uint32_t slab = k / slab_sz;
        uint32_t r = k - slab * slab_sz;
        const uint32_t ez = min(bz, nz - slab * bz);
        const uint32_t row_sz = 16 * nx * ez;
        const uint32_t row = r / row_sz;
        r -= row * row_sz;
        const uint32_t ey = min(16u, ny - row * 16);
        const uint32_t brick_sz = 16 * ey * ez;
        const uint32_t bxi = r / brick_sz;
        const uint32_t rk = r - bxi * brick_sz;
        const uint32_t ex = min(16u, nx - bxi * 16);
        const uint32_t slot = (ex != 16) | ((ey != 16) << 1) | ((ez != bz) << 2);
        const uint32_t loc = local[slot * 256 * bz + rk];
        const uint32_t lx = loc & 15, ly = (loc >> 4) & 15, lz = loc >> 8;
        return (slab * bz + lz) * plane + (row * 16 + ly) * nx + bxi * 16 + lx;
    }
};

// Dequantises block t of the chunk starting at `first` (packed magnitudes w,
// negative mask nm) into the row-major coefficients as four 16-byte rows.
template <class T, bool Tall>
__device__ __forceinline__ void store_block(const BrickMap& map, T* coeff, uint32_t first, uint32_t t,
                                            const uint32_t (&w)[8], uint32_t nm, T q) {
    using Sh = BlockShape<Tall>;
    const uint32_t plane = map.nx * map.ny;
    uint32_t lx, ly, lz;
    block_origin(t & ((1u << (map.lb - 4)) - 1u), map.lb - 8, lx, ly, lz);
    const uint32_t b = (first >> map.lb) + ((t << 4) >> map.lb);
    const uint32_t at0 = map.brick_base(b) + lz * plane + ly * map.nx + lx;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        constexpr int dd = Sh::d;
        const int e0 = Sh::e0(r), e1 = e0 + dd;
        const uint32_t pa = w[e0 >> 1], pb = w[e1 >> 1];
        const uint32_t mg[4] = {pa & 0xffffu, pa >> 16, pb & 0xffffu, pb >> 16};
        T v4[4];
#pragma unroll
        for (int x = 0; x < 4; ++x) {
            const int e = (x < 2 ? e0 : e1) + (x & 1);
            const T mag = Lift<T>::mul(T(mg[x]), q);
            v4[x] = ((nm >> e) & 1u) ? -mag : mag;
        }
        store4(coeff + at0 + Sh::row_offset(r, map.nx, plane), v4);
    }
}

struct WzpDecodeSmem {
    uint32_t bbase[32];                // row-major base of each whole brick of the chunk (fast map)
    uint16_t m[kChunk + 16];           // staged magnitude bytes, then the decoded magnitudes
    uint8_t sb[1024 + 32];             // staged sign bytes
    uint32_t xsel[16];                 // byte_perm selectors: spread 4-bit-mask bytes into place
    // full chunks: planes at pitch kEncPitch; a partial chunk: natural, then
    // repacked to pitch kPlanePitch
    uint8_t planes[16 * (kEncPitch > kPlanePitch ? kEncPitch : kPlanePitch) * 4];
    uint8_t lv[2048 + 256 + 32 + 4];
    uint32_t gprefix[kChunk / 32];
    uint32_t gmask[kChunk / 32];       // nonzero magnitudes of each 32-group
    uint32_t tmp[40];
    uint32_t off, mbytes, sbytes, raw, bad;
};

struct WzpChunkInfo {
    uint32_t mbytes, sbytes;
    bool raw, ok;
};
__device__ __forceinline__ WzpChunkInfo wzp_meta(uint32_t meta, uint32_t count) {
    WzpChunkInfo r{0, 0, false, true};
    const uint32_t code = meta & kRawCode, scode = meta >> 14;
    if (!code) {
        r.ok = scode == 0;
        return r;
    }
    r.raw = code == kRawCode;
    if (!r.raw && (code < 4 || code + 2 >= 2 * count)) r.ok = false;
    r.sbytes = scode ? scode : 1024;
    if (r.sbytes > (count + 7) / 8) r.ok = false;
    r.mbytes = r.raw ? 2 * count : code;
    return r;
}

// Copies src[0, len) to dst[mis, mis + len), mis = src mod 16 (dst 16-byte
// aligned): 16-byte loads for granules wholly inside the range, bytes at its
// ends. Returns mis.
__device__ __forceinline__ uint32_t stage_bytes(uint8_t* dst, const uint8_t* src, uint32_t len, int tid, int nt) {
    const uint32_t mis = uint32_t(reinterpret_cast<uintptr_t>(src) & 15u);
    const uint8_t* a0 = src - mis;
    const uint32_t n16 = (mis + len + 15) / 16;
    for (uint32_t i = tid; i < n16; i += nt) {
        const uint32_t lo = 16 * i;
        if (lo >= mis && lo + 16 <= mis + len) {
            reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(a0)[i];
        } else {
            for (uint32_t k = 0; k < 16; ++k) {
                const uint32_t r = lo + k;
                if (r >= mis && r < mis + len) dst[r] = a0[r];
            }
        }
    }
    return mis;
}

template <class T> struct WzpDecodeArgs {
    JobRef job;         // archive base, WZP stream length, quantum
    uint32_t n;
    BrickMap map;
    T* coeff;           // row-major dequantised coefficients (output)
    uint32_t* status;
};

template <class T> struct WzpDecodeOp {
    static constexpr int kThreads = kWzpThreads, kMinBlocks = 4; // 32 registers: four CTAs per SM
    using Params = WzpDecodeArgs<T>;
    static __device__ __forceinline__ void run(const Params A, uint32_t block, uint32_t);
};

template <class T>
__device__ __forceinline__ void WzpDecodeOp<T>::run(const Params A, uint32_t block, uint32_t) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WzpDecodeSmem& S = *reinterpret_cast<WzpDecodeSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kWzpThreads / 32;
    const uint32_t chunks = wzp_chunks(A.n), groups = wzp_groups(A.n);
    const uint32_t c = block;
    const uint32_t first = c * kChunk, count = min(kChunk, A.n - first);
    const size_t header = size_t(groups) * 4 + size_t(chunks) * 3;
    const DecodeJob J = A.job.get();
    const uint8_t* in = J.base + 32;
    const T q = T(J.q);
    const uint8_t* meta = in + size_t(groups) * 4;
    const uint8_t* payload = in + header;
    const size_t payload_bytes = J.wzp - header;
    // whole bricks (chunks are runs of them): one thread per 16-sample block
    const bool blockwise = A.map.fast && (reinterpret_cast<uintptr_t>(A.coeff) & 15u) == 0;

    if (warp == 0) {
        // Lane k reads the metadata of the group's chunk k; the chunk's payload
        // offset is the group offset plus its predecessors' lengths.
        const uint32_t g = c / kGroup, k = g * kGroup + lane;
        WzpChunkInfo ci{0, 0, false, true};
        if (lane < int(kGroup) && k <= c) ci = wzp_meta(load_u24(meta + size_t(k) * 3), min(kChunk, A.n - k * kChunk));
        const uint32_t len = (lane < int(kGroup) && k < c) ? ci.mbytes + ci.sbytes : 0u;
        const uint32_t before = __reduce_add_sync(0xffffffffu, len);
        const bool ok_all = __all_sync(0xffffffffu, ci.ok);
        const int me = int(c - g * kGroup);
        const uint32_t mb = __shfl_sync(0xffffffffu, ci.mbytes, me);
        const uint32_t sb = __shfl_sync(0xffffffffu, ci.sbytes, me);
        const bool raw = __shfl_sync(0xffffffffu, ci.raw ? 1u : 0u, me) != 0;
        if (lane == 0) {
            const uint64_t off = uint64_t(load_u32(in + size_t(g) * 4)) + before;
            const bool ok = ok_all && off + mb + sb <= payload_bytes;
            S.off = uint32_t(off);
            S.mbytes = mb;
            S.sbytes = sb;
            S.raw = raw;
            S.bad = !ok;
            if (!ok) atomicOr(A.status, ST_BAD_STREAM);
        }
    }
    __syncthreads();
    if (S.bad) return;
    const uint8_t* gsrc = payload + S.off;
    const uint32_t mbytes = S.mbytes, sbytes = S.sbytes;
    const uint32_t raw_bytes = 2 * count;
    const uint32_t blocks = count / 16;
    bool bad = false;
    // stage the chunk's compressed magnitude bytes and its sign bytes
    uint8_t* mstage = reinterpret_cast<uint8_t*>(S.m);
    uint32_t mis_m = 0, mis_s = 0;
    if (mbytes && !S.raw) mis_m = stage_bytes(mstage, gsrc, mbytes, tid, kWzpThreads);
    if (sbytes) mis_s = stage_bytes(S.sb, gsrc + mbytes, sbytes, tid, kWzpThreads);
    if (tid < 16) {
        uint32_t sel = 0, k = 0;
        for (int b = 0; b < 4; ++b) sel |= (((tid >> b) & 1) ? k++ : 4u) << (4 * b);
        S.xsel[tid] = sel;
    }
    __syncthreads();
    const uint8_t* src = mstage + mis_m; // compressed magnitude bytes (RZE chunks)
    const uint8_t* sgn = S.sb + mis_s;

    if (mbytes == 0) {
        for (int i = tid; i < int(kChunk); i += kWzpThreads) S.m[i] = 0;
    } else if (S.raw) {
        for (int i = tid; i < int(kChunk); i += kWzpThreads)
            S.m[i] = i < int(count) ? uint16_t(gsrc[2 * i] | (gsrc[2 * i + 1] << 8)) : 0;
    } else {
        // ---- undo repetition elimination from the back of the stream
        uint32_t pos = mbytes - 4;
        uint8_t* L3 = S.lv + 2048 + 256 + 32;
        uint8_t* L2 = S.lv + 2048 + 256;
        uint8_t* L1 = S.lv + 2048;
        uint8_t* L0 = S.lv;
        if (tid < 4) L3[tid] = src[pos + tid];
        __syncthreads();
        // level 2 (32 bytes) from L3
        if (warp == 0) {
            const uint32_t mark = uint32_t(L3[0]) | (uint32_t(L3[1]) << 8) | (uint32_t(L3[2]) << 16) | (uint32_t(L3[3]) << 24);
            const uint32_t cnt = __popc(mark);
            const bool under = cnt > pos;
            const uint32_t base = under ? 0 : pos - cnt;
            const uint32_t rank = __popc(mark & ((2u << lane) - 1u)); // inclusive (lane 31 ok: 2u<<31 == 0)
            const uint32_t r = lane == 31 ? cnt : rank;
            uint8_t v = 0;
            if (!under && r) v = src[base + r - 1];
            if (!under && ((mark >> lane) & 1u)) {
                const uint8_t prev = r > 1 ? src[base + r - 2] : 0;
                if (v == prev) bad = true;
            }
            L2[lane] = v;
            if (under) bad = true;
            if (lane == 0) S.tmp[36] = base;
        }
        __syncthreads();
        pos = S.tmp[36];
        // level 1 (256 bytes) from L2
        {
            uint32_t bit = 0;
            if (tid < 256) bit = (L2[tid >> 3] >> (tid & 7)) & 1u;
            uint32_t cnt;
            const uint32_t ex = block_excl_scan<kWzpThreads>(bit, S.tmp, cnt);
            const bool under = cnt > pos;
            const uint32_t base = under ? 0 : pos - cnt;
            if (tid < 256) {
                const uint32_t r = ex + bit;
                uint8_t v = 0;
                if (!under && r) v = src[base + r - 1];
                if (!under && bit) {
                    const uint8_t prev = r > 1 ? src[base + r - 2] : 0;
                    if (v == prev) bad = true;
                }
                L1[tid] = v;
            }
            if (under) bad = true;
            pos = base;
        }
        __syncthreads();
        // level 0 (2048 bytes) from L1: four entries per thread
        {
            uint32_t bits4 = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int i = tid * 4 + k;
                bits4 |= ((L1[i >> 3] >> (i & 7)) & 1u) << k;
            }
            uint32_t cnt;
            const uint32_t ex = block_excl_scan<kWzpThreads>(__popc(bits4), S.tmp, cnt);
            const bool under = cnt > pos;
            const uint32_t base = under ? 0 : pos - cnt;
            uint32_t r = ex;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t bit = (bits4 >> k) & 1u;
                r += bit;
                uint8_t v = 0;
                if (!under && r) v = src[base + r - 1];
                if (!under && bit) {
                    const uint8_t prev = r > 1 ? src[base + r - 2] : 0;
                    if (v == prev) bad = true;
                }
                L0[tid * 4 + k] = v;
            }
            if (under) bad = true;
            pos = base;
        }
        __syncthreads();
        // nonzero bytes: 32 per thread
        {
            const uint32_t bits = uint32_t(L0[4 * tid]) | (uint32_t(L0[4 * tid + 1]) << 8) |
                                  (uint32_t(L0[4 * tid + 2]) << 16) | (uint32_t(L0[4 * tid + 3]) << 24);
            uint32_t cnt;
            const uint32_t ex = block_excl_scan<kWzpThreads>(__popc(bits), S.tmp, cnt);
            if (cnt == 0 || cnt != pos) bad = true;
            const uint32_t b0 = tid * 32;
            // bitmap beyond the chunk's bytes must be empty
            if (b0 + 32 > raw_bytes) {
                const uint32_t keep = b0 >= raw_bytes ? 0u : (raw_bytes - b0 >= 32 ? 32u : raw_bytes - b0);
                const uint32_t allowed = keep == 32 ? 0xffffffffu : ((1u << keep) - 1u);
                if (bits & ~allowed) bad = true;
            }
            // spread the next popc(mask) stream bytes over each word's set
            // bytes; every one of them must be nonzero and inside the stream
            uint32_t r = ex;
            if (r + __popc(bits) > pos) bad = true;
            const uint32_t* sw = reinterpret_cast<const uint32_t*>(mstage);
            uint32_t words[8];
#pragma unroll
            for (int w = 0; w < 8; ++w) {
                const uint32_t m4 = (bits >> (4 * w)) & 15u;
                const uint32_t b = mis_m + r, wi = b >> 2;
                const uint32_t val = __funnelshift_r(sw[wi], sw[wi + 1], 8 * (b & 3u));
                const uint32_t word = __byte_perm(val, 0u, S.xsel[m4]);
                if (nonzero_nibble(word) != m4) bad = true;
                words[w] = bad ? 0u : word;
                r += __popc(m4);
            }
            __syncthreads(); // every thread has read the staged bytes it needs
            // full chunks write the padded layout (plane t / 32 at pitch
            // kEncPitch) straight away; a partial chunk writes the natural one
            const uint32_t pad = blocks == kChunk / 16 ? 4 * (kEncPitch - kChunk / 32) * (uint32_t(tid) >> 5) : 0u;
            uint4* out = reinterpret_cast<uint4*>(S.planes + b0 + pad);
            out[0] = make_uint4(words[0], words[1], words[2], words[3]);
            out[1] = make_uint4(words[4], words[5], words[6], words[7]);
        }
        __syncthreads();
        // the verbatim tail (samples past the last whole block) while a
        // partial chunk's planes are still in the natural layout
        const uint16_t* pl = reinterpret_cast<const uint16_t*>(S.planes);
        uint16_t tail = 0;
        const uint32_t ti = blocks * 16 + tid;
        if (ti < count) tail = pl[ti];
        const bool full = blocks == kChunk / 16;
        if (!full) planes_repack(S.planes, blocks, true, tid);
        __syncthreads();
        if (!blockwise) { // else each thread transposes its own block below
        // ---- inverse bit planes, two groups per warp step: lane l holds plane
        // l % 16 of group g0 + l / 16 (bit 31-e = magnitude e's bit 15-p); one
        // 32x32 transpose leaves magnitude e of g0 in the high half of lane e's
        // word and of g0 + 1 in the low half
        const uint32_t pitch = full ? kEncPitch : kPlanePitch, in_planes = blocks * 16;
        for (int k = warp; k < int(kChunk / 64); k += NW) {
            const int g0 = 2 * k;
            if (uint32_t(g0 * 32) >= in_planes) break;
            const uint32_t g = uint32_t(g0) + (uint32_t(lane) >> 4);
            uint32_t w = 0;
            if (2 * g < blocks) {
                const uint32_t word = reinterpret_cast<const uint32_t*>(S.planes)[(uint32_t(lane) & 15u) * pitch + g];
                w = __funnelshift_l(word, word, 16);
                if (2 * g + 1 >= blocks) w &= 0xffff0000u;
            }
            const uint32_t r = __brev(warp_transpose32(__brev(w), lane));
            const uint32_t e0 = uint32_t(g0) * 32 + lane, m0 = r >> 16, m1 = r & 0xffffu;
            if (e0 < in_planes) S.m[e0] = uint16_t(m0);
            if (e0 + 32 < in_planes) S.m[e0 + 32] = uint16_t(m1);
            // groups wholly inside the planes: their nonzero counts now
            const uint32_t nzm0 = __ballot_sync(0xffffffffu, m0 != 0), nzm1 = __ballot_sync(0xffffffffu, m1 != 0);
            if (lane < 2 && (uint32_t(g0) + lane) * 32 + 32 <= in_planes) {
                S.gprefix[g0 + lane] = __popc(lane ? nzm1 : nzm0);
                S.gmask[g0 + lane] = lane ? nzm1 : nzm0;
            }
        }
        for (uint32_t i = blocks * 16 + tid; i < kChunk; i += kWzpThreads)
            S.m[i] = i == ti ? tail : 0;
        }
    }
    __syncthreads();

    if (blockwise) {
        // ---- one thread per 16-sample block (whole bricks): magnitudes from
        // its 16 bit planes (one transpose) or the verbatim ones, nonzero
        // ranks by one block scan, signs spread from the sign stream, then the
        // dequantised block stored as four 16-byte rows
        const uint32_t t = uint32_t(tid);
        uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (t < blocks && mbytes != 0) {
            if (S.raw) {
                const uint4* sm = reinterpret_cast<const uint4*>(S.m + 16 * t);
                const uint4 a = sm[0], b = sm[1];
                w[0] = a.x, w[1] = a.y, w[2] = a.z, w[3] = a.w, w[4] = b.x, w[5] = b.y, w[6] = b.z, w[7] = b.w;
            } else {
                const uint16_t* pl = reinterpret_cast<const uint16_t*>(S.planes);
                const uint32_t stride = blocks == kChunk / 16 ? 2 * kEncPitch : 2 * kPlanePitch;
#pragma unroll
                for (int i = 0; i < 8; ++i)
                    w[i] = uint32_t(pl[2 * i * stride + t]) | (uint32_t(pl[(2 * i + 1) * stride + t]) << 16);
                if ((w[0] | w[1] | w[2] | w[3] | w[4] | w[5] | w[6] | w[7]) != 0) bit_transpose16(w);
            }
        }
        uint32_t zm = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t nzh = __vsetne2(w[i], 0u); // 0xffff per nonzero half
            zm |= ((nzh & 1u) | ((nzh >> 15) & 2u)) << (2 * i);
        }
        const uint32_t cnt = __popc(zm);
        uint32_t nnz;
        const uint32_t base = block_excl_scan<kWzpThreads>(cnt, S.tmp, nnz);
        if (mbytes != 0) {
            if (nnz == 0 || (nnz + 7) / 8 != sbytes) bad = true;
            else if ((nnz & 7) && (sgn[sbytes - 1] >> (nnz & 7))) bad = true;
        }
        if (t < blocks) {
            uint32_t nm = 0;
            if (cnt && !bad) {
                const uint32_t by = base >> 3;
                const uint32_t bits = uint32_t(sgn[by]) | (uint32_t(sgn[by + 1]) << 8) | (uint32_t(sgn[by + 2]) << 16);
                nm = expand16((bits >> (base & 7u)) & ((1u << cnt) - 1u), zm);
            }
            if (A.map.bz == 16) store_block<T, true>(A.map, A.coeff, first, t, w, nm, q);
            else store_block<T, false>(A.map, A.coeff, first, t, w, nm, q);
        }
        if (bad) atomicOr(A.status, ST_BAD_STREAM);
        return;
    }

    // ---- signs and dequantisation: nonzero counts of the remaining groups
    const int counted = (mbytes != 0 && !S.raw) ? int(blocks * 16 / 32) : 0;
    for (int g = counted + warp; g < int(kChunk / 32); g += NW) {
        const uint32_t nzm = __ballot_sync(0xffffffffu, S.m[g * 32 + lane] != 0);
        if (lane == 0) {
            S.gprefix[g] = __popc(nzm);
            S.gmask[g] = nzm;
        }
    }
    if (A.map.fast && tid < int(kChunk >> A.map.lb)) S.bbase[tid] = A.map.brick_base((first >> A.map.lb) + tid);
    __syncthreads();
    uint32_t nnz = 0;
    {
        const uint32_t gc = tid < int(kChunk / 32) ? S.gprefix[tid] : 0;
        const uint32_t gp = block_excl_scan<kWzpThreads>(gc, S.tmp, nnz);
        if (tid < int(kChunk / 32)) S.gprefix[tid] = gp;
    }
    if (mbytes != 0) {
        if (nnz == 0 || (nnz + 7) / 8 != sbytes) bad = true;
        else if ((nnz & 7) && (sgn[sbytes - 1] >> (nnz & 7))) bad = true;
    }
    __syncthreads();
    // sign of the magnitude at Morton slot e: the sign bit at its rank among
    // the chunk's nonzero magnitudes
    auto negative = [&](uint32_t e, uint32_t v) {
        if (!v || bad) return false;
        const uint32_t rank = S.gprefix[e >> 5] + __popc(S.gmask[e >> 5] & ((1u << (e & 31u)) - 1u));
        return rank < 8 * sbytes && ((sgn[rank >> 3] >> (rank & 7)) & 1u);
    };
    if (A.map.fast && A.map.rank &&
        ((reinterpret_cast<uintptr_t>(A.coeff) & 15u) | (reinterpret_cast<uintptr_t>(A.map.rank) & 7u)) == 0) {
        // whole bricks: four consecutive samples of a brick row per step,
        // gathered from their Morton slots, one 16-byte store
        const uint32_t bsz = 1u << A.map.lb, plane = A.map.nx * A.map.ny;
        for (uint32_t e = 4 * uint32_t(tid); e < count; e += 4 * kWzpThreads) {
            const uint32_t j = e >> A.map.lb, i = e & (bsz - 1u);
            const uint32_t at = S.bbase[j] + (i >> 8) * plane + ((i >> 4) & 15u) * A.map.nx + (i & 15u);
            const uint2 rk = *reinterpret_cast<const uint2*>(A.map.rank + i);
            T v4[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t slot = (j << A.map.lb) + (((k < 2 ? rk.x : rk.y) >> (16 * (k & 1))) & 0xffffu);
                const uint32_t v = S.m[slot];
                const T mag = Lift<T>::mul(T(v), q);
                v4[k] = negative(slot, v) ? -mag : mag;
            }
            store4(A.coeff + at, v4);
        }
    } else {
        for (int g = warp; g < int(kChunk / 32); g += NW) {
            if (uint32_t(g * 32) >= count) break;
            const int e = g * 32 + lane;
            const uint32_t v = S.m[e];
            if (uint32_t(e) < count) {
                const T mag = Lift<T>::mul(T(v), q);
                const uint32_t at = A.map.fast ? A.map.in_full_brick(S.bbase[uint32_t(e) >> A.map.lb],
                                                                     uint32_t(e) & ((1u << A.map.lb) - 1u))
                                               : A.map.rowmajor(first + uint32_t(e));
                A.coeff[at] = negative(uint32_t(e), v) ? -mag : mag;
            }
        }
    }
    if (bad) atomicOr(A.status, ST_BAD_STREAM);
}

} // namespace wb

// Uniform scalar quantisation fused with the block Morton reorder, and the
// side-record kernels (ordered compaction, decode patches, extrema).
#pragma once
#include "common.cuh"
#include "compact.cuh"
#include "scan.cuh"

namespace wb {

// Brick grid of the coefficient array: 16 x 16 x bz bricks in raster order.
struct Bricks {
    uint32_t nx, ny, nz, bz;
    uint32_t nbx, nby, nbz;
    __host__ __device__ static Bricks make(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t bz) {
        return {nx, ny, nz, bz, (nx + 15) / 16, (ny + 15) / 16, (nz + bz - 1) / bz};
    }
    __host__ __device__ uint64_t count() const { return uint64_t(nbx) * nby * nbz; }
};

// q = T(1.5 eb), inv = T(1 / (1.5 eb)); code = llrint(T(c * inv)) saturated to
// +-INT32_MAX; the dequantised value T(+-|code|) * q replaces the coefficient
// (cpu/src/codec.cpp:211-220). Magnitudes are clamped to 16 bits at their
// Morton position; larger ones become q-outliers (index, magnitude).
template <class T> struct QuantArgs {
    T* coeff;                 // in: coefficients, out: dequantised values
    Bricks b;
    const uint16_t* rank;     // 8 slots x 256*bz: local row-major index -> rank
    T q, inv;
    uint16_t* mag;            // Morton-packed magnitudes
    uint32_t* sign;           // Morton-packed sign bits (zeroed before launch)
    uint32_t* qbits;          // row-major q-outlier bitmap (zeroed before launch)
    uint32_t* qval;           // row-major q-outlier magnitudes (dense, sparse use)
    uint32_t* status;
};

constexpr int kQuantThreads = 256;

// Rounds x (|x| below kFastQuant) to the nearest integer, ties to even,
// with one add of 1.5 * 2^(mantissa bits): the sum's low bits then hold the
// rounded value. Returns the integer; `back` receives it as T exactly.
template <class T> struct FastRound;
template <> struct FastRound<float> {
    static constexpr float kLimit = 4194304.0f; // 2^22
    static __device__ __forceinline__ int32_t round(float x, float& back) {
        const float t = __fadd_rn(x, 12582912.0f); // 1.5 * 2^23
        back = __fsub_rn(t, 12582912.0f);
        return int32_t(__float_as_uint(t) & 0x7fffffu) - 0x400000;
    }
};
template <> struct FastRound<double> {
    static constexpr double kLimit = 1073741824.0; // 2^30
    static __device__ __forceinline__ int32_t round(double x, double& back) {
        const double t = __dadd_rn(x, 6755399441055744.0); // 1.5 * 2^52
        back = __dsub_rn(t, 6755399441055744.0);
        return int32_t(int64_t(uint64_t(__double_as_longlong(t)) & 0xfffffffffffffull) - (int64_t(1) << 51));
    }
};

// Quantisation of one coefficient: code = llrint(T(c * inv)) saturated to
// +-INT32_MAX (magnitude m, sign neg); returns the dequantised T(+-m) * q.
// Sets bad for a non-finite or out-of-range scaled value (then m = 0).
template <class T>
__device__ __forceinline__ T quantize_one(T c, T inv, T q, int32_t& m, bool& neg, uint32_t& bad) {
    const T scaled = Lift<T>::mul(c, inv);
    m = 0;
    neg = false;
    if (fabs(scaled) < FastRound<T>::kLimit) {
        T back;
        const int32_t r = FastRound<T>::round(scaled, back);
        neg = r < 0;
        m = neg ? -r : r;
        return m ? Lift<T>::mul(back, q) : T(0);
    }
    if (!finite_bits(scaled) || fabs(double(scaled)) >= 9223372036854775808.0) {
        bad = 1;
        return T(0);
    }
    long long r;
    if constexpr (sizeof(T) == 4) r = __float2ll_rn(scaled);
    else r = __double2ll_rn(scaled);
    neg = r < 0;
    const unsigned long long m64 = neg ? (unsigned long long)(-r) : (unsigned long long)r;
    m = m64 > 0x7fffffffull ? 0x7fffffff : int32_t(m64);
    return Lift<T>::mul(T(neg ? -m : m), q);
}

template <class T> struct QuantizeOp {
    static constexpr int kThreads = kQuantThreads, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    using Params = QuantArgs<T>;
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t);
};

template <class T>
__device__ __forceinline__ void QuantizeOp<T>::run(const Params A, uint32_t block, uint32_t) {
    __shared__ __align__(16) uint16_t smag[kChunk];
    __shared__ __align__(16) uint8_t ssign[kChunk];
    const Bricks& B = A.b;
    const uint64_t bi = block;
    const uint32_t bxi = uint32_t(bi % B.nbx), byi = uint32_t((bi / B.nbx) % B.nby), bzi = uint32_t(bi / (uint64_t(B.nbx) * B.nby));
    const uint32_t ex = min(16u, B.nx - bxi * 16), ey = min(16u, B.ny - byi * 16), ez = min(B.bz, B.nz - bzi * B.bz);
    const uint32_t slot = (ex != 16) | ((ey != 16) << 1) | ((ez != B.bz) << 2);
    const uint64_t plane = uint64_t(B.nx) * B.ny;
    const uint64_t base = uint64_t(bzi) * B.bz * plane + uint64_t(byi) * 16 * B.nx * ez + uint64_t(bxi) * 16 * ey * ez;
    const uint32_t size = ex * ey * ez;
    const bool full = ex == 16 && ey == 16;
    const uint16_t* rank = A.rank + slot * 256 * B.bz;
    const T* corner = A.coeff + (uint64_t(bzi) * B.bz) * plane + uint64_t(byi) * 16 * B.nx + bxi * 16;
    uint32_t bad = 0;
    for (uint32_t i = threadIdx.x; i < size; i += kQuantThreads) {
        uint32_t lx, ly, lz;
        if (full) {
            lx = i & 15u;
            ly = (i >> 4) & 15u;
            lz = i >> 8;
        } else {
            lx = i % ex;
            ly = (i / ex) % ey;
            lz = i / (ex * ey);
        }
        T* cp = const_cast<T*>(corner) + lz * plane + uint64_t(ly) * B.nx + lx;
        int32_t m;
        bool neg;
        *cp = quantize_one<T>(*cp, A.inv, A.q, m, neg, bad);
        const uint32_t rk = rank[i];
        smag[rk] = uint16_t(m > 65535 ? 65535 : m);
        ssign[rk] = neg && m;
        if (m > 65535) {
            const uint64_t at = uint64_t(cp - A.coeff);
            atomicOr(&A.qbits[at >> 5], 1u << (at & 31));
            A.qval[at] = uint32_t(m);
        }
    }
    if (bad) atomicOr(A.status, ST_QUANT_DOMAIN);
    __syncthreads();
    if (base % 32 == 0 && size % 32 == 0) {
        // brick on whole sign words: 16-byte magnitude stores (base is a
        // multiple of 8 magnitudes), sign words owned outright
        for (uint32_t i = threadIdx.x; i < size / 8; i += kQuantThreads)
            reinterpret_cast<uint4*>(A.mag + base)[i] = reinterpret_cast<const uint4*>(smag)[i];
        for (uint32_t w = threadIdx.x; w < size / 32; w += kQuantThreads) {
            const uint32_t* sw = reinterpret_cast<const uint32_t*>(ssign + 32 * w);
            uint32_t bits = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) bits |= (((sw[k] & 0x01010101u) * 0x01020408u) >> 24) << (4 * k);
            if (bits) A.sign[(base >> 5) + w] = bits;
        }
        return;
    }
    for (uint32_t i = threadIdx.x; i < size; i += kQuantThreads) A.mag[base + i] = smag[i];
    // sign words overlapping [base, base+size)
    const uint64_t w0 = base >> 5, w1 = (base + size + 31) >> 5;
    for (uint64_t w = w0 + threadIdx.x; w < w1; w += kQuantThreads) {
        uint32_t bits = 0;
        for (int k = 0; k < 32; ++k) {
            const uint64_t p = w * 32 + k;
            if (p >= base && p < base + size && ssign[p - base]) bits |= 1u << k;
        }
        if (bits) atomicOr(&A.sign[w], bits);
    }
}

// Copy with a finiteness check (zero-level transform: coefficients = input).
template <class T> struct CopyFiniteOp {
    static constexpr int kThreads = 256, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        const T* in;
        T* out;
        uint64_t n;
        uint32_t* status;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t blocks) {
        bool bad = false;
        for (uint64_t i = block * uint64_t(kThreads) + threadIdx.x; i < P.n; i += uint64_t(blocks) * kThreads) {
            const T v = P.in[i];
            bad |= !finite_bits(v);
            P.out[i] = v;
        }
        if (bad) atomicOr(P.status, ST_NONFINITE_INPUT);
    }
};

// Encoder repair emitter for the finest synthesis: err = T(value - orig);
// a sample is patched iff |err| > T(eb); the corrected value must be finite
// and strictly within eb of the original (cpu/src/repair_avx2.cpp:57-74).
// The original is fetched ahead of the synthesis (kPrefetch). A corrected
// value whose rounded float difference is at most `safe` (eb shrunk by
// 2^-21, rounded down) passes the strict double check for certain, so only
// values near the bound take the two-difference test; float only.
template <class T> struct RepairOut {
    const T* orig;
    size_t sy, sz;
    double bound;
    T nb;
    uint32_t* pbits;  // row-major bitmap of patched samples
    T* perr;          // dense errors (sparse use)
    uint32_t* status;
    T safe;           // float: fast-accept threshold; double: unused
    static constexpr bool kPrefetch = true;
    __device__ __forceinline__ T fetch(uint32_t x, uint32_t y, uint32_t z) const {
        return __ldg(orig + size_t(z) * sz + size_t(y) * sy + x);
    }
    // asks L2 for the line holding original (x, y, z) ahead of its fetch
    __device__ __forceinline__ void warm(uint32_t x, uint32_t y, uint32_t z) const {
        asm volatile("prefetch.global.L2 [%0];" ::"l"(orig + size_t(z) * sz + size_t(y) * sy + x));
    }
    __device__ __forceinline__ void emit(uint32_t x, uint32_t y, uint32_t z, T v, T o) const {
        const T err = Lift<T>::sub(v, o);
        const bool patched = fabs(err) > nb;
        const T w = patched ? Lift<T>::sub(v, err) : v;
        bool ok = finite_bits(v) && finite_bits(err) && finite_bits(w);
        if (ok) {
            if constexpr (sizeof(T) == 4) {
                if (!(fabsf(Lift<T>::sub(w, o)) <= safe)) ok = strictly_within(double(w), double(o), bound);
            } else {
                ok = strictly_within(double(w), double(o), bound);
            }
        }
        if (patched) {
            const size_t i = size_t(z) * sz + size_t(y) * sy + x;
            atomicOr(&pbits[i >> 5], 1u << (i & 31));
            perr[i] = err;
        }
        if (!ok) atomicOr(status, ST_BOUND);
    }
    __device__ __forceinline__ void operator()(uint32_t x, uint32_t y, uint32_t z, T v) const {
        emit(x, y, z, v, fetch(x, y, z));
    }
};

// Decoder final store with the finiteness check fused in.
template <class T> struct FinalOut {
    static constexpr bool kPrefetch = false;
    T* dst;
    size_t sy, sz;
    uint32_t* status;
    __device__ __forceinline__ void operator()(uint32_t x, uint32_t y, uint32_t z, T v) const {
        dst[size_t(z) * sz + size_t(y) * sy + x] = v;
        if (!finite_bits(v)) atomicOr(status, ST_NONFINITE_INPUT);
    }
};

// Output into a strided box whose base address is read from the device job
// table at each store, so a replayed decode graph writes wherever the job
// table says (a fresh tensor per batch).
template <class T> struct JobOut {
    static constexpr bool kPrefetch = false;
    const DecodeJob* job;
    size_t sy, sz;
    uint32_t* status;
    __device__ __forceinline__ void operator()(uint32_t x, uint32_t y, uint32_t z, T v) const {
        T* dst = reinterpret_cast<T*>(__ldg(reinterpret_cast<const unsigned long long*>(&job->out)));
        dst[size_t(z) * sz + size_t(y) * sy + x] = v;
        if (!finite_bits(v)) atomicOr(status, ST_NONFINITE_INPUT);
    }
};

// ----------------------------------------------- ordered bitmap compaction
// Set bits of a row-major bitmap, in ascending index order, become
// (index, value) records: pass 1 counts per block, pass 2 scans the block
// counts (single CTA) and lays out the archive, pass 3 writes. Ordered by
// construction, no sort. Both record lists (repair records, q-outliers) go
// through each pass together: the second half of the grid takes the
// q-outlier list.
constexpr int kCompactThreads = 256;
constexpr int kCompactWords = kCompactThreads * 4; // bitmap words per block

// Grid: 2 x cblocks blocks, the second half on the q-outlier list.
struct CompactCountOp {
    static constexpr int kThreads = kCompactThreads, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        const uint32_t *pbits, *qbits;
        uint64_t words;
        uint32_t *counts_p, *counts_q;
        uint32_t cblocks;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t) {
        __shared__ uint32_t tmp[40];
        const bool q = block >= P.cblocks;
        const uint32_t bx = q ? block - P.cblocks : block;
        const uint32_t* bits = q ? P.qbits : P.pbits;
        const uint64_t w0 = uint64_t(bx) * kCompactWords + threadIdx.x * 4;
        uint32_t c = 0;
        for (int k = 0; k < 4; ++k)
            if (w0 + k < P.words) c += __popc(bits[w0 + k]);
        const uint32_t total = block_sum<kCompactThreads>(c, tmp);
        if (threadIdx.x == 0) (q ? P.counts_q : P.counts_p)[bx] = total;
    }
};

// Record sink: indices as u32 LE, values of sizeof(V) bytes, both at
// device-side offsets inside the archive (given by `layout`).
template <class V>
__device__ __forceinline__ void compact_write_block(uint32_t bx, const uint32_t* bits, uint64_t words,
                                                    const uint32_t* offsets, const V* values, uint8_t* archive,
                                                    const uint64_t* layout, int idx_slot, int val_slot,
                                                    uint64_t cap_records, uint32_t* tmp) {
    const uint64_t w0 = uint64_t(bx) * kCompactWords + threadIdx.x * 4;
    uint32_t wv[4];
    uint32_t c = 0;
    for (int k = 0; k < 4; ++k) {
        wv[k] = w0 + k < words ? bits[w0 + k] : 0;
        c += __popc(wv[k]);
    }
    uint32_t total;
    uint32_t r = offsets[bx] + block_excl_scan<kCompactThreads>(c, tmp, total);
    if (layout[7]) return; // layout overflow: nothing is written
    uint8_t* idx = archive + layout[idx_slot];
    uint8_t* val = archive + layout[val_slot];
    const bool aligned = (reinterpret_cast<uintptr_t>(archive) & 7u) == 0;
    for (int k = 0; k < 4; ++k)
        for (uint32_t b = wv[k]; b; b &= b - 1) {
            const uint64_t i = (w0 + k) * 32 + (__ffs(b) - 1);
            if (r < cap_records) {
                const uint32_t ii = uint32_t(i);
                const V v = values[i];
                if (aligned) {
                    // sections start on 8-byte offsets: whole-word stores
                    reinterpret_cast<uint32_t*>(idx)[r] = ii;
                    reinterpret_cast<V*>(val)[r] = v;
                } else {
                    idx[4 * uint64_t(r) + 0] = uint8_t(ii);
                    idx[4 * uint64_t(r) + 1] = uint8_t(ii >> 8);
                    idx[4 * uint64_t(r) + 2] = uint8_t(ii >> 16);
                    idx[4 * uint64_t(r) + 3] = uint8_t(ii >> 24);
                    const uint8_t* vb = reinterpret_cast<const uint8_t*>(&v);
                    for (int j = 0; j < int(sizeof(V)); ++j) val[sizeof(V) * uint64_t(r) + j] = vb[j];
                }
            }
            ++r;
        }
}

// Grid: 2 x cblocks blocks, the second half on the q-outlier list.
template <class T> struct CompactWriteOp {
    static constexpr int kThreads = kCompactThreads, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        const uint32_t *pbits, *qbits;
        uint64_t words;
        const uint32_t *offsets_p, *offsets_q;
        const T* perr;
        const uint32_t* qval;
        uint8_t* archive;
        const uint64_t* layout;
        uint64_t cap_records;
        uint32_t cblocks;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t) {
        __shared__ uint32_t tmp[40];
        if (block < P.cblocks)
            compact_write_block<T>(block, P.pbits, P.words, P.offsets_p, P.perr, P.archive, P.layout, 0, 1,
                                   P.cap_records, tmp);
        else
            compact_write_block<uint32_t>(block - P.cblocks, P.qbits, P.words, P.offsets_q, P.qval, P.archive,
                                          P.layout, 2, 3, P.cap_records, tmp);
    }
};

// Exclusive scan of both lists' block counts in place, then the archive
// layout from the totals. layout[]: 0 pi, 1 pv, 2 qi, 3 qv, 4 end, 5 np,
// 6 nq, 7 overflow flag, 8 the pipeline's status word. Also writes the
// 32-byte header and zeroes every padding byte between sections.
struct ScanLayoutOp {
    static constexpr int kThreads = kCompactThreads, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        uint32_t *counts_p, *counts_q;
        uint32_t count;
        const uint64_t* wzp_total;
        const uint32_t* status;
        uint8_t* archive;
        size_t capacity;
        uint32_t width;
        uint8_t flags, lxy, lz, bz;
        double quantum;
        uint64_t* layout;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t, uint32_t);
};

__device__ __forceinline__ void ScanLayoutOp::run(const Params P, uint32_t, uint32_t) {
    uint32_t* const counts_p = P.counts_p;
    uint32_t* const counts_q = P.counts_q;
    const uint32_t count = P.count, width = P.width;
    const uint64_t* wzp_total = P.wzp_total;
    const uint32_t* status = P.status;
    uint8_t* const archive = P.archive;
    const size_t capacity = P.capacity;
    const uint8_t flags = P.flags, lxy = P.lxy, lz = P.lz, bz = P.bz;
    const double quantum = P.quantum;
    uint64_t* const layout = P.layout;
    __shared__ uint32_t tmp[40];
    uint32_t totals[2];
    // each thread takes a run of consecutive block counts: its run's sum, one
    // block scan for the runs' offsets, then the run rewritten as exclusive
    // prefixes (two block scans in all instead of one per kCompactThreads)
    const uint32_t per = (count + kCompactThreads - 1) / kCompactThreads;
    const uint32_t b0 = min(count, threadIdx.x * per), b1 = min(count, b0 + per);
    for (int list = 0; list < 2; ++list) {
        uint32_t* counts = list ? counts_q : counts_p;
        uint32_t run = 0;
        for (uint32_t i = b0; i < b1; ++i) run += counts[i];
        uint32_t sum;
        uint32_t at = block_excl_scan<kCompactThreads>(run, tmp, sum);
        for (uint32_t i = b0; i < b1; ++i) {
            const uint32_t v = counts[i];
            counts[i] = at;
            at += v;
        }
        totals[list] = sum;
    }
    if (threadIdx.x != 0) return;
    const uint64_t wb = *wzp_total; // includes the WZP header
    const uint32_t np = totals[0], nq = totals[1];
    const uint64_t pi = 32 + pad8(wb);
    const uint64_t pv = pi + pad8(uint64_t(np) * 4);
    const uint64_t qi = pv + pad8(uint64_t(np) * width);
    const uint64_t qv = qi + pad8(uint64_t(nq) * 4);
    const uint64_t end = qv + pad8(uint64_t(nq) * 4);
    layout[0] = pi;
    layout[1] = pv;
    layout[2] = qi;
    layout[3] = qv;
    layout[4] = end;
    layout[5] = np;
    layout[6] = nq;
    layout[7] = end > capacity;
    layout[8] = *status;
    if (end > capacity) return;
    archive[0] = flags;
    archive[1] = lxy;
    archive[2] = lz;
    archive[3] = bz;
    const uint32_t pb = np * width;
    for (int k = 0; k < 4; ++k) archive[4 + k] = uint8_t(pb >> (8 * k));
    uint64_t qb;
    memcpy(&qb, &quantum, 8);
    for (int k = 0; k < 8; ++k) archive[8 + k] = uint8_t(qb >> (8 * k));
    for (int k = 0; k < 8; ++k) archive[16 + k] = uint8_t(wb >> (8 * k));
    for (int k = 0; k < 4; ++k) archive[24 + k] = uint8_t(np >> (8 * k));
    for (int k = 0; k < 4; ++k) archive[28 + k] = uint8_t(nq >> (8 * k));
    // zero padding: after WZP, after each section
    for (uint64_t p = 32 + wb; p < pi; ++p) archive[p] = 0;
    for (uint64_t p = pi + uint64_t(np) * 4; p < pv; ++p) archive[p] = 0;
    for (uint64_t p = pv + uint64_t(np) * width; p < qi; ++p) archive[p] = 0;
    for (uint64_t p = qi + uint64_t(nq) * 4; p < qv; ++p) archive[p] = 0;
    for (uint64_t p = qv + uint64_t(nq) * 4; p < end; ++p) archive[p] = 0;
}

// ------------------------------------------------------------ decode patches
// Validates ascending/in-range indices (flags unordered lists for an exact
// duplicate check) and patches q-outliers: coeff = +-T(v) * q with the sign of
// the clamped value already in place. Grid-stride over the archive's count,
// which a graph-replayed launch reads from device memory.
template <class T> struct QPatchOp {
    static constexpr int kThreads = 256, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        JobRef job;
        uint64_t n;
        T* coeff;
        uint32_t* status;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t blocks);
};

template <class T>
__device__ __forceinline__ void QPatchOp<T>::run(const Params P, uint32_t block, uint32_t blocks) {
    const uint64_t n = P.n;
    T* const coeff = P.coeff;
    uint32_t* const status = P.status;
    const DecodeJob J = P.job.get();
    const uint8_t *qi = J.base + J.qi, *qv = J.base + J.qv;
    const bool aligned = (reinterpret_cast<uintptr_t>(J.base) & 7u) == 0; // sections on 8-byte offsets
    const T q = T(J.q);
    for (uint32_t i = block * kThreads + threadIdx.x; i < J.nq; i += blocks * kThreads) {
        uint32_t at, v, prev = 0;
        if (aligned) {
            at = reinterpret_cast<const uint32_t*>(qi)[i];
            v = reinterpret_cast<const uint32_t*>(qv)[i];
            if (i) prev = reinterpret_cast<const uint32_t*>(qi)[i - 1];
        } else {
            memcpy(&at, qi + 4 * uint64_t(i), 4);
            memcpy(&v, qv + 4 * uint64_t(i), 4);
            if (i) memcpy(&prev, qi + 4 * uint64_t(i - 1), 4);
        }
        if (at >= n) { atomicOr(status, ST_BAD_INDEX); continue; }
        if (i && prev >= at) atomicOr(status, ST_UNORDERED);
        if (v <= 65535u || v > 0x7fffffffu) { atomicOr(status, ST_BAD_QOUT); continue; }
        const T x = Lift<T>::mul(T(v), q);
        coeff[at] = coeff[at] < T(0) ? -x : x;
    }
}

// Repair patch targets: a row-major output, a strided box at the job
// table's output address, or a tile clipped into a frame.
template <class T> struct RowPatch {
    T* out;
    __device__ __forceinline__ T* at(uint32_t i) const { return out + i; }
};
template <class T> struct JobPatch {
    const DecodeJob* job;
    uint32_t nx, ny;
    size_t sy, sz;
    __device__ __forceinline__ T* at(uint32_t i) const {
        const uint32_t x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
        return static_cast<T*>(job->out) + size_t(z) * sz + size_t(y) * sy + x;
    }
};

// Repair records: validate, then out[i] -= err (after synthesis).
template <class T, class Patch> struct RPatchOp {
    static constexpr int kThreads = 256, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        JobRef job;
        uint64_t n;
        Patch patch;
        uint32_t* status;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t blocks);
};

template <class T, class Patch>
__device__ __forceinline__ void RPatchOp<T, Patch>::run(const Params P, uint32_t block, uint32_t blocks) {
    const uint64_t n = P.n;
    const Patch patch = P.patch;
    uint32_t* const status = P.status;
    const DecodeJob J = P.job.get();
    const uint8_t *pi = J.base + J.pi, *pv = J.base + J.pv;
    const bool aligned = (reinterpret_cast<uintptr_t>(J.base) & 7u) == 0; // sections on 8-byte offsets
    for (uint32_t i = block * kThreads + threadIdx.x; i < J.np; i += blocks * kThreads) {
        uint32_t at, prev = 0;
        T err;
        if (aligned) {
            at = reinterpret_cast<const uint32_t*>(pi)[i];
            if (!J.compact) err = reinterpret_cast<const T*>(pv)[i];
            if (i) prev = reinterpret_cast<const uint32_t*>(pi)[i - 1];
        } else {
            memcpy(&at, pi + 4 * uint64_t(i), 4);
            if (!J.compact) memcpy(&err, pv + sizeof(T) * uint64_t(i), sizeof(T));
            if (i) memcpy(&prev, pi + 4 * uint64_t(i - 1), 4);
        }
        // compact section: the record's correction from its group (validated
        // header, directory entry and span; never a trap)
        if (J.compact && !wpw_correction<T>(pv, J.pwe_bytes, J.np, i, err)) {
            atomicOr(status, ST_BAD_REPAIR);
            continue;
        }
        if (at >= n) { atomicOr(status, ST_BAD_INDEX); continue; }
        if (i && prev >= at) atomicOr(status, ST_UNORDERED);
        if (!finite_bits(err)) { atomicOr(status, ST_BAD_REPAIR); continue; }
        T* p = patch.at(at);
        if (!p) continue;
        const T r = Lift<T>::sub(*p, err);
        *p = r;
        if (!finite_bits(r)) atomicOr(status, ST_NONFINITE_INPUT);
    }
}

// Exact duplicate test of an unordered index list (test-and-set bitmap).
__global__ void duplicate_kernel(const uint8_t* idx, uint32_t count, uint32_t* seen, uint32_t* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint32_t at;
    memcpy(&at, idx + 4 * uint64_t(i), 4);
    const uint32_t old = atomicOr(&seen[at >> 5], 1u << (at & 31));
    if (old & (1u << (at & 31))) atomicOr(status, ST_BAD_INDEX);
}

// ------------------------------------------------------------------ extrema
// Min/max through order-preserving integer keys (sign-magnitude -> two's
// complement style flip), one atomic pair per CTA.
__device__ __forceinline__ unsigned long long order_key(double v) {
    const unsigned long long b = __double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double key_value(unsigned long long k) {
    const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double(b);
}

template <class T>
__global__ void extrema_kernel(const T* in, uint64_t n, unsigned long long* keys) {
    double lo = 1.0 / 0.0, hi = -1.0 / 0.0;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const double v = double(in[i]);
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
    for (int d = 16; d; d >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, d));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, d));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&keys[0], order_key(lo));
        atomicMax(&keys[1], order_key(hi));
    }
}

} // namespace wb

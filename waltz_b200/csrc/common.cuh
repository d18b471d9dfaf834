// Shared device/host helpers of the Waltz B200 codec.
//
// Arithmetic profile: every lifting step is one explicit correctly-rounded
// fused multiply-add of a plain rounded sum (the reference profile of
// cpu/src/transform.cpp:114-147), written with the __f*_rn intrinsics so that
// no compiler contraction can change a bit. The library is also built with
// --fmad=false and without fast-math or flush-to-zero.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <atomic>
#include <stdexcept>
#include <string>

namespace wb {

// ------------------------------------------------------------ instruments
// Every kernel launch of the library bumps this counter (bench evidence of
// the GPU path); stage events are recorded only while profiling is enabled.
inline std::atomic<unsigned long long>& launch_counter() {
    static std::atomic<unsigned long long> c{0};
    return c;
}
inline void note_launch() { launch_counter().fetch_add(1, std::memory_order_relaxed); }
// Batch graphs captured and instantiated (a replayed graph does not count).
inline std::atomic<unsigned long long>& graph_counter() {
    static std::atomic<unsigned long long> c{0};
    return c;
}

struct StageClock {
    static constexpr int kMax = 16;
    bool enabled = false;
    int count = 0;
    const char* names[kMax] = {};
    cudaEvent_t ev[kMax + 1] = {};
    int device = -1;
    void begin(cudaStream_t s) {
        if (!enabled) return;
        int dev = 0;
        cudaGetDevice(&dev);
        if (device != dev) {
            for (auto& e : ev) cudaEventCreate(&e);
            device = dev;
        }
        count = 0;
        cudaEventRecord(ev[0], s);
    }
    // marks the end of stage `name` (started at the previous mark)
    void mark(const char* name, cudaStream_t s) {
        if (!enabled || count >= kMax) return;
        names[count] = name;
        cudaEventRecord(ev[++count], s);
    }
    int read(double* ms, int cap) const {
        int n = 0;
        for (int i = 0; i < count && i < cap; ++i, ++n) {
            float t = 0;
            cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
            ms[i] = t;
        }
        return n;
    }
};
inline StageClock& stage_clock() {
    static thread_local StageClock c;
    return c;
}

// ------------------------------------------------------------------ errors
struct Error : std::runtime_error {
    explicit Error(const std::string& s) : std::runtime_error(s) {}
};
inline void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(std::string(what) + ": " + cudaGetErrorString(e));
}
inline void need(bool ok, const char* msg) {
    if (!ok) throw Error(msg);
}

// Device status word bits (read back once per call at the existing sync point).
enum Status : uint32_t {
    ST_NONFINITE_INPUT = 1u << 0,   // input or reconstruction not finite
    ST_QUANT_DOMAIN = 1u << 1,      // |coefficient/q| >= 2^63 or not finite
    ST_BOUND = 1u << 2,             // repaired value fails the strict bound
    ST_LOOKBACK_TIMEOUT = 1u << 3,  // a decoupled-lookback wait hit its cap
    ST_CAPACITY = 1u << 4,          // archive section would exceed capacity
    ST_BAD_STREAM = 1u << 5,        // malformed WZP chunk (decode)
    ST_BAD_INDEX = 1u << 6,         // side-record index out of range / duplicate
    ST_UNORDERED = 1u << 7,         // side records not strictly ascending (needs dup check)
    ST_BAD_QOUT = 1u << 8,          // q-outlier value outside (65535, INT32_MAX]
    ST_BAD_REPAIR = 1u << 9,        // nonfinite repair value
    ST_DIRECTORY = 1u << 10,        // WZP directory not in canonical order
    ST_WAIT_TIMEOUT = 1u << 11,     // a bounded wait for an asynchronous copy expired
    ST_MATRIX_RANGE = 1u << 12,     // precision form: a double sample beyond the float range
};

// ------------------------------------------------------------ geometry
struct Dims {
    uint32_t x, y, z;
};

__host__ __device__ inline uint32_t half_len(uint32_t n) { return n - n / 2; }

// Whole-sample symmetric reflection into [0,n), period 2n-2.
__host__ __device__ inline uint32_t mirror(int64_t p, uint32_t n) {
    if (n <= 1) return 0;
    if (p >= 0 && p < (int64_t)n) return (uint32_t)p;
    // one reflection at either end covers every halo of an array longer
    // than the halo; the general periodic form is the fallback
    const int64_t once = p < 0 ? -p : 2 * (int64_t)n - 2 - p;
    if (once >= 0 && once < (int64_t)n) return (uint32_t)once;
    const int64_t period = 2 * (int64_t)n - 2;
    int64_t r = p % period;
    if (r < 0) r += period;
    return (uint32_t)(r < (int64_t)n ? r : period - r);
}
// Split-band address of a reflected spatial position (low half = evens).
__host__ __device__ inline uint32_t split_of(uint32_t r, uint32_t n) {
    return (r >> 1) + ((r & 1) ? half_len(n) : 0);
}
__host__ __device__ inline uint32_t coeff_at(int64_t p, uint32_t n) { return split_of(mirror(p, n), n); }

inline unsigned levels_of(uint32_t length) {
    unsigned l = 0;
    while (length > 8 && l < 5) { length -= length / 2; ++l; }
    return l;
}

// Morton z-band height (include/lossless/reorder.hpp:130-144).
inline unsigned zband_of(uint32_t nx, uint32_t ny, uint32_t nz, unsigned lz, bool dyadic) {
    if (dyadic) {
        const uint32_t b = (nz + ((1u << lz) - 1)) >> lz;
        return b > 16 ? 16 : (b < 1 ? 1 : b);
    }
    if (nz < 4) return nz;
    const uint64_t bricks = uint64_t((nx + 15) / 16) * ((ny + 15) / 16);
    const uint64_t full = uint64_t(nx / 16) * (ny / 16);
    return (bricks - full) * 32 >= bricks ? 4 : 2;
}

// ------------------------------------------------------------ lifting math
template <class T> struct Lift;
template <> struct Lift<float> {
    static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
};
template <> struct Lift<double> {
    static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
};

// CDF 9/7 lifting constants cast to T (cpu/src/transform.cpp:41-48).
template <class T> struct K97 {
    static constexpr T a = T(-1.586134342059924);
    static constexpr T b = T(-0.052980118572961);
    static constexpr T g = T(0.882911075530934);
    static constexpr T d = T(0.443506852043971);
    static constexpr T k = T(1.1496043988602418);
    static constexpr T ik = T(1) / T(1.1496043988602418);
};

// One halo window of P even/odd pairs (samples start-4 .. start+2P-5).
// Forward: restricted four-step analysis then scaling of the interior.
// Inverse: scaling of everything, then the four synthesis steps with the
// window's two endpoint normalisations folded into one FMA when Folded.
template <class T, int P>
__device__ __forceinline__ void lift_forward(T (&e)[P], T (&o)[P]) {
    using L = Lift<T>;
#pragma unroll
    for (int j = 0; j < P - 1; ++j) o[j] = L::fma(K97<T>::a, L::add(e[j], e[j + 1]), o[j]);
#pragma unroll
    for (int j = 1; j < P - 1; ++j) e[j] = L::fma(K97<T>::b, L::add(o[j - 1], o[j]), e[j]);
#pragma unroll
    for (int j = 1; j < P - 2; ++j) o[j] = L::fma(K97<T>::g, L::add(e[j], e[j + 1]), o[j]);
#pragma unroll
    for (int j = 2; j < P - 2; ++j) e[j] = L::fma(K97<T>::d, L::add(o[j - 1], o[j]), e[j]);
#pragma unroll
    for (int j = 2; j < P - 2; ++j) {
        e[j] = L::mul(e[j], K97<T>::k);
        o[j] = L::mul(o[j], -K97<T>::ik);
    }
}

template <class T, int P, bool Folded>
__device__ __forceinline__ void lift_inverse(T (&e)[P], T (&o)[P]) {
    using L = Lift<T>;
    const T raw_first = o[0], raw_last = o[P - 1];
#pragma unroll
    for (int j = 0; j < P; ++j) {
        e[j] = L::mul(e[j], K97<T>::ik);
        o[j] = L::mul(o[j], -K97<T>::k);
    }
#pragma unroll
    for (int j = 1; j < P; ++j) {
        T s;
        if (Folded && j == 1) s = L::fma(raw_first, -K97<T>::k, o[1]);
        else if (Folded && j == P - 1) s = L::fma(raw_last, -K97<T>::k, o[P - 2]);
        else s = L::add(o[j - 1], o[j]);
        e[j] = L::fma(-K97<T>::d, s, e[j]);
    }
#pragma unroll
    for (int j = 1; j < P - 1; ++j) o[j] = L::fma(-K97<T>::g, L::add(e[j], e[j + 1]), o[j]);
#pragma unroll
    for (int j = 2; j < P - 1; ++j) e[j] = L::fma(-K97<T>::b, L::add(o[j - 1], o[j]), e[j]);
#pragma unroll
    for (int j = 2; j < P - 2; ++j) o[j] = L::fma(-K97<T>::a, L::add(e[j], e[j + 1]), o[j]);
}

// Finite (neither NaN nor infinite): the magnitude compares at most the
// largest finite value, one compare (a NaN compares false).
template <class T> __device__ __forceinline__ bool finite_bits(T v);
template <> __device__ __forceinline__ bool finite_bits<float>(float v) { return fabsf(v) <= 3.40282346638528859812e+38f; }
template <> __device__ __forceinline__ bool finite_bits<double>(double v) {
    return fabs(v) <= 1.79769313486231570815e+308;
}

// |value - original| <= bound on the exact difference: the double difference
// plus its rounding error (two-difference) settles the tie case
// (cpu/src/repair_avx2.cpp:48-55).
__device__ __forceinline__ bool strictly_within(double value, double original, double bound) {
    const double diff = __dsub_rn(value, original);
    const double m = fabs(diff);
    if (!finite_bits(diff) || m > bound) return false;
    if (m < bound) return true;
    const double vpart = __dsub_rn(value, diff);
    const double opart = __dadd_rn(diff, vpart);
    const double err = __dadd_rn(__dsub_rn(value, opart), __dsub_rn(vpart, original));
    return !((diff > 0 && err > 0) || (diff < 0 && err < 0));
}

__host__ __device__ inline size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }

constexpr uint32_t kChunk = 8192;     // magnitudes per WZP chunk
constexpr uint32_t kGroup = 16;       // chunks per directory group
constexpr uint32_t kRawCode = 0x3fff; // metadata code of a verbatim chunk

__host__ __device__ inline uint32_t wzp_chunks(uint32_t n) { return n ? 1 + (n - 1) / kChunk : 0; }
__host__ __device__ inline uint32_t wzp_groups(uint32_t n) { return (wzp_chunks(n) + kGroup - 1) / kGroup; }
__host__ __device__ inline size_t wzp_header(uint32_t n) {
    return size_t(wzp_groups(n)) * 4 + size_t(wzp_chunks(n)) * 3;
}
__host__ __device__ inline size_t wzp_max_bytes(uint32_t n) {
    return wzp_header(n) + size_t(n) * 2 + (size_t(n) + 7) / 8;
}

// Where one archive's sections lie, as the host validated them from its
// 32-byte header: base, WZP stream length, section offsets from the base,
// quantum and side-record counts.
struct DecodeJob {
    const uint8_t* base;
    uint64_t wzp, pi, pv, qi, qv;
    double q;
    uint32_t np, nq;
    void* out; // where the samples go (read by JobOut / JobPatch)
    uint32_t pwe_bytes; // repair section bytes
    uint32_t compact;   // the repair section is a compact (WPW1) section
};

// A decode kernel's archive parameters: by value (one archive decoded by
// direct launches), or in device memory (a captured decode graph replayed
// over other archives of the same shapes, parameters rewritten each time).
struct JobRef {
    const DecodeJob* ptr;
    DecodeJob val;
    __device__ __forceinline__ DecodeJob get() const { return ptr ? *ptr : val; }
};

} // namespace wb

// Batched device decode of many same-shaped tile archives into one frame
// tensor (the DataLoader back end): waltz_gpu_decode_batch, with the exact
// signature, validation rules and scratch contract of the reference
// (src/batch_decode.cuh:74-186). Everything runs in the caller's scratch on
// the caller's stream; nothing is allocated.
#pragma once

namespace wb {

// A tile's samples clipped into its place inside the (z, y, x) frame.
template <class T> struct FrameOut {
    static constexpr bool kPrefetch = false;
    T* dst;                 // frame base of this job's (side, sample)
    uint32_t fx, fy, fz;    // frame dims
    uint32_t ox, oy, oz;    // tile origin inside the frame
    uint32_t* status;
    __device__ __forceinline__ void operator()(uint32_t x, uint32_t y, uint32_t z, T v) const {
        const uint32_t gx = ox + x, gy = oy + y, gz = oz + z;
        if (gx < fx && gy < fy && gz < fz) {
            dst[(size_t(gz) * fy + gy) * fx + gx] = v;
            if (!finite_bits(v)) atomicOr(status, ST_NONFINITE_INPUT);
        }
    }
};

template <class T> struct FramePatch {
    T* dst;
    uint32_t tx, ty;        // tile dims (x, y)
    uint32_t fx, fy, fz;
    uint32_t ox, oy, oz;
    __device__ __forceinline__ T* at(uint32_t i) const {
        const uint32_t x = i % tx, y = (i / tx) % ty, z = i / (tx * ty);
        const uint32_t gx = ox + x, gy = oy + y, gz = oz + z;
        if (gx >= fx || gy >= fy || gz >= fz) return nullptr;
        return dst + (size_t(gz) * fy + gy) * fx + gx;
    }
};

template <class T>
__global__ void fill_tile_kernel(T* dst, uint32_t fx, uint32_t fy, uint32_t fz, uint32_t ox, uint32_t oy, uint32_t oz,
                                 uint32_t tx, uint32_t ty, uint32_t tz, T value) {
    const uint64_t n = uint64_t(tx) * ty * tz;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t x = uint32_t(i % tx), y = uint32_t((i / tx) % ty), z = uint32_t(i / (uint64_t(tx) * ty));
        const uint32_t gx = ox + x, gy = oy + y, gz = oz + z;
        if (gx < fx && gy < fy && gz < fz) dst[(size_t(gz) * fy + gy) * fx + gx] = value;
    }
}

static inline unsigned divup(unsigned n, unsigned k) { return 1 + (n - 1) / k; }

template <class T>
static void decode_batch(const waltz_batch_shape& d, const uint8_t* host, const uint8_t* packed, size_t bytes,
                         uint8_t* scratch, size_t cap, T* output, size_t outbytes, double fill, cudaStream_t stream) {
    need(d.x && d.y && d.z && d.fx && d.fy && d.fz && d.samples && (d.sides == 1 || d.sides == 2),
         "invalid batch geometry");
    const Dims grid{divup(d.fx, d.x), divup(d.fy, d.y), divup(d.fz, d.z)};
    const uint64_t n64 = uint64_t(d.x) * d.y * d.z;
    const uint64_t jobs64 = uint64_t(grid.x) * grid.y * grid.z * uint64_t(d.samples) * d.sides;
    need(n64 <= 0x7fffffffull / sizeof(T) && jobs64 <= 65535 && d.y <= 65535 && d.z <= 65535, "batch launch limit");
    const uint64_t frame = uint64_t(d.fx) * d.fy * d.fz;
    need(outbytes == frame * d.samples * d.sides * sizeof(T), "incorrect output size");
    const uint64_t stride = (n64 + 3) & ~uint64_t(3), bank = stride * jobs64;
    const Geometry g = Geometry::make(d.x, d.y, d.z);
    need(cap >= 3 * bank * sizeof(T) + 8ull * 256 * g.bz * 4 + 4 && bytes >= 16 * jobs64, "short batch buffers");
    const uint64_t table = bytes - 16 * jobs64;
    need(!(table % 16), "unaligned batch spans");
    struct Job {
        uint64_t at, size;
        Header h;
        Layout L;
    };
    std::vector<Job> list(jobs64);
    for (uint64_t j = 0; j < jobs64; ++j) {
        uint64_t pair[2];
        std::memcpy(pair, host + table + 16 * j, 16);
        Job& job = list[j];
        job.at = pair[0];
        job.size = pair[1];
        if (!job.size) continue;
        need(!(job.at % 16) && job.at <= table && job.size >= 32 && job.size <= table - job.at, "invalid batch span");
        job.h = Header::parse(host + job.at);
        try {
            job.L = validate_header<T>(job.h, g, job.size, true);
        } catch (const std::exception&) {
            throw Error("invalid canonical batch archive");
        }
    }
    // Scratch carve: three banks (only one job's worth is live at a time),
    // the inverse Morton table and the status word.
    T* C = reinterpret_cast<T*>(scratch);
    T* bank1 = C + bank;
    T* bank2 = bank1 + bank;
    uint16_t* irank = reinterpret_cast<uint16_t*>(bank2 + bank);
    uint32_t* status = reinterpret_cast<uint32_t*>(irank + 8ull * 256 * g.bz);
    {
        const auto tab = morton_tables(d.x, d.y, d.z, g.bz, true);
        check(cudaMemcpyAsync(irank, tab.data(), tab.size() * 2, cudaMemcpyHostToDevice, stream), "table upload");
    }
    check(cudaMemsetAsync(status, 0, 4, stream), "memset");
    Sink sink{stream};
    for (uint64_t j = 0; j < jobs64; ++j) {
        uint64_t r = j;
        const uint32_t ox = uint32_t(r % grid.x) * d.x;
        r /= grid.x;
        const uint32_t oy = uint32_t(r % grid.y) * d.y;
        r /= grid.y;
        const uint32_t oz = uint32_t(r % grid.z) * d.z;
        r /= grid.z;
        T* dst = output + ((r % d.sides) * uint64_t(d.samples) + r / d.sides) * frame;
        const Job& job = list[j];
        if (!job.size) {
            fill_tile_kernel<T><<<grid_for(n64), 256, 0, stream>>>(dst, d.fx, d.fy, d.fz, ox, oy, oz, d.x, d.y, d.z,
                                                                   T(fill)); note_launch();
            continue;
        }
        FrameOut<T> fin{dst, d.fx, d.fy, d.fz, ox, oy, oz, status};
        FramePatch<T> patch{dst, d.x, d.y, d.fx, d.fy, d.fz, ox, oy, oz};
        decode_launch<T>(JobRef{nullptr, decode_job(packed + job.at, job.h, job.L)}, job.h.split,
                         g, irank, nullptr, C, bank1, bank2, fin, patch, status, sink);
    }
    check(cudaGetLastError(), "batch launch");
    uint32_t word = 0;
    check(cudaMemcpyAsync(&word, status, 4, cudaMemcpyDeviceToHost, stream), "readback");
    check(cudaStreamSynchronize(stream), "batch decode");
    if (word & ST_DIRECTORY) {
        // Non-canonical group order: exact check on the host copy.
        for (const Job& job : list)
            if (job.size) {
                const uint64_t header = wzp_header(uint32_t(n64));
                host_directory_check(host + job.at + 32, uint32_t(n64), job.h.wzp - header);
            }
        word &= ~ST_DIRECTORY;
    }
    if (word & (ST_UNORDERED | ST_BAD_INDEX)) throw Error("invalid batch repair index");
    if (word & ST_BAD_STREAM) throw Error("malformed WZP stream");
    if (word & ST_BAD_QOUT) throw Error("invalid quantization outlier");
    if (word & ST_BAD_REPAIR) throw Error("nonfinite correction");
    if (word & ST_NONFINITE_INPUT) throw Error("nonfinite reconstruction");
    if (word & ST_WAIT_TIMEOUT) throw Error("Waltz: asynchronous copy wait exceeded its bound");
}

} // namespace wb

extern "C" const char* waltz_gpu_decode_batch(const waltz_batch_shape* d, const void* host, const void* packed,
                                              size_t bytes, void* scratch, size_t cap, void* out, size_t outbytes,
                                              double fill, void* raw_stream) {
    using namespace wb;
    static thread_local char err[256];
    try {
        need(d && host && packed && scratch && out && (d->width == 4 || d->width == 8), "invalid batch arguments");
        auto s = reinterpret_cast<cudaStream_t>(raw_stream);
        auto* h = static_cast<const uint8_t*>(host);
        auto* p = static_cast<const uint8_t*>(packed);
        auto* sc = static_cast<uint8_t*>(scratch);
        if (d->width == 4) decode_batch(*d, h, p, bytes, sc, cap, static_cast<float*>(out), outbytes, fill, s);
        else decode_batch(*d, h, p, bytes, sc, cap, static_cast<double*>(out), outbytes, fill, s);
        return nullptr;
    } catch (const std::exception& e) {
        std::snprintf(err, sizeof(err), "%s", e.what());
        return err;
    }
}

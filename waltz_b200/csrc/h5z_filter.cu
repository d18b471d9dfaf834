// HDF5 filter 61197 ("Waltz canonical") backed by the GPU codec: the
// counterpart of the reference's CPU plugin (python/hdf5/filter.cpp:16-58 of
// the reference project), with the same client data and the same chunk
// archives, so files written by either plugin are read by the other.
//
// Client data (6 unsigned values, set by pywaltz.hdf5.create_dataset):
//   cd[0..2] chunk extents nx, ny, nz (x fastest; (y,x) chunks have nz = 1)
//   cd[3]    sample width in bytes, 4 (float) or 8 (double)
//   cd[4..5] the absolute bound as a little-endian double, low word first
// Forward: buffer holds nx*ny*nz samples; it is replaced by the archive.
// Reverse (flags & H5Z_FLAG_REVERSE): buffer holds an archive; it is
// replaced by the samples. On any failure the filter returns 0 and leaves
// *buffer and *buffer_size untouched, as H5Z requires.
//
// The chunk runs on the calling thread's current CUDA device, through
// per-thread device buffers that grow to the largest chunk seen (released
// at thread exit). The plugin needs no HDF5 headers: the two entry points
// HDF5 looks up in a plugin library and the filter class record are
// declared below with the layout of HDF5's public H5PLextern.h / H5Zpublic.h
// (H5Z_class2_t, H5Z_CLASS_T_VERS = 1, H5PL_TYPE_FILTER = 0,
// H5Z_FLAG_REVERSE = 0x0100).
#include "../../include/waltz_b200.h"
#include "../../include/waltz_h5z.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>

namespace {

constexpr int kFilterId = 61197;
constexpr unsigned kFlagReverse = 0x0100u;

using can_apply_fn = int (*)(long long, long long, long long);
using set_local_fn = int (*)(long long, long long, long long);
using filter_fn = size_t (*)(unsigned, size_t, const unsigned[], size_t, size_t*, void**);

struct FilterClass {  // H5Z_class2_t
    int version;
    int id;
    unsigned encoder_present;
    unsigned decoder_present;
    const char* name;
    can_apply_fn can_apply;
    set_local_fn set_local;
    filter_fn filter;
};

static_assert(sizeof(unsigned) == 4 && sizeof(double) == 8 && std::numeric_limits<double>::is_iec559,
              "the client data packs a double into two 32-bit words");

// Per-thread device buffers: samples and archive of the largest chunk seen.
struct Buffers {
    int device = -1;
    void* samples = nullptr;
    void* archive = nullptr;
    size_t samples_cap = 0, archive_cap = 0;
    cudaStream_t stream = nullptr;

    ~Buffers() { release(); }
    void release() {
        if (device >= 0) {
            int prev = 0;
            if (cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(device) == cudaSuccess) {
                cudaFree(samples);
                cudaFree(archive);
                if (stream) cudaStreamDestroy(stream);
                cudaSetDevice(prev);
            }
        }
        samples = archive = nullptr;
        samples_cap = archive_cap = 0;
        stream = nullptr;
        device = -1;
    }
    bool reserve(size_t samples_bytes, size_t archive_bytes) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return false;
        if (dev != device) {
            release();
            device = dev;
            if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
                stream = nullptr;
                return false;
            }
        }
        if (samples_bytes > samples_cap) {
            cudaFree(samples);
            samples = nullptr;
            samples_cap = 0;
            if (cudaMalloc(&samples, samples_bytes) != cudaSuccess) return false;
            samples_cap = samples_bytes;
        }
        if (archive_bytes > archive_cap) {
            cudaFree(archive);
            archive = nullptr;
            archive_cap = 0;
            if (cudaMalloc(&archive, archive_bytes) != cudaSuccess) return false;
            archive_cap = archive_bytes;
        }
        return true;
    }
};
thread_local Buffers t_buffers;

} // namespace

// The filter callback (declared in include/waltz_h5z.h), also the class
// record's `filter`.
extern "C" size_t waltz_b200_h5z_filter(unsigned flags, size_t count, const unsigned cd[], size_t bytes,
                                        size_t* buffer_size, void** buffer) {
    const uint16_t one = 1;
    if (*reinterpret_cast<const uint8_t*>(&one) != 1 || count != 6 || !cd || !buffer || !*buffer ||
        !buffer_size || !bytes || bytes > *buffer_size || (cd[3] != 4 && cd[3] != 8))
        return 0;
    const uint32_t nx = cd[0], ny = cd[1], nz = cd[2];
    const int width = int(cd[3]);
    if (!nx || !ny || !nz || uint64_t(nx) * ny > 0xffffffffull / unsigned(width) / nz) return 0;
    const uint64_t bits = uint64_t(cd[4]) | (uint64_t(cd[5]) << 32);
    double bound;
    std::memcpy(&bound, &bits, sizeof(bound));
    const uint64_t n = uint64_t(nx) * ny * nz;
    const size_t raw = size_t(n) * unsigned(width);
    const size_t max_archive = waltz_b200_compressed_capacity(n, width);
    if (!max_archive) return 0;
    const bool decode = (flags & kFlagReverse) != 0;
    if (decode ? (bytes < 32 || bytes > max_archive) : (bytes != raw || !(bound > 0) || !(bound < 1e300)))
        return 0;

    Buffers& b = t_buffers;
    if (!b.reserve(raw, max_archive)) return 0;
    size_t written = raw;
    void* out = nullptr;
    if (decode) {
        out = std::malloc(raw);
        if (!out) return 0;
        if (cudaMemcpyAsync(b.archive, *buffer, bytes, cudaMemcpyHostToDevice, b.stream) != cudaSuccess ||
            waltz_b200_decompress(b.archive, bytes, width, nx, ny, nz, b.samples, raw, b.stream) != 0 ||
            cudaMemcpyAsync(out, b.samples, raw, cudaMemcpyDeviceToHost, b.stream) != cudaSuccess ||
            cudaStreamSynchronize(b.stream) != cudaSuccess) {
            std::free(out);
            return 0;
        }
    } else {
        if (cudaMemcpyAsync(b.samples, *buffer, raw, cudaMemcpyHostToDevice, b.stream) != cudaSuccess ||
            waltz_b200_compress(b.samples, width, nx, ny, nz, bound, b.archive, max_archive, &written, b.stream) != 0)
            return 0;
        out = std::malloc(written);
        if (!out) return 0;
        if (cudaMemcpyAsync(out, b.archive, written, cudaMemcpyDeviceToHost, b.stream) != cudaSuccess ||
            cudaStreamSynchronize(b.stream) != cudaSuccess) {
            std::free(out);
            return 0;
        }
    }
    std::free(*buffer);
    *buffer = out;
    *buffer_size = written;
    return written;
}

namespace {
const FilterClass kClass{1, kFilterId, 1, 1, "Waltz canonical (B200 GPU)", nullptr, nullptr, waltz_b200_h5z_filter};
} // namespace

extern "C" {
// H5PL_type_t H5PLget_plugin_type(void): H5PL_TYPE_FILTER.
int H5PLget_plugin_type(void) { return 0; }
// const void* H5PLget_plugin_info(void): the filter class record.
const void* H5PLget_plugin_info(void) { return &kClass; }
}

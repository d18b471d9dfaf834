// The reference's C++ device API (include/waltz.hpp:35-46 of the reference
// project) over this library's C ABI, exported with the reference's mangled
// names so that programs built against either header link here unchanged.
//
// Each entry checks the arguments the reference checks before any device
// work (src/waltz.cu:327-349: dimensions, null buffers, overlap, bound) and
// throws std::invalid_argument for them; a failure of the codec itself
// (archive checks, device errors) is thrown as std::runtime_error with the C
// ABI's diagnostic.
#include "../../include/waltz.hpp"
#include "../../include/waltz_b200.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace WALTZ {
namespace {

void fail_runtime(const char* what) {
    throw std::runtime_error(std::string(what) + ": " + waltz_b200_last_error());
}

// The three extents as the C ABI takes them; the reference's checks on
// Config (src/waltz.cu:337-342): nonzero extents whose product equals num
// and fits the archive's 32-bit sample indices.
template <typename T> void extents(const Config& c, uint32_t& nx, uint32_t& ny, uint32_t& nz) {
    const uint64_t limit = 0xffffffffull / sizeof(T);
    if (!c.dimx || !c.dimy || !c.dimz || c.dimx > limit || c.dimy > limit / c.dimx ||
        c.dimz > limit / (c.dimx * c.dimy) || c.num != c.dimx * c.dimy * c.dimz)
        throw std::invalid_argument("Waltz: invalid buffers or shape for WZP");
    nx = uint32_t(c.dimx);
    ny = uint32_t(c.dimy);
    nz = uint32_t(c.dimz);
}

} // namespace

void calculate_dwt_levels(dim3 d, uint8_t& levels_xy, uint8_t& levels_z) {
    auto levels = [](uint32_t n) {
        uint8_t l = 0;
        for (; n > 8 && l < 5; ++l) n -= n / 2;
        return l;
    };
    levels_xy = levels(d.x < d.y ? d.x : d.y);
    levels_z = levels(d.z);
}

template <typename T, int NDIMS>
size_t d_WALTZ_compress(T* d_oridata, char* d_cmpData, const Config& config, const char* /*cmpPath*/,
                        void* stream) {
    static_assert(NDIMS == 3, "the archive codec is three-dimensional");
    uint32_t nx, ny, nz;
    extents<T>(config, nx, ny, nz);
    if (!d_oridata || !d_cmpData) throw std::invalid_argument("Waltz: invalid buffers or shape for WZP");
    const size_t capacity = compressed_buffer_capacity<T>(config.num);
    const uintptr_t a = reinterpret_cast<uintptr_t>(d_oridata), b = reinterpret_cast<uintptr_t>(d_cmpData);
    if (a <= b ? b - a < config.num * sizeof(T) : a - b < capacity)
        throw std::invalid_argument("Waltz: input and output buffers overlap");
    const double eb = config.absErrorBound;
    if (!(eb > 0) || !std::isfinite(1.5 * eb)) throw std::invalid_argument("Waltz: invalid bound or rounding mode");
    // the reference's compact repair profile switch (src/waltz.cu:162-172):
    // WALTZ_SMALL_PWE_SCALE = 0 (default), 16 or 64, for this call
    int scale = 0;
    if (const char* v = std::getenv("WALTZ_SMALL_PWE_SCALE")) {
        char* end = nullptr;
        const double d = std::strtod(v, &end);
        if (end == v || *end != '\0' || (d != 0.0 && d != 16.0 && d != 64.0))
            throw std::invalid_argument("Waltz: WALTZ_SMALL_PWE_SCALE must be 0, 16 or 64");
        scale = int(d);
    }
    waltz_b200_set_option(WALTZ_B200_OPT_COMPACT_REPAIRS, scale);
    size_t written = 0;
    const int rc = waltz_b200_compress(d_oridata, int(sizeof(T)), nx, ny, nz, eb, d_cmpData, capacity, &written, stream);
    waltz_b200_set_option(WALTZ_B200_OPT_COMPACT_REPAIRS, 0);
    if (rc) fail_runtime("Waltz compress");
    return written;
}

template <typename T, int NDIMS>
size_t d_WALTZ_decompress(char* d_cmpData, T* d_decData, const Config& config, const char* decPath, void* stream) {
    static_assert(NDIMS == 3, "the archive codec is three-dimensional");
    uint32_t nx, ny, nz;
    extents<T>(config, nx, ny, nz);
    if (!d_cmpData || !d_decData) throw std::invalid_argument("Waltz: null buffer");
    const size_t out_bytes = size_t(config.num) * sizeof(T);
    // Length 0: the decoder takes the archive's length from its header.
    if (waltz_b200_decompress(d_cmpData, 0, int(sizeof(T)), nx, ny, nz, d_decData, out_bytes, stream))
        fail_runtime("Waltz decompress");
    if (decPath) {
        std::vector<T> host(config.num);
        if (cudaMemcpy(host.data(), d_decData, out_bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("Waltz decompress: reconstruction readback failed");
        if (FILE* f = std::fopen(decPath, "wb")) {
            std::fwrite(host.data(), sizeof(T), host.size(), f);
            std::fclose(f);
        }
    }
    return out_bytes;
}

template <typename T> void d_extrema(T* d_data, uint64_t n, double& out_min, double& out_max, void* stream) {
    if (waltz_b200_extrema(d_data, int(sizeof(T)), n, &out_min, &out_max, stream)) fail_runtime("Waltz extrema");
}

template size_t d_WALTZ_compress<float, 3>(float*, char*, const Config&, const char*, void*);
template size_t d_WALTZ_compress<double, 3>(double*, char*, const Config&, const char*, void*);
template size_t d_WALTZ_decompress<float, 3>(char*, float*, const Config&, const char*, void*);
template size_t d_WALTZ_decompress<double, 3>(char*, double*, const Config&, const char*, void*);
template void d_extrema<float>(float*, uint64_t, double&, double&, void*);
template void d_extrema<double>(double*, uint64_t, double&, double&, void*);

} // namespace WALTZ

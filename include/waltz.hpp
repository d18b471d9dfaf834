/*
 * Waltz B200: the reference's C++ device API, served by libwaltz_b200.so.
 *
 * A program written against the reference's C++ API (include/waltz.hpp:15-81
 * of the reference project) compiles against this header, or against the
 * reference's own header, and links to libwaltz_b200.so unchanged: the
 * library exports the same mangled entry points
 *   WALTZ::d_WALTZ_compress<float|double, 3>   (include/waltz.hpp:35-37)
 *   WALTZ::d_WALTZ_decompress<float|double, 3> (include/waltz.hpp:42-44)
 *   WALTZ::d_extrema<float|double>             (include/waltz.hpp:39-40)
 *   WALTZ::calculate_dwt_levels                (src/waltz.cu:302-305)
 * and reads WALTZ::Config with the reference's member layout
 * (include/utils/Config.hpp:135-215), the one type whose bytes cross the
 * boundary.
 *
 * Conventions are the reference's: device pointers, the stream passed as
 * void*, REL resolved by the caller into Config::absErrorBound (d_extrema
 * gives the range), output capacity >= compressed_buffer_capacity<T>(num),
 * synchronous on return, errors thrown as std::invalid_argument (arguments)
 * or std::runtime_error (archive or device failures). cmpPath is ignored;
 * a non-null decPath receives a host copy of the reconstruction. The
 * archive length is not an argument of the decoder: it follows from the
 * 32-byte header.
 */
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <limits>
#include <stdexcept>

namespace WALTZ {

enum EB { EB_ABS, EB_REL, EB_PSNR, EB_L2NORM, EB_ABS_AND_REL, EB_ABS_OR_REL };

// Field description. Axes of extent <= 1 are dropped (a 1 x 64 x 64 field
// becomes 2-D): the archive codec needs ndims == 3. The member order and
// types are part of the binary interface and must not change.
class Config {
  public:
    Config() : Config(1) {}

    template <class... Dims> Config(Dims... extents) {
        const std::initializer_list<uint64_t> list{static_cast<uint64_t>(extents)...};
        setDims(list.begin(), list.end());
    }

    template <class It> uint64_t setDims(It first, It last) {
        dimx = dimy = dimz = dimw = 1;
        ndims = 0;
        num = 1;
        for (It it = first; it != last; ++it) {
            const uint64_t extent = static_cast<uint64_t>(*it);
            if (extent <= 1) continue;
            if (ndims == 4) throw std::invalid_argument("Config supports at most 4 dimensions");
            if (extent > std::numeric_limits<uint64_t>::max() / num)
                throw std::overflow_error("Config element count exceeds uint64 capacity");
            setDim(ndims++, extent);
            num *= extent;
        }
        if (ndims == 0) ndims = 1;
        return num;
    }

    void setDim(uint8_t axis, uint64_t extent) {
        uint64_t* slot[4] = {&dimx, &dimy, &dimz, &dimw};
        if (axis > 3) throw std::invalid_argument("dimension index out of range");
        *slot[axis] = extent;
    }

    uint8_t ndims;
    uint64_t dimx, dimy, dimz, dimw;
    uint64_t chunkx{256}, chunky{256}, chunkz{256}, chunkw{256};
    uint64_t num;
    uint64_t blockSize = 0;
    uint8_t errorBoundMode = EB_ABS;
    double absErrorBound = 0;
    double relErrorBound = 0;
    double psnrErrorBound = 0;
    double l2normErrorBound = 0;
};

// Archive capacity for num samples of T: one input volume, the fixed caps of
// the repair list (2^22 records) and the q-outlier list (2^20 records), plus
// 1 MiB (include/waltz.hpp:21-33 of the reference).
template <typename T> size_t compressed_buffer_capacity(uint64_t num) {
    const uint64_t repairs = num < (uint64_t(1) << 22) ? num : (uint64_t(1) << 22);
    const uint64_t outliers = num < (uint64_t(1) << 20) ? num : (uint64_t(1) << 20);
    const uint64_t side = repairs * (4 + sizeof(T)) + outliers * 8 + (uint64_t(1) << 20);
    if (num > (std::numeric_limits<size_t>::max() - side) / sizeof(T))
        throw std::overflow_error("Waltz compressed buffer capacity exceeds size_t");
    return static_cast<size_t>(num * sizeof(T) + side);
}

template <typename T, int NDIMS>
size_t d_WALTZ_compress(T* d_oridata, char* d_cmpData, const WALTZ::Config& config, const char* cmpPath,
                        void* stream);

template <typename T>
void d_extrema(T* d_data, uint64_t n, double& out_min, double& out_max, void* stream);

template <typename T, int NDIMS>
size_t d_WALTZ_decompress(char* d_cmpData, T* d_decData, const WALTZ::Config& config, const char* decPath,
                          void* stream);

// Level counts of the archive geometry: halve (ceil) while the extent is
// above 8, at most five times; XY from min(x, y), Z from z.
void calculate_dwt_levels(dim3 data_dims, uint8_t& levels_xy, uint8_t& levels_z);

// Returns the archive length in bytes.
template <typename T>
size_t d_compress(const WALTZ::Config& config, T* d_oridata, char* d_cmpData, const char* cmpPath, void* stream) {
    if (config.ndims != 3) throw std::invalid_argument("compression currently only supports 3D data.");
    return d_WALTZ_compress<T, 3>(d_oridata, d_cmpData, config, cmpPath, stream);
}

// Returns the decoded byte count. config must hold the original dimensions
// (the archive does not store them) and T the archived sample type.
template <typename T>
size_t d_decompress(const WALTZ::Config& config, char* d_cmpData, T* d_decData, const char* decPath, void* stream) {
    if (config.ndims != 3) throw std::invalid_argument("decompression currently only supports 3D data.");
    return d_WALTZ_decompress<T, 3>(d_cmpData, d_decData, config, decPath, stream);
}

} // namespace WALTZ

// A caller written the way a program using the reference's C++ device API
// calls it (include/waltz.hpp:47-81 of the reference project, and its
// examples/waltz.cu:50-80): a Config from the three extents, REL resolved
// through d_extrema, d_compress into a compressed_buffer_capacity<T> buffer,
// then d_decompress with no archive length. It is compiled twice: against
// this repository's include/waltz.hpp and, where the reference tree is
// present, against the reference's own header; both builds link to
// libwaltz_b200.so. The tests drive it through ctypes.
#include "waltz.hpp"

#include <cstddef>
#include <cstdio>
#include <exception>

// Exported by both libraries, declared by no public header of the reference
// (src/waltz.cu:302-305 of the reference project).
namespace WALTZ {
void calculate_dwt_levels(dim3 data_dims, uint8_t& levels_xy, uint8_t& levels_z);
}

namespace {
template <typename T>
int round_trip(T* d_in, unsigned long long nx, unsigned long long ny, unsigned long long nz, double rel,
               double abs_bound, char* d_cmp, T* d_out, void* stream, unsigned long long* archive_bytes,
               double* bound_used, char* err, unsigned long long err_len) {
    try {
        WALTZ::Config conf(nx, ny, nz);
        if (rel > 0) {
            double lo = 0, hi = 0;
            WALTZ::d_extrema<T>(d_in, conf.num, lo, hi, stream);
            conf.absErrorBound = rel * (hi - lo);
        } else {
            conf.absErrorBound = abs_bound;
        }
        *bound_used = conf.absErrorBound;
        *archive_bytes = WALTZ::d_compress<T>(conf, d_in, d_cmp, nullptr, stream);
        const size_t decoded = WALTZ::d_decompress<T>(conf, d_cmp, d_out, nullptr, stream);
        if (decoded != conf.num * sizeof(T)) throw std::runtime_error("unexpected decoded size");
        return 0;
    } catch (const std::invalid_argument& e) {
        std::snprintf(err, err_len, "invalid_argument: %s", e.what());
        return 1;
    } catch (const std::exception& e) {
        std::snprintf(err, err_len, "runtime_error: %s", e.what());
        return 2;
    }
}

template <typename T>
int decode_only(char* d_cmp, unsigned long long nx, unsigned long long ny, unsigned long long nz, T* d_out,
                void* stream, char* err, unsigned long long err_len) {
    try {
        WALTZ::Config conf(nx, ny, nz);
        WALTZ::d_decompress<T>(conf, d_cmp, d_out, nullptr, stream);
        return 0;
    } catch (const std::invalid_argument& e) {
        std::snprintf(err, err_len, "invalid_argument: %s", e.what());
        return 1;
    } catch (const std::exception& e) {
        std::snprintf(err, err_len, "runtime_error: %s", e.what());
        return 2;
    }
}
} // namespace

extern "C" {
int caller_round_trip_f32(float* in, unsigned long long nx, unsigned long long ny, unsigned long long nz, double rel,
                          double abs_bound, char* cmp, float* out, void* stream, unsigned long long* bytes,
                          double* bound, char* err, unsigned long long err_len) {
    return round_trip<float>(in, nx, ny, nz, rel, abs_bound, cmp, out, stream, bytes, bound, err, err_len);
}
int caller_round_trip_f64(double* in, unsigned long long nx, unsigned long long ny, unsigned long long nz, double rel,
                          double abs_bound, char* cmp, double* out, void* stream, unsigned long long* bytes,
                          double* bound, char* err, unsigned long long err_len) {
    return round_trip<double>(in, nx, ny, nz, rel, abs_bound, cmp, out, stream, bytes, bound, err, err_len);
}
int caller_decode_f32(char* cmp, unsigned long long nx, unsigned long long ny, unsigned long long nz, float* out,
                      void* stream, char* err, unsigned long long err_len) {
    return decode_only<float>(cmp, nx, ny, nz, out, stream, err, err_len);
}
unsigned long long caller_capacity_f32(unsigned long long n) { return WALTZ::compressed_buffer_capacity<float>(n); }
unsigned long long caller_capacity_f64(unsigned long long n) { return WALTZ::compressed_buffer_capacity<double>(n); }
// Byte offsets of the Config members the library reads, and its size: the
// binary interface both headers must agree on.
int caller_config_layout(unsigned long long* out, int cap) {
    const unsigned long long v[] = {offsetof(WALTZ::Config, ndims), offsetof(WALTZ::Config, dimx),
                                    offsetof(WALTZ::Config, dimy), offsetof(WALTZ::Config, dimz),
                                    offsetof(WALTZ::Config, num), offsetof(WALTZ::Config, errorBoundMode),
                                    offsetof(WALTZ::Config, absErrorBound), sizeof(WALTZ::Config)};
    const int n = int(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < n && i < cap; ++i) out[i] = v[i];
    return n;
}
// Config built from extents the way the reference's callers build it.
int caller_config_dims(unsigned long long x, unsigned long long y, unsigned long long z, unsigned long long* out) {
    WALTZ::Config c(x, y, z);
    out[0] = c.ndims; out[1] = c.dimx; out[2] = c.dimy; out[3] = c.dimz; out[4] = c.num;
    return 0;
}
int caller_levels(unsigned x, unsigned y, unsigned z, unsigned char* lxy, unsigned char* lz) {
    WALTZ::calculate_dwt_levels(dim3(x, y, z), *lxy, *lz);
    return 0;
}
}

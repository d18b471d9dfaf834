// Test-infrastructure shim: exposes internals of the reference CPU codec
// (compiled from its own sources by oracle/Makefile into oracle/_ref/) through
// plain C entry points, so tests can pin the oracle restatement stage by stage.
// Nothing in the product links or loads this file.
//
// Wrapped reference interfaces:
//   waltz_cpu::forward_f32/f64, inverse_f32/f64   cpu/src/transform.hpp:27-38
//   waltz_cpu_detail::wzp_encode/wzp_decode       cpu/src/wzp_cpu.hpp:23-35
#include "transform.hpp"
#include "wzp_cpu.hpp"

#include <cstdio>
#include <exception>

namespace {
thread_local char g_error[256];
int fail_with(const std::exception& e) {
    std::snprintf(g_error, sizeof(g_error), "%s", e.what());
    return -1;
}
}

extern "C" {

const char* ref_last_error(void) { return g_error; }

int ref_transform(void* data, void* scratch, int width, unsigned nx, unsigned ny, unsigned nz,
                  unsigned lxy, unsigned lz, int dyadic, int inverse, int avx2) {
    try {
        const waltz_cpu::Shape s{nx, ny, nz};
        if (width == 4) {
            auto* d = static_cast<float*>(data);
            auto* t = static_cast<float*>(scratch);
            if (inverse) waltz_cpu::inverse_f32(d, t, s, lxy, lz, dyadic != 0, 2, avx2 != 0);
            else waltz_cpu::forward_f32(d, t, s, lxy, lz, dyadic != 0, 2, avx2 != 0);
        } else {
            auto* d = static_cast<double*>(data);
            auto* t = static_cast<double*>(scratch);
            if (inverse) waltz_cpu::inverse_f64(d, t, s, lxy, lz, dyadic != 0, 2, avx2 != 0);
            else waltz_cpu::forward_f64(d, t, s, lxy, lz, dyadic != 0, 2, avx2 != 0);
        }
        return 0;
    } catch (const std::exception& e) {
        return fail_with(e);
    }
}

size_t ref_transform_scratch_elements(unsigned nx, unsigned ny, unsigned nz) {
    try {
        return waltz_cpu::workspace_elements(waltz_cpu::Shape{nx, ny, nz});
    } catch (...) {
        return 0;
    }
}

size_t ref_wzp_max_bytes(unsigned n) {
    try {
        return waltz_cpu_detail::wzp_max_bytes(n);
    } catch (...) {
        return 0;
    }
}

long long ref_wzp_encode(const unsigned short* mag, const unsigned* sign, unsigned n,
                         unsigned char* out, size_t capacity, int avx2) {
    try {
        return (long long)waltz_cpu_detail::wzp_encode(mag, sign, n, out, capacity, avx2 != 0);
    } catch (const std::exception& e) {
        return fail_with(e);
    }
}

int ref_wzp_decode(const unsigned char* in, size_t bytes, unsigned n,
                   unsigned short* mag, unsigned* sign, int avx2) {
    try {
        waltz_cpu_detail::wzp_decode(in, bytes, n, mag, sign, avx2 != 0);
        return 0;
    } catch (const std::exception& e) {
        return fail_with(e);
    }
}

} // extern "C"

// Baseline shim: plain C entry points over the reference's own CUDA library
// (src/waltz.cu, src/lossless/wzp.cu of the reference, compiled from its
// sources by oracle/Makefile into oracle/_ref/libwaltz_refgpu.so together with
// this file). The benchmark times it on the same GPU as the reference GPU
// baseline; nothing in the product links or loads it.
//
// Wrapped reference interfaces:
//   WALTZ::d_compress<T> / d_decompress<T>          include/waltz.hpp:47-81
//   WALTZ::compressed_buffer_capacity<T>            include/waltz.hpp:21-34
//   WALTZ::Waltz_report_enabled (stage tables, off unless refgpu_report(1))
//                                                   include/utils/Statistics.hpp:118
#include "waltz.hpp"

#include <cstdio>
#include <exception>

namespace {
thread_local char g_error[256];
thread_local bool g_report = false; // the reference's per-stage timing tables
int fail_with(const std::exception& e) {
    std::snprintf(g_error, sizeof(g_error), "%s", e.what());
    return -1;
}
}

extern "C" {

const char* refgpu_last_error(void) { return g_error; }

// Lets the reference print its own per-stage timing tables on later calls of
// this thread (off by default).
void refgpu_report(int on) { g_report = on != 0; }

size_t refgpu_capacity(uint64_t n, int width) {
    try {
        return width == 4 ? WALTZ::compressed_buffer_capacity<float>(n) : WALTZ::compressed_buffer_capacity<double>(n);
    } catch (const std::exception& e) {
        fail_with(e);
        return 0;
    }
}

// Device-to-device compression at an absolute bound (REL resolved by the
// caller, as the reference API requires); *written = archive bytes.
int refgpu_compress(void* d_in, int width, uint32_t nx, uint32_t ny, uint32_t nz, double abs_error, void* d_out,
                    size_t* written, void* stream) {
    try {
        WALTZ::Waltz_report_enabled = g_report;
        WALTZ::Config conf(nx, ny, nz);
        conf.errorBoundMode = WALTZ::EB_ABS;
        conf.absErrorBound = abs_error;
        *written = width == 4
                       ? WALTZ::d_compress<float>(conf, static_cast<float*>(d_in), static_cast<char*>(d_out), nullptr,
                                                  stream)
                       : WALTZ::d_compress<double>(conf, static_cast<double*>(d_in), static_cast<char*>(d_out),
                                                   nullptr, stream);
        return 0;
    } catch (const std::exception& e) {
        return fail_with(e);
    }
}

int refgpu_decompress(void* d_archive, int width, uint32_t nx, uint32_t ny, uint32_t nz, void* d_out, void* stream) {
    try {
        WALTZ::Waltz_report_enabled = g_report;
        WALTZ::Config conf(nx, ny, nz);
        if (width == 4)
            WALTZ::d_decompress<float>(conf, static_cast<char*>(d_archive), static_cast<float*>(d_out), nullptr,
                                       stream);
        else
            WALTZ::d_decompress<double>(conf, static_cast<char*>(d_archive), static_cast<double*>(d_out), nullptr,
                                        stream);
        return 0;
    } catch (const std::exception& e) {
        return fail_with(e);
    }
}

} // extern "C"

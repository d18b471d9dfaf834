/*
 * Waltz oracle: a plain-C, single-threaded restatement of the reference CPU
 * scalar codec (the byte-exact default profile). TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, the package smoke check and the CPU-baseline leg of bench.py
 * may load this library, and only as a checker. The GPU product never links,
 * loads or calls it.
 *
 * Parity pin: tests/test_oracle.py compares every entry point below against
 * the reference CPU codec compiled from its own sources (oracle/_ref) and
 * against the committed fixtures in tests/golden/.
 *
 * Reference correspondence (paths inside the reference project):
 *   wo_levels           include/utils/Blob.hpp:197-204 (dwt_levels)
 *   wo_zband            cpu/src/codec.cpp:89-95 (zband)
 *   wo_transform        cpu/src/transform.cpp:110-179, 409-456
 *   wo_wzp_encode       cpu/src/wzp_cpu.cpp:769-867
 *   wo_wzp_decode       cpu/src/wzp_cpu.cpp:869-949
 *   wo_compress         cpu/src/codec.cpp:177-258 (scalar backend)
 *   wo_decompress       cpu/src/codec.cpp:276-336 (native and compact repairs)
 *   wo_compact_repairs  src/small_pwe.cuh:21-105 (the compact WPW1 repair
 *                       section; groups placed in order, as this library's
 *                       encoder does, where the reference's CUDA packer
 *                       places them by an atomic counter)
 */
#ifndef WALTZ_ORACLE_H
#define WALTZ_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint32_t nx, ny, nz; /* x fastest */
    int width;           /* 4 = float32, 8 = float64 */
    double abs_error;    /* absolute pointwise bound (encode only) */
} wo_config;

unsigned wo_levels(uint32_t length);
unsigned wo_zband(uint32_t nx, uint32_t ny, uint32_t nz, unsigned lz, int dyadic);
/* Morton rank of (x,y,z) inside an nx*ny*nz brick (recursive ceil-half octants). */
uint32_t wo_morton(uint32_t x, uint32_t y, uint32_t z, uint32_t nx, uint32_t ny, uint32_t nz);

/* In-place all-level transform (synthesis mode 2, halo lifting). Returns 0 or -1. */
int wo_transform(void* data, int width, uint32_t nx, uint32_t ny, uint32_t nz,
                 unsigned lxy, unsigned lz, int dyadic, int inverse);

/* WZP stream of n u16 magnitudes and a natural sign bitmap (ceil(n/32) words). */
size_t wo_wzp_max_bytes(uint32_t n);
long long wo_wzp_encode(const uint16_t* mag, const uint32_t* sign, uint32_t n,
                        uint8_t* out, size_t capacity, char* err, size_t errlen);
int wo_wzp_decode(const uint8_t* in, size_t bytes, uint32_t n, uint16_t* mag, uint32_t* sign,
                  char* err, size_t errlen);

/* Quantize + Morton emit of a forward-transformed coefficient array (in place:
 * coefficients become their dequantized values). mag has n entries, sign
 * ceil(n/32) words (zeroed here), q-outliers are returned in ascending index
 * order. Returns the q-outlier count, or -1 on a domain failure. */
long long wo_quantize(void* coeff, int width, uint32_t nx, uint32_t ny, uint32_t nz, unsigned bz,
                      double quantum, uint16_t* mag, uint32_t* sign,
                      uint32_t* qidx, uint32_t* qval, char* err, size_t errlen);

size_t wo_max_compressed_bytes(const wo_config* c);
int wo_compress(const wo_config* c, const void* input, uint8_t* archive, size_t capacity,
                size_t* written, char* err, size_t errlen);
int wo_decompress(const wo_config* c, const uint8_t* archive, size_t bytes, void* output,
                  size_t output_bytes, char* err, size_t errlen);
/* The archive with its native repair section replaced by the compact one
 * (step, the originals of the compressed field), when that is smaller; else
 * a copy. out may not overlap archive. Returns 0 or -1. */
int wo_compact_repairs(const uint8_t* archive, size_t bytes, int width, const void* original, double step,
                       uint8_t* out, size_t capacity, size_t* written, char* err, size_t errlen);

#ifdef __cplusplus
}
#endif
#endif

/*
 * Batched device decode, same signature and contract as the reference
 * (include/waltz_gpu_batch.h:7-17 of the reference project).
 *
 * `host` and `packed` (device) hold identical bytes: 16-byte-aligned archive
 * blobs followed by 16-byte-aligned (u64 offset, u64 size) pairs in
 * sample/side/ZYX tile order; size 0 means "fill". Every archive is a
 * canonical archive of one x*y*z tile. The output is contiguous
 * (side, sample, fz, fy, fx); edge tiles are clipped to the frame. Scratch
 * must hold at least 3*stride*jobs*width + 8*256*bz*4 + 4 bytes with
 * stride = (x*y*z + 3) & ~3. Uses the caller's stream, is synchronous and
 * allocates nothing. Returns NULL on success, else a thread-local diagnostic.
 */
#pragma once
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct {
    uint32_t x, y, z, fx, fy, fz, samples, sides, width;
} waltz_batch_shape;
const char* waltz_gpu_decode_batch(const waltz_batch_shape* shape,
    const void* host, const void* packed, size_t bytes, void* scratch, size_t scratch_bytes,
    void* output, size_t output_bytes, double fill, void* stream);
#ifdef __cplusplus
}
#endif

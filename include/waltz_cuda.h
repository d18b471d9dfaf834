/*
 * Single-chunk device decode, same signature and contract as the reference
 * (include/waltz_cuda.h:11-13 of the reference project): decode a trusted
 * canonical archive on the calling thread's current CUDA device and stream.
 * Both pointers are device pointers; the call is synchronous and serialised
 * by a process-wide lock. Returns NULL on success, else a thread-local
 * diagnostic. Only canonical-profile archives are accepted (flags, levels,
 * z band and length must match the chunk geometry exactly).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
const char* waltz_cuda_decode_chunk(uint32_t nx, uint32_t ny, uint32_t nz, int width,
                                    const void* archive, size_t archive_bytes,
                                    void* output, size_t output_bytes, void* stream);
#ifdef __cplusplus
}
#endif

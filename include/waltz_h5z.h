/*
 * HDF5 filter 61197 ("Waltz canonical") on the GPU codec, exported by
 * waltz_b200/plugins/libwaltz_h5z.so (an HDF5 plugin library: it also exports
 * H5PLget_plugin_type / H5PLget_plugin_info for HDF5_PLUGIN_PATH discovery).
 *
 * Replaces the reference's CPU filter callback (python/hdf5/filter.cpp:16-58
 * of the reference project): same signature, same 6-word client data
 * (nx, ny, nz, width, bound low word, bound high word), same chunk archives,
 * and the same failure contract (returns 0 and leaves *buffer untouched).
 * flags & 0x0100 (H5Z_FLAG_REVERSE) decodes. The buffer is malloc'd memory
 * owned by the caller; on success it is freed and replaced.
 */
#ifndef WALTZ_H5Z_H
#define WALTZ_H5Z_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
size_t waltz_b200_h5z_filter(unsigned flags, size_t count, const unsigned cd[], size_t bytes, size_t* buffer_size,
                             void** buffer);
#ifdef __cplusplus
}
#endif
#endif

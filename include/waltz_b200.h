/*
 * Waltz B200: C ABI of the GPU codec (one CUDA device per process, the
 * calling thread's current device, the caller's stream).
 *
 * All pointers named d_* are device pointers. Every call is synchronous on
 * its stream when it returns. Functions returning int give 0 on success and
 * -1 on failure with the diagnostic in waltz_b200_last_error() (thread local).
 * Archives are the reference's 32-byte-header native archives: in the default
 * profile they are byte-identical to the reference CPU scalar codec.
 *
 * Reference interfaces these replace (paths inside the reference project):
 *   waltz_b200_compressed_capacity  include/waltz.hpp:21-33 (compressed_buffer_capacity<T>)
 *   waltz_b200_compress             include/waltz.hpp:51-61 (d_compress<T>) -> src/waltz.cu:327-609
 *   waltz_b200_decompress           include/waltz.hpp:70-81 (d_decompress<T>) -> src/waltz.cu:612-834
 *   waltz_b200_extrema              include/waltz.hpp:39-40 (d_extrema<T>) -> src/waltz.cu:867-876
 * The reference's own C entry points keep their exact signatures in
 * waltz_cuda.h and waltz_gpu_batch.h, exported by the same library.
 */
#ifndef WALTZ_B200_H
#define WALTZ_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Archive capacity the caller must provide for n samples of `width` bytes
 * (4 or 8): one input volume plus the fixed side-record caps plus 1 MiB. */
size_t waltz_b200_compressed_capacity(uint64_t n, int width);

/* Compress nx*ny*nz samples (x fastest) of width 4 (float) or 8 (double) at
 * the absolute pointwise bound abs_error. *written receives the archive size. */
int waltz_b200_compress(const void* d_input, int width, uint32_t nx, uint32_t ny, uint32_t nz,
                        double abs_error, void* d_archive, size_t capacity, size_t* written,
                        void* stream);

/* Transform forms. PLAIN is the default profile (lifting, archives
 * byte-identical to the reference CPU codec). The MATRIX forms are the
 * precision form: the plane schedule's Z stage (all Z levels) runs as one
 * nz x nz matrix on the tensor cores and the repair pass restores the bound.
 * They differ in the tensor-core arithmetic:
 *   MATRIX        TF32x3: TF32 hi/lo halves, three products, FP32 accumulation
 *                 (about 21 bits);
 *   MATRIX_BF16   BF16x3: three bf16 slices, six products, FP32 accumulation
 *                 (fp32-accurate);
 *   MATRIX_EXACT  five 7-bit integer slices in bf16 per column and matrix row
 *                 (power-of-two scaled), every product order accumulated
 *                 exactly in its own FP32 tile and recombined in double:
 *                 about 2^-35 relative error, for double fields (nz <= 96).
 * Such archives set header flag bit 6 (which the reference's decoders
 * reject) and record the form in the two top bits of header byte 3, the z
 * band (0 TF32x3, 1 BF16x3, 2 exact slices). The matrix forms need the plane
 * schedule (Z levels differ from XY levels) with 1 <= nz <= 128 (96 for
 * MATRIX_EXACT) and nx*ny a multiple of 4; float and double fields (TF32x3
 * and BF16x3 round double samples to float first; a double field's
 * quantisation and repair decisions stay in double). New surface: the
 * reference has no counterpart (its header reserves the bits,
 * include/utils/Blob.hpp:46-53). */
#define WALTZ_B200_FORM_PLAIN 0
#define WALTZ_B200_FORM_MATRIX 1
#define WALTZ_B200_FORM_MATRIX_BF16 2
#define WALTZ_B200_FORM_MATRIX_EXACT 3
int waltz_b200_compress_form(const void* d_input, int width, uint32_t nx, uint32_t ny, uint32_t nz,
                             double abs_error, int form, void* d_archive, size_t capacity, size_t* written,
                             void* stream);

/* Batched compress of many independent fields of any shapes (the chunked
 * datasets of the reference's loaders, one archive per chunk): one call,
 * one CUDA graph replayed while the batch description stays the same, every
 * chunk's archive byte-identical to waltz_b200_compress of that chunk.
 * written[i] receives archive i's size. Fails (naming the item) if any item
 * fails. New surface: the reference has no batched encoder. */
typedef struct waltz_b200_chunk {
    const void* input;  /* device, nx*ny*nz samples of `width` bytes */
    uint32_t nx, ny, nz;
    double abs_error;
    void* archive;      /* device */
    uint64_t capacity;  /* >= waltz_b200_compressed_capacity(nx*ny*nz, width) */
} waltz_b200_chunk;
int waltz_b200_compress_batch(const waltz_b200_chunk* chunks, uint32_t count, int width, uint64_t* written,
                              void* stream);

/* Batched decode of many archives of any shapes and either form into caller
 * buffers (views of one preallocated tensor, or boxes inside a larger frame
 * through the output strides): one call, one CUDA graph. Archive and output
 * addresses and headers reach the graph through a device table, so the graph
 * is captured once per description (count, shapes, forms, output strides)
 * and replayed for later batches of other archives and other outputs with
 * the same description. `header` optionally points to a host copy of an
 * archive's first 32 bytes (NULL: read from the device). Every output equals
 * waltz_b200_decompress of that archive. Fails (naming the item) if any item
 * fails. New surface: the reference batch decoder needs one tile shape for
 * the whole batch (waltz_gpu_decode_batch, src/batch_decode.cuh:74-186). */
typedef struct waltz_b200_archive {
    const void* archive;  /* device */
    uint64_t bytes;
    const void* header;   /* optional host copy of the 32-byte header */
    uint32_t nx, ny, nz;
    void* output;         /* device; sample (x,y,z) at output[z*stride_z + y*stride_y + x] */
    uint64_t output_bytes;/* bytes from `output` to the end of the chunk's box */
    uint64_t stride_y;    /* elements between rows; 0 = nx */
    uint64_t stride_z;    /* elements between planes; 0 = stride_y*ny */
} waltz_b200_archive;
int waltz_b200_decompress_batch(const waltz_b200_archive* archives, uint32_t count, int width, void* stream);

/* Execution form of the batch graphs that the calling thread captures next
 * (a performance knob: results do not depend on it).
 * WALTZ_B200_BATCH_STAGES: fields split round-robin into `width` groups; per
 *   group every pipeline stage is one launch over all its fields' tiles (a
 *   chunk-tile work list); groups run as parallel graph branches.
 * WALTZ_B200_BATCH_FIELDS: each field's own launches, fields round-robin on
 *   `width` parallel graph branches. Default, width 32.
 * WALTZ_B200_BATCH_QUEUE: as STAGES, but every stage launch is a persistent
 *   work queue: a grid of resident CTAs pulling chunk-tile items (a field's
 *   block of that stage) from a device ticket, reset by the graph itself.
 * width 1..64. Returns 0, or -1 for an invalid configuration. */
/* Tuning options of the calling thread (performance knobs: results do not
 * depend on them). Returns 0, or -1 for an unknown option or value.
 * WALTZ_B200_OPT_STAGE_KERNELS (1 default, 0): plane schedule, run a whole Z
 *   or XY stage in one kernel where its lines or planes fit in shared memory.
 * WALTZ_B200_OPT_ZMARCH_PLANES (0 = automatic, else >= 16): planes per CTA of
 *   the forward dyadic z-march (work per tile against the 8-plane halo).
 * WALTZ_B200_OPT_SMALL_LEVEL (samples, default 2^15, 0 = none): inverse
 *   levels (dyadic, and the plane schedule's XY levels) of at most this many
 *   samples stage their tiles with reflecting loads instead of tensor-map
 *   copies (their tiles are almost all edge tiles).
 * WALTZ_B200_OPT_SMALL_FWD (samples, default 2^20, 0 = none): the same for
 *   forward levels (dyadic and XY), whose z-march may then also use 8-plane
 *   ranges. */
#define WALTZ_B200_OPT_STAGE_KERNELS 1
#define WALTZ_B200_OPT_ZMARCH_PLANES 2
#define WALTZ_B200_OPT_SMALL_LEVEL 3
#define WALTZ_B200_OPT_SMALL_FWD 4
/* WALTZ_B200_OPT_COMPACT_REPAIRS (0 default, 16 or 64): not a performance
 *   knob but an opt-in archive profile, the reference's compact repair
 *   section (WPW1, src/small_pwe.cuh:21-152; its CUDA library selects it with
 *   WALTZ_SMALL_PWE_SCALE): the calling thread's later compressions store
 *   their repair errors as int8 multiples of step = eb / value where that
 *   provably keeps the sample within step of the original, in groups of 32,
 *   when that section is smaller than the native errors (header flag bit 1).
 *   Such archives decode with waltz_b200_decompress(_batch) and the reference
 *   CPU decoder; the canonical decoders (waltz_cuda_decode_chunk,
 *   waltz_gpu_decode_batch) refuse them, as the reference's do. */
#define WALTZ_B200_OPT_COMPACT_REPAIRS 5
/* WALTZ_B200_OPT_XY_MARCH (0 default; bit 0: forward levels, bit 1:
 *   inverse levels): plane schedule, run those XY levels that the
 *   whole-stage kernels do not take as a warp march (a warp per strip of 56 x
 *   and plane walking down y in registers, each lane holding an even/odd pair
 *   and X lifted across the lanes by shuffles) instead of the shared-memory
 *   staged kernels. A performance knob like the others: the bytes do not
 *   change. */
#define WALTZ_B200_OPT_XY_MARCH 6
/* WALTZ_B200_OPT_SMALL_MARCH (samples, default 0 = none): dyadic inverse
 *   levels of at most this many samples run as two register marches (the Z
 *   synthesis, then the X and Y synthesis) instead of the tile inverse, whose
 *   tiles cannot fill the GPU on small levels. A performance knob like the
 *   others: the bytes do not change. */
#define WALTZ_B200_OPT_SMALL_MARCH 7
/* WALTZ_B200_OPT_SMALL_MARCH_FWD (samples, default 0 = none): the same for
 *   dyadic forward levels (the Y and X analysis as the warp march, then the
 *   Z analysis as the register march). */
#define WALTZ_B200_OPT_SMALL_MARCH_FWD 8
int waltz_b200_set_option(int option, int value);

#define WALTZ_B200_BATCH_STAGES 0
#define WALTZ_B200_BATCH_FIELDS 1
#define WALTZ_B200_BATCH_QUEUE 2
int waltz_b200_batch_config(int mode, int width);

/* Decode an archive of `bytes` bytes into nx*ny*nz samples (the archive does
 * not store its dimensions); either form. bytes == 0 takes the length from
 * the archive's 32-byte header (its section sizes), as the reference's
 * d_decompress does, which has no length argument (src/waltz.cu:612-626). */
int waltz_b200_decompress(const void* d_archive, size_t bytes, int width, uint32_t nx, uint32_t ny,
                          uint32_t nz, void* d_output, size_t output_bytes, void* stream);

/* Minimum and maximum of n samples (the REL -> ABS bound resolution). */
int waltz_b200_extrema(const void* d_input, int width, uint64_t n, double* min_out, double* max_out,
                       void* stream);

const char* waltz_b200_last_error(void);

/* Diagnostic stage entry points (used by the parity tests).
 * waltz_b200_transform: in-place all-level CDF 9/7 analysis (inverse = 0)
 *   into the split-band coefficient layout, or synthesis (inverse = 1);
 *   replaces allhalo::forward / allhalo::inverse
 *   (include/transformers/all_halo.cuh:278-380 of the reference).
 * waltz_b200_wzp_encode: WZP stream of n Morton-packed u16 magnitudes (16-byte
 *   aligned) and a natural sign bitmap (ceil(n/32) words); replaces lossless::wzp_enqueue
 *   (src/lossless/wzp.cu:1102-1126 of the reference). */
int waltz_b200_transform(void* d_data, int width, uint32_t nx, uint32_t ny, uint32_t nz, int inverse,
                         void* stream);
int waltz_b200_wzp_encode(const uint16_t* d_mag, const uint32_t* d_sign, uint32_t n, void* d_out,
                          size_t capacity, size_t* written, void* stream);
/* waltz_b200_zmatrix / _f64: the precision form's Z transform in place on a
 *   z-major float / double field (nx*ny a multiple of 4, 1 <= nz <= 128): all
 *   Z levels of the CDF 9/7 analysis (inverse = 0, coefficients in split-band
 *   order) or synthesis (inverse = 1) as one nz x nz matrix on the tensor
 *   cores (TF32 hi/lo halves, FP32 accumulation; double input is rounded to
 *   float first, results are written back in the field's type). Counterpart
 *   of the reference's plane schedule Z stage,
 *   include/transformers/all_halo.cuh:143-224. */
int waltz_b200_zmatrix(float* d_data, uint32_t nx, uint32_t ny, uint32_t nz, int inverse, void* stream);
int waltz_b200_zmatrix_f64(double* d_data, uint32_t nx, uint32_t ny, uint32_t nz, int inverse, void* stream);
/* waltz_b200_zmatrix_split: the same Z transform of a float (width 4) or
 *   double (width 8) field in any matrix form (WALTZ_B200_FORM_MATRIX,
 *   _MATRIX_BF16, _MATRIX_EXACT). */
int waltz_b200_zmatrix_split(void* d_data, int width, uint32_t nx, uint32_t ny, uint32_t nz, int inverse, int form,
                             void* stream);
/* Allocation-free variant of waltz_b200_wzp_encode (same arguments, same
 * stream bytes), for callers that cannot allocate device memory when they
 * call: a framework whose allocator owns the device budget, a plugin or filter
 * callback, or a loop that cannot take cudaMalloc's device synchronisation.
 * No counterpart in the reference. Its working state lives in one static
 * device array of about 256 KiB that every GPU loading the library holds
 * until exit; n is limited to 134217728 magnitudes (16384 chunks) and larger
 * n is rejected with an error. The first call on a device looks up the
 * array's device address (make that first call before any stream capture);
 * the address stays valid for the life of the device's context, so a
 * cudaDeviceReset of that device voids it for the rest of the process.
 * Calls share the array, so calls that overlap on the GPU (other streams,
 * threads or processes sharing a context) race: serialise them. */
int waltz_b200_wzp_encode_noalloc(const uint16_t* d_mag, const uint32_t* d_sign, uint32_t n, void* d_out,
                                  size_t capacity, size_t* written, void* stream);
/* Test hook for the bounded-wait path: compress with chunk `skip_chunk`
 * never publishing its lookback state and every wait capped at `spin_cap`
 * polls (~0.5 us each). Must fail with a lookback-timeout diagnostic. */
int waltz_b200_test_lookback_timeout(const void* d_input, int width, uint32_t nx, uint32_t ny, uint32_t nz,
                                     double abs_error, void* d_archive, size_t capacity, uint32_t skip_chunk,
                                     uint32_t spin_cap, void* stream);

/* Instrumentation. waltz_b200_launch_count: kernels launched by this library
 * since load. waltz_b200_profile(1) makes the calling thread record CUDA
 * events between the pipeline stages of its next calls; after a call,
 * waltz_b200_stage_times fills up to `cap` stage durations (ms) and names and
 * returns how many stages were timed (the reference's per-stage GPUTimer
 * report, include/utils/Timer.hpp:5-63). */
unsigned long long waltz_b200_launch_count(void);
/* Batch graphs captured since load (replays do not count). */
unsigned long long waltz_b200_graph_count(void);
void waltz_b200_profile(int enable);
int waltz_b200_stage_times(double* ms, const char** names, int cap);

#ifdef __cplusplus
}
#endif
#endif

/*
 * Waltz oracle: plain-C restatement of the reference CPU scalar codec.
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU library, never the
 * product. See waltz_oracle.h for the reference correspondence and pinning.
 *
 * Build flags must keep IEEE semantics: -ffp-contract=off -fno-fast-math,
 * round-to-nearest, no flush-to-zero (the defaults of a C program).
 */
#include "waltz_oracle.h"

#include <fenv.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- helpers */

static void say(char* err, size_t len, const char* msg) {
    if (err && len) snprintf(err, len, "%s", msg);
}
static void put32(uint8_t* p, uint32_t v) { p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24); }
static void put64(uint8_t* p, uint64_t v) { put32(p, (uint32_t)v); put32(p + 4, (uint32_t)(v >> 32)); }
static uint32_t get32(const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24); }
static uint64_t get64(const uint8_t* p) { return get32(p) | ((uint64_t)get32(p + 4) << 32); }
static uint32_t get24(const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16); }
static void put24(uint8_t* p, uint32_t v) { p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); }
static size_t pad8(size_t n) { return (n + 7) & ~(size_t)7; }
static uint32_t half_len(uint32_t n) { return n - n / 2; }

/* Whole-sample symmetric reflection into [0,n), period 2n-2
 * (cpu/src/transform.cpp:60-66). */
static uint32_t mirror_index(int64_t p, uint32_t n) {
    int64_t period, r;
    if (n <= 1) return 0;
    period = 2 * (int64_t)n - 2;
    r = p % period;
    if (r < 0) r += period;
    return (uint32_t)(r < (int64_t)n ? r : period - r);
}
/* Split-band address of spatial position p: evens to the low half, odds after
 * ceil(n/2) (cpu/src/transform.cpp:68-71). */
static uint32_t coeff_index(int64_t p, uint32_t n) {
    const uint32_t r = mirror_index(p, n);
    return r / 2 + ((r & 1) ? half_len(n) : 0);
}

static int cmp_pair(const void* a, const void* b) {
    const uint32_t x = ((const uint32_t*)a)[0], y = ((const uint32_t*)b)[0];
    return x < y ? -1 : x > y;
}
/* Sort (index,value) pairs by index; indices are unique. */
static void sort_pairs(uint32_t* idx, uint32_t* val, size_t count) {
    uint32_t* tmp;
    size_t i;
    if (count < 2) return;
    tmp = (uint32_t*)malloc(count * 8);
    if (!tmp) abort();
    for (i = 0; i < count; ++i) { tmp[2 * i] = idx[i]; tmp[2 * i + 1] = val[i]; }
    qsort(tmp, count, 8, cmp_pair);
    for (i = 0; i < count; ++i) { idx[i] = tmp[2 * i]; val[i] = tmp[2 * i + 1]; }
    free(tmp);
}

/* 0 when all `count` LE indices are < n and pairwise distinct. */
static int check_indices(const uint8_t* p, uint32_t count, size_t n, uint8_t* seen) {
    uint32_t i, prev = 0;
    int ordered = 1;
    for (i = 0; i < count; ++i) {
        const uint32_t v = get32(p + 4 * (size_t)i);
        if (v >= n) return -1;
        if (i && v <= prev) ordered = 0;
        prev = v;
    }
    if (ordered) return 0;
    memset(seen, 0, n);
    for (i = 0; i < count; ++i) {
        const uint32_t v = get32(p + 4 * (size_t)i);
        if (seen[v]) return -1;
        seen[v] = 1;
    }
    return 0;
}

unsigned wo_levels(uint32_t length) {
    unsigned l = 0;
    while (length > 8 && l < 5) { length -= length / 2; ++l; }
    return l;
}

unsigned wo_zband(uint32_t nx, uint32_t ny, uint32_t nz, unsigned lz, int dyadic) {
    uint64_t bricks, full;
    if (dyadic) {
        const uint32_t b = (nz + ((1u << lz) - 1)) >> lz;
        return b > 16 ? 16 : b;
    }
    if (nz < 4) return nz;
    bricks = (uint64_t)((nx + 15) / 16) * ((ny + 15) / 16);
    full = (uint64_t)(nx / 16) * (ny / 16);
    return (bricks - full) * 32 >= bricks ? 4 : 2;
}

/* Recursive octant rank: at every step the box splits into a lower half of
 * ceil(len/2) and an upper half of floor(len/2) on each axis; octants are
 * ordered z-half first, then y-half, then x-half (cpu/src/codec.cpp:96-107). */
uint32_t wo_morton(uint32_t x, uint32_t y, uint32_t z, uint32_t nx, uint32_t ny, uint32_t nz) {
    uint32_t rank = 0;
    while (nx > 1 || ny > 1 || nz > 1) {
        const uint32_t lx = nx - nx / 2, ly = ny - ny / 2, lzz = nz - nz / 2;
        const int ux = x >= lx, uy = y >= ly, uz = z >= lzz;
        const uint32_t hz = uz ? nz / 2 : lzz, hy = uy ? ny / 2 : ly;
        if (uz) rank += lzz * nx * ny;
        if (uy) rank += hz * ly * nx;
        if (ux) rank += hz * hy * lx;
        if (ux) x -= lx;
        if (uy) y -= ly;
        if (uz) z -= lzz;
        nx = ux ? nx / 2 : lx;
        ny = hy;
        nz = hz;
    }
    return rank;
}

/* Eight rank tables: slot bit0 = short x edge, bit1 = short y, bit2 = short z. */
static uint16_t* build_ranks(const uint32_t d[3], unsigned bz) {
    uint16_t* t = (uint16_t*)calloc(8 * 8192, 2);
    unsigned s;
    if (!t) return NULL;
    for (s = 0; s < 8; ++s) {
        const uint32_t bx = (s & 1) ? d[0] % 16 : 16, by = (s & 2) ? d[1] % 16 : 16, bzz = (s & 4) ? d[2] % bz : bz;
        uint32_t x, y, z;
        for (z = 0; z < bzz; ++z)
            for (y = 0; y < by; ++y)
                for (x = 0; x < bx; ++x)
                    t[s * 8192 + (z * by + y) * bx + x] = (uint16_t)wo_morton(x, y, z, bx, by, bzz);
    }
    return t;
}

/* -------------------------------------------------------------------- WZP */
/* Stream layout (cpu/src/wzp_cpu.cpp:769-867):
 *   u32 LE payload offset per 16-chunk group (first nonzero chunk, 0 if empty)
 *   u24 LE metadata per 8192-magnitude chunk: low 14 bits 0 = zero chunk,
 *       0x3fff = raw, else RZE length; high 10 bits sign-byte count (0 = 1024)
 *   payload: per nonzero chunk the magnitude bytes then ceil(nnz/8) sign bytes. */
#define CHUNK 8192u
#define GROUP 16u
#define RAW_CODE 0x3fffu

static uint32_t wzp_chunks(uint32_t n) { return n ? 1 + (n - 1) / CHUNK : 0; }

size_t wo_wzp_max_bytes(uint32_t n) {
    const uint64_t chunks = wzp_chunks(n), groups = (chunks + GROUP - 1) / GROUP;
    return (size_t)(groups * 4 + chunks * 3 + (uint64_t)n * 2 + ((uint64_t)n + 7) / 8);
}

/* Bit-plane transpose of each 16-magnitude block: plane word p holds bit
 * (15-p) of the block's 16 magnitudes, magnitude e at bit (15-e); words are
 * stored plane-major over the chunk's blocks; a tail of fewer than 16
 * magnitudes follows verbatim (the LC BIT_2 component). */
static void bit_planes(const uint16_t* m, uint32_t count, uint8_t* out) {
    const uint32_t blocks = count / 16;
    uint32_t b, p, e, i;
    for (b = 0; b < blocks; ++b)
        for (p = 0; p < 16; ++p) {
            uint32_t w = 0;
            for (e = 0; e < 16; ++e) w |= (uint32_t)((m[b * 16 + e] >> (15 - p)) & 1) << (15 - e);
            out[(p * blocks + b) * 2] = (uint8_t)w;
            out[(p * blocks + b) * 2 + 1] = (uint8_t)(w >> 8);
        }
    for (i = blocks * 16; i < count; ++i) { out[2 * i] = (uint8_t)m[i]; out[2 * i + 1] = (uint8_t)(m[i] >> 8); }
}
static void bit_planes_inverse(const uint8_t* in, uint32_t count, uint16_t* m) {
    const uint32_t blocks = count / 16;
    uint32_t b, p, e, i;
    for (b = 0; b < blocks; ++b)
        for (e = 0; e < 16; ++e) {
            uint32_t v = 0;
            for (p = 0; p < 16; ++p) {
                const uint32_t w = in[(p * blocks + b) * 2] | ((uint32_t)in[(p * blocks + b) * 2 + 1] << 8);
                v |= ((w >> (15 - e)) & 1) << (15 - p);
            }
            m[b * 16 + e] = (uint16_t)v;
        }
    for (i = blocks * 16; i < count; ++i) m[i] = (uint16_t)(in[2 * i] | (in[2 * i + 1] << 8));
}

/* Zero + repetition elimination of up to 16384 bytes: keep the nonzero bytes,
 * then a 2048-byte nonzero bitmap, reduced three times by keeping only the
 * bytes that differ from their predecessor (the first compared with 0) and
 * marking them in an eight-times smaller bitmap; the final 4 bytes are kept
 * verbatim (the LC RZE_1 component). Returns the length, 0 for all-zero. */
static uint32_t rze_encode(const uint8_t* in, uint32_t bytes, uint8_t* out) {
    uint8_t levels[2048 + 256 + 32 + 4];
    uint32_t pos = 0, i, base = 0, range;
    memset(levels, 0, sizeof(levels));
    for (i = 0; i < bytes; ++i)
        if (in[i]) { levels[i >> 3] |= (uint8_t)(1u << (i & 7)); out[pos++] = in[i]; }
    if (!pos) return 0;
    for (range = 2048; range > 4; range /= 8) {
        uint8_t prev = 0;
        for (i = 0; i < range; ++i) {
            const uint8_t v = levels[base + i];
            if (v != prev) { levels[base + range + (i >> 3)] |= (uint8_t)(1u << (i & 7)); out[pos++] = v; }
            prev = v;
        }
        base += range;
    }
    memcpy(out + pos, levels + base, 4);
    return pos + 4;
}

static unsigned pop8(uint8_t v) { unsigned c = 0; while (v) { c += v & 1; v >>= 1; } return c; }

static int rze_decode(const uint8_t* in, uint32_t stored, uint32_t bytes, uint8_t* out) {
    uint8_t levels[2048 + 256 + 32 + 4];
    uint32_t pos, base = 2048 + 256 + 32, range, i, nonzero = 0, rd;
    if (stored < 4) return -1;
    pos = stored - 4;
    memcpy(levels + base, in + pos, 4);
    for (range = 32; range <= 2048; range *= 8) {
        const uint8_t* mark = levels + base;
        uint32_t changes = 0;
        uint8_t v = 0;
        for (i = 0; i < range / 8; ++i) changes += pop8(mark[i]);
        if (changes > pos) return -1;
        pos -= changes;
        rd = pos;
        base -= range;
        for (i = 0; i < range; ++i) {
            if ((mark[i >> 3] >> (i & 7)) & 1) {
                if (in[rd] == v) return -1; /* a recorded change must change */
                v = in[rd++];
            }
            levels[base + i] = v;
        }
    }
    for (i = 0; i < 2048; ++i) nonzero += pop8(levels[i]);
    if (!nonzero || nonzero != pos) return -1;
    if ((bytes & 7) && (levels[bytes / 8] >> (bytes & 7))) return -1;
    for (i = bytes / 8 + ((bytes & 7) != 0); i < 2048; ++i)
        if (levels[i]) return -1;
    rd = 0;
    for (i = 0; i < bytes; ++i) {
        uint8_t v = 0;
        if ((levels[i >> 3] >> (i & 7)) & 1) {
            v = in[rd++];
            if (!v) return -1;
        }
        out[i] = v;
    }
    return 0;
}

long long wo_wzp_encode(const uint16_t* mag, const uint32_t* sign, uint32_t n,
                        uint8_t* out, size_t cap, char* err, size_t errlen) {
    const uint32_t chunks = wzp_chunks(n), groups = (chunks + GROUP - 1) / GROUP;
    const size_t header = (size_t)groups * 4 + (size_t)chunks * 3;
    uint8_t* meta = out + (size_t)groups * 4;
    size_t cursor = header;
    uint8_t planes[2 * CHUNK], packed[2 * CHUNK + 2048 + 256 + 32 + 4 + 8]; /* worst case before the raw test */
    uint32_t g, c;
    if (n > 0x7fffffffu) { say(err, errlen, "WZP element count exceeds the GPU format limit"); return -1; }
    if (!n) return 0;
    if (cap < header) { say(err, errlen, "WZP output capacity is too small"); return -1; }
    for (g = 0; g < groups; ++g) {
        int seen_nonzero = 0;
        put32(out + 4 * (size_t)g, 0);
        for (c = g * GROUP; c < chunks && c < (g + 1) * GROUP; ++c) {
            const uint32_t first = c * CHUNK, count = n - first < CHUNK ? n - first : CHUNK;
            const uint16_t* m = mag + first;
            uint32_t nnz = 0, i, rze, stored, sign_bytes, rank = 0;
            int raw;
            for (i = 0; i < count; ++i) nnz += m[i] != 0;
            if (!nnz) { put24(meta + 3 * (size_t)c, 0); continue; }
            bit_planes(m, count, planes);
            rze = rze_encode(planes, 2 * count, packed);
            raw = rze + 2 >= 2 * count;
            stored = raw ? 2 * count : rze;
            sign_bytes = (nnz + 7) / 8;
            if (stored + sign_bytes > cap - cursor) { say(err, errlen, "WZP output capacity is too small"); return -1; }
            if (cursor - header > 0xffffffffu - (stored + sign_bytes)) { say(err, errlen, "WZP payload exceeds its 32-bit directory"); return -1; }
            if (!seen_nonzero) { put32(out + 4 * (size_t)g, (uint32_t)(cursor - header)); seen_nonzero = 1; }
            if (raw) {
                for (i = 0; i < count; ++i) { out[cursor + 2 * i] = (uint8_t)m[i]; out[cursor + 2 * i + 1] = (uint8_t)(m[i] >> 8); }
            } else {
                memcpy(out + cursor, packed, rze);
            }
            memset(out + cursor + stored, 0, sign_bytes);
            for (i = 0; i < count; ++i) {
                const uint32_t at = first + i;
                if (!m[i]) continue;
                out[cursor + stored + (rank >> 3)] |= (uint8_t)(((sign[at >> 5] >> (at & 31)) & 1) << (rank & 7));
                ++rank;
            }
            put24(meta + 3 * (size_t)c, (raw ? RAW_CODE : stored) | ((sign_bytes == 1024 ? 0 : sign_bytes) << 14));
            cursor += stored + sign_bytes;
        }
    }
    return (long long)cursor;
}

/* Metadata of one chunk -> (magnitude bytes, sign bytes, raw); -1 if invalid
 * (cpu/src/wzp_cpu.cpp:668-684). */
static int chunk_sizes(uint32_t meta, uint32_t count, uint32_t* mbytes, uint32_t* sbytes, int* raw) {
    const uint32_t code = meta & RAW_CODE, scode = meta >> 14;
    if (!code) {
        if (scode) return -1;
        *mbytes = *sbytes = 0; *raw = 0;
        return 0;
    }
    *raw = code == RAW_CODE;
    if (!*raw && (code < 4 || code + 2 >= 2 * count)) return -1;
    *sbytes = scode ? scode : 1024;
    if (*sbytes > (count + 7) / 8) return -1;
    *mbytes = *raw ? 2 * count : code;
    return 0;
}

typedef struct { uint32_t offset, length; } span_t;
static int cmp_span(const void* a, const void* b) {
    const uint32_t x = ((const span_t*)a)->offset, y = ((const span_t*)b)->offset;
    return x < y ? -1 : x > y;
}

int wo_wzp_decode(const uint8_t* in, size_t bytes, uint32_t n, uint16_t* mag, uint32_t* sign,
                  char* err, size_t errlen) {
    const uint32_t chunks = wzp_chunks(n), groups = (chunks + GROUP - 1) / GROUP;
    const size_t header = (size_t)groups * 4 + (size_t)chunks * 3;
    const uint8_t* meta = in + (size_t)groups * 4;
    const uint8_t* payload = in + header;
    size_t payload_bytes, cursor_all = 0;
    span_t* spans;
    uint8_t planes[2 * CHUNK];
    uint32_t g, c, i;
    if (n > 0x7fffffffu) { say(err, errlen, "WZP element count exceeds the GPU format limit"); return -1; }
    if (!n) { if (bytes) { say(err, errlen, "WZP nonempty archive for zero elements"); return -1; } return 0; }
    if (bytes < header || bytes > wo_wzp_max_bytes(n)) { say(err, errlen, "WZP archive size is outside its valid bounds"); return -1; }
    payload_bytes = bytes - header;
    if (payload_bytes > 0xffffffffu) { say(err, errlen, "WZP payload exceeds its 32-bit directory"); return -1; }
    /* Directory: the nonempty groups must tile the payload exactly. */
    spans = (span_t*)malloc(sizeof(span_t) * groups);
    if (!spans) { say(err, errlen, "out of memory"); return -1; }
    for (g = 0; g < groups; ++g) {
        uint32_t len = 0;
        for (c = g * GROUP; c < chunks && c < (g + 1) * GROUP; ++c) {
            const uint32_t count = n - c * CHUNK < CHUNK ? n - c * CHUNK : CHUNK;
            uint32_t mb, sb;
            int raw;
            if (chunk_sizes(get24(meta + 3 * (size_t)c), count, &mb, &sb, &raw)) { free(spans); say(err, errlen, "WZP invalid chunk metadata"); return -1; }
            len += mb + sb;
        }
        spans[g].offset = get32(in + 4 * (size_t)g);
        spans[g].length = len;
        if (spans[g].offset > payload_bytes || len > payload_bytes - spans[g].offset || (!len && spans[g].offset)) {
            free(spans); say(err, errlen, "WZP directory range is outside the payload"); return -1;
        }
    }
    if (groups == 1 && spans[0].offset != 0) { free(spans); say(err, errlen, "WZP directory does not cover the payload"); return -1; }
    {
        span_t* sorted = (span_t*)malloc(sizeof(span_t) * groups);
        if (!sorted) { free(spans); say(err, errlen, "out of memory"); return -1; }
        memcpy(sorted, spans, sizeof(span_t) * groups);
        qsort(sorted, groups, sizeof(span_t), cmp_span);
        for (g = 0; g < groups; ++g) {
            if (!sorted[g].length) continue;
            if (sorted[g].offset != cursor_all) { free(sorted); free(spans); say(err, errlen, "WZP payload groups overlap or leave a gap"); return -1; }
            cursor_all += sorted[g].length;
        }
        free(sorted);
        if (cursor_all != payload_bytes) { free(spans); say(err, errlen, "WZP trailing or missing payload bytes"); return -1; }
    }
    memset(sign, 0, (((size_t)n + 31) / 32) * 4);
    for (g = 0; g < groups; ++g) {
        size_t cursor = spans[g].offset;
        for (c = g * GROUP; c < chunks && c < (g + 1) * GROUP; ++c) {
            const uint32_t first = c * CHUNK, count = n - first < CHUNK ? n - first : CHUNK;
            uint16_t* m = mag + first;
            const uint8_t* src = payload + cursor;
            uint32_t mb, sb, nnz = 0, rank = 0;
            int raw;
            chunk_sizes(get24(meta + 3 * (size_t)c), count, &mb, &sb, &raw);
            if (!mb) { memset(m, 0, 2 * (size_t)count); continue; }
            if (raw) {
                for (i = 0; i < count; ++i) m[i] = (uint16_t)(src[2 * i] | (src[2 * i + 1] << 8));
            } else {
                if (rze_decode(src, mb, 2 * count, planes)) { free(spans); say(err, errlen, "WZP malformed RZE stream"); return -1; }
                bit_planes_inverse(planes, count, m);
            }
            for (i = 0; i < count; ++i) nnz += m[i] != 0;
            if (!nnz || (nnz + 7) / 8 != sb) { free(spans); say(err, errlen, "WZP compact sign length does not match nonzero magnitudes"); return -1; }
            if ((nnz & 7) && (src[mb + sb - 1] >> (nnz & 7))) { free(spans); say(err, errlen, "WZP nonzero compact sign padding"); return -1; }
            for (i = 0; i < count; ++i) {
                const uint32_t at = first + i;
                if (!m[i]) continue;
                sign[at >> 5] |= (uint32_t)((src[mb + (rank >> 3)] >> (rank & 7)) & 1) << (at & 31);
                ++rank;
            }
            cursor += mb + sb;
        }
    }
    free(spans);
    return 0;
}

/* Strict bound of a corrected value: |value - original| <= bound evaluated on
 * the exact real difference. The double difference and its rounding error
 * (a two-difference split) decide ties (cpu/src/repair_avx2.cpp:48-55). */
static int within_bound(double value, double original, double bound) {
    const double diff = value - original;
    const double m = fabs(diff);
    double vpart, opart, err;
    if (!isfinite(diff) || m > bound) return 0;
    if (m < bound) return 1;
    vpart = value - diff;                 /* the part of `value` that diff used */
    opart = diff + vpart;
    err = (value - opart) + (vpart - original); /* diff + err == value - original exactly */
    return !((diff > 0 && err > 0) || (diff < 0 && err < 0));
}

/* Compact repair section checks (cpu/src/codec.cpp:305-316): header,
 * groups, step and every group's span inside the payload. */
static int popc32(uint32_t v) { int c = 0; while (v) { v &= v - 1; ++c; } return c; }
static int wpw_validate(const uint8_t* sec, size_t bytes, uint32_t np, size_t width, char* err, size_t errlen) {
    const uint32_t groups = (np + 31) / 32;
    const size_t prefix = 24 + 8 * (size_t)groups;
    double step;
    size_t payload;
    uint32_t g;
    if (bytes < prefix || get32(sec) != 0x31575057u || get32(sec + 4) != groups || get64(sec + 8) != bytes - prefix) {
        say(err, errlen, "invalid WPW1 directory"); return -1;
    }
    payload = bytes - prefix;
    { uint64_t u = get64(sec + 16); memcpy(&step, &u, 8); }
    if (!(step > 0) || !isfinite(step)) { say(err, errlen, "invalid compact repair step"); return -1; }
    for (g = 0; g < groups; ++g) {
        const uint32_t off = get32(sec + 24 + 8 * (size_t)g), mask = get32(sec + 28 + 8 * (size_t)g);
        const uint32_t count = np - g * 32 < 32 ? np - g * 32 : 32;
        const size_t start = off & 0x7fffffffu;
        const size_t span = (off >> 31) ? count * width : (count + width - 1) / width * width + (size_t)popc32(mask) * width;
        if (count < 32 && (mask >> count)) { say(err, errlen, "invalid compact repair mask"); return -1; }
        if (start % 8 || start > payload || span > payload - start) { say(err, errlen, "invalid compact repair group span"); return -1; }
    }
    return 0;
}

/* ------------------------------------------------------ typed codec parts */

#define REAL float
#define SFX f32
#define FMA fmaf
#define FABS fabsf
#include "waltz_oracle_real.inc"
#undef REAL
#undef SFX
#undef FMA
#undef FABS

#define REAL double
#define SFX f64
#define FMA fma
#define FABS fabs
#include "waltz_oracle_real.inc"
#undef REAL
#undef SFX
#undef FMA
#undef FABS

/* -------------------------------------------------------------- public API */

int wo_transform(void* data, int width, uint32_t nx, uint32_t ny, uint32_t nz,
                 unsigned lxy, unsigned lz, int dyadic, int inverse) {
    const uint32_t full[3] = {nx, ny, nz};
    if (!nx || !ny || !nz) return -1;
    return width == 4 ? transform_f32((float*)data, full, lxy, lz, dyadic, inverse)
                      : transform_f64((double*)data, full, lxy, lz, dyadic, inverse);
}

long long wo_quantize(void* coeff, int width, uint32_t nx, uint32_t ny, uint32_t nz, unsigned bz,
                      double quantum, uint16_t* mag, uint32_t* sign,
                      uint32_t* qidx, uint32_t* qval, char* err, size_t errlen) {
    const uint32_t d[3] = {nx, ny, nz};
    uint16_t* ranks = build_ranks(d, bz);
    long long r;
    if (!ranks) { say(err, errlen, "out of memory"); return -1; }
    if (width == 4) r = quantize_emit_f32((float*)coeff, d, bz, (float)quantum, (float)(1.0 / quantum), mag, sign, qidx, qval, ranks);
    else r = quantize_emit_f64((double*)coeff, d, bz, quantum, 1.0 / quantum, mag, sign, qidx, qval, ranks);
    free(ranks);
    if (r < 0) say(err, errlen, "coefficient exceeds portable integer conversion domain");
    return r;
}

static int check_config(const wo_config* c, int encoding, char* err, size_t errlen) {
    uint64_t n;
    if (!c || !c->nx || !c->ny || !c->nz) { say(err, errlen, "nonzero dimensions required"); return -1; }
    if (c->width != 4 && c->width != 8) { say(err, errlen, "type must be FP32 or FP64"); return -1; }
    if (encoding && (!(c->abs_error > 0) || !isfinite(c->abs_error))) { say(err, errlen, "positive finite absolute error required"); return -1; }
    n = (uint64_t)c->nx * c->ny * c->nz;
    if (n > 0xffffffffull / (unsigned)c->width) { say(err, errlen, "volume exceeds WLT2 section limits"); return -1; }
    return 0;
}

size_t wo_max_compressed_bytes(const wo_config* c) {
    size_t n;
    if (check_config(c, 1, NULL, 0)) return 0;
    n = (size_t)c->nx * c->ny * c->nz;
    return 32 + pad8(wo_wzp_max_bytes((uint32_t)n)) + 2 * pad8(n * 4) + pad8(n * 4) + pad8(n * (size_t)c->width);
}

int wo_compress(const wo_config* c, const void* input, uint8_t* archive, size_t capacity,
                size_t* written, char* err, size_t errlen) {
    if (written) *written = 0;
    if (!input || !archive || !written) { say(err, errlen, "null argument"); return -1; }
    if (check_config(c, 1, err, errlen)) return -1;
    return c->width == 4 ? encode_f32(c, (const float*)input, archive, capacity, written, err, errlen)
                         : encode_f64(c, (const double*)input, archive, capacity, written, err, errlen);
}

int wo_decompress(const wo_config* c, const uint8_t* archive, size_t bytes, void* output,
                  size_t output_bytes, char* err, size_t errlen) {
    if (!archive || !output) { say(err, errlen, "null argument"); return -1; }
    if (check_config(c, 0, err, errlen)) return -1;
    if (output_bytes < (size_t)c->nx * c->ny * c->nz * (size_t)c->width) { say(err, errlen, "output capacity too small"); return -1; }
    return c->width == 4 ? decode_f32(c, archive, bytes, (float*)output, err, errlen)
                         : decode_f64(c, archive, bytes, (double*)output, err, errlen);
}

int wo_compact_repairs(const uint8_t* archive, size_t bytes, int width, const void* original, double step,
                       uint8_t* out, size_t capacity, size_t* written, char* err, size_t errlen) {
    uint32_t np, nq;
    size_t pi, pv, qi, qv, end, section, sec8, qb;
    uint64_t wb;
    uint8_t* tmp;
    if (written) *written = 0;
    if (!archive || !original || !out || !written || bytes < 32 || (width != 4 && width != 8) || !(step > 0)) {
        say(err, errlen, "invalid argument"); return -1;
    }
    wb = get64(archive + 16); np = get32(archive + 24); nq = get32(archive + 28);
    pi = 32 + pad8((size_t)wb); pv = pi + pad8((size_t)np * 4); qi = pv + pad8((size_t)np * width);
    qv = qi + pad8((size_t)nq * 4); end = qv + pad8((size_t)nq * 4);
    if ((archive[0] & 2) || end != bytes || capacity < bytes) { say(err, errlen, "not a native archive"); return -1; }
    tmp = (uint8_t*)calloc((size_t)np * width + 64, 1);
    if (!tmp) { say(err, errlen, "out of memory"); return -1; }
    section = np ? (width == 4 ? wpw_pack_f32(archive + pi, archive + pv, np, (const float*)original, step, tmp)
                               : wpw_pack_f64(archive + pi, archive + pv, np, (const double*)original, step, tmp))
                 : 0;
    if (!section) {
        memcpy(out, archive, bytes);
        *written = bytes;
        free(tmp);
        return 0;
    }
    sec8 = pad8(section);
    qb = pad8((size_t)nq * 4);
    memmove(out, archive, pv);
    out[0] |= 2;
    put32(out + 4, (uint32_t)section);
    memcpy(out + pv, tmp, section);
    memset(out + pv + section, 0, sec8 - section);
    memmove(out + pv + sec8, archive + qi, 2 * qb);
    *written = pv + sec8 + 2 * qb;
    free(tmp);
    return 0;
}

// Waltz B200 pipeline driver and C ABI.
//
// Compress (default profile, src/waltz.cu:327-609 of the reference):
//   forward all-level lifting -> quantise + Morton reorder -> WZP encode
//   (decoupled lookback, writes the archive in place) -> inverse lifting with
//   the repair emitter on the finest level -> ordered compaction of repairs
//   and q-outliers straight into their archive sections -> header.
// Decompress (src/waltz.cu:612-834): header checks -> WZP decode fused with
// dequantisation and the row-major scatter -> q-outlier patches -> inverse
// lifting -> repair patches. Every status is gathered in one device word and
// read at the call's single synchronisation point.
#include "common.cuh"
#include "compact.cuh"
#include "inverse.cuh"
#include "launch.cuh"
#include "ops.cuh"
#include "quantize.cuh"
#include "stage.cuh"
#include "stream.cuh"
#include "transform.cuh"
#include "wzp.cuh"
#include "xylevel.cuh"
#include "zlevel.cuh"
#include "zmatrix.cuh"

#include "../../include/waltz_b200.h"
#include "../../include/waltz_cuda.h"
#include "../../include/waltz_gpu_batch.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

namespace wb {

// ---------------------------------------------------------------- workspace
// Grow-only device arena per host thread (and device). Content never
// outlives a call; geometry tables are cached separately.
class Arena {
    int device_ = -1;
    char* base_ = nullptr;
    size_t cap_ = 0;

  public:
    ~Arena() { release(); }
    void release() {
        if (base_) {
            int prev = 0;
            if (cudaGetDevice(&prev) == cudaSuccess) {
                cudaSetDevice(device_);
                cudaFree(base_);
                cudaSetDevice(prev);
            }
        }
        base_ = nullptr;
        cap_ = 0;
    }
    char* reserve(size_t bytes) {
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        if (dev != device_ || bytes > cap_) {
            release();
            device_ = dev;
            check(cudaMalloc(&base_, std::max<size_t>(bytes, 256)), "Waltz: cannot allocate device workspace");
            cap_ = std::max<size_t>(bytes, 256);
        }
        return base_;
    }
};

struct Carver {
    char* base;
    size_t used = 0;
    template <class V> V* take(size_t count) {
        used = (used + 255) & ~size_t(255);
        V* p = reinterpret_cast<V*>(base ? base + used : nullptr);
        used += std::max<size_t>(count, 1) * sizeof(V);
        return p;
    }
};

// ----------------------------------------------------------- Morton tables
static uint32_t morton_rank(uint32_t x, uint32_t y, uint32_t z, uint32_t nx, uint32_t ny, uint32_t nz) {
    uint32_t rank = 0;
    while (nx > 1 || ny > 1 || nz > 1) {
        const uint32_t lx = nx - nx / 2, ly = ny - ny / 2, lz = nz - nz / 2;
        const bool ux = x >= lx, uy = y >= ly, uz = z >= lz;
        const uint32_t hz = uz ? nz / 2 : lz, hy = uy ? ny / 2 : ly;
        if (uz) rank += lz * nx * ny;
        if (uy) rank += hz * ly * nx;
        if (ux) rank += hz * hy * lx;
        if (ux) x -= lx;
        if (uy) y -= ly;
        if (uz) z -= lz;
        nx = ux ? nx / 2 : lx;
        ny = hy;
        nz = hz;
    }
    return rank;
}

// 8 slots x 256*bz entries; slot bits: short x edge, short y edge, short z
// edge. forward: local row-major index -> rank; inverse: rank -> packed local
// coordinates x | y << 4 | z << 8.
static std::vector<uint16_t> morton_tables(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t bz, bool inverse) {
    const uint32_t stride = 256 * bz;
    std::vector<uint16_t> t(8 * stride, 0);
    for (unsigned s = 0; s < 8; ++s) {
        const uint32_t ex = (s & 1) ? nx % 16 : 16, ey = (s & 2) ? ny % 16 : 16, ez = (s & 4) ? nz % bz : bz;
        for (uint32_t z = 0; z < ez; ++z)
            for (uint32_t y = 0; y < ey; ++y)
                for (uint32_t x = 0; x < ex; ++x) {
                    const uint32_t local = (z * ey + y) * ex + x;
                    const uint32_t r = morton_rank(x, y, z, ex, ey, ez);
                    if (inverse) t[s * stride + r] = uint16_t(x | (y << 4) | (z << 8));
                    else t[s * stride + local] = uint16_t(r);
                }
    }
    return t;
}

struct TableCache {
    int device = -1;
    uint32_t nx = 0, ny = 0, nz = 0, bz = 0;
    bool inverse = false;
    uint16_t* ptr = nullptr;
    ~TableCache() {
        if (ptr) cudaFree(ptr);
    }
    const uint16_t* get(uint32_t x, uint32_t y, uint32_t z, uint32_t b, bool inv, cudaStream_t stream) {
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        if (ptr && dev == device && x == nx && y == ny && z == nz && b == bz && inv == inverse) return ptr;
        if (ptr && dev != device) ptr = nullptr; // belongs to another device's context; keep it alive
        if (!ptr) check(cudaMalloc(&ptr, 8 * kChunk * sizeof(uint16_t)), "Waltz: cannot allocate Morton table");
        const auto host = morton_tables(x, y, z, b, inv);
        check(cudaMemcpyAsync(ptr, host.data(), host.size() * 2, cudaMemcpyHostToDevice, stream), "Morton table upload");
        check(cudaStreamSynchronize(stream), "Morton table upload");
        device = dev;
        nx = x; ny = y; nz = z; bz = b; inverse = inv;
        return ptr;
    }
};

// ------------------------------------------------------------ level plans
struct Geometry {
    uint32_t nx, ny, nz;
    uint64_t n;
    unsigned lxy, lz, bz;
    bool dyadic;
    Dims dyad[5], xyl[5], zl[5];
    static Geometry make(uint32_t nx, uint32_t ny, uint32_t nz) {
        Geometry g{};
        g.nx = nx; g.ny = ny; g.nz = nz;
        g.n = uint64_t(nx) * ny * nz;
        g.lxy = levels_of(std::min(nx, ny));
        g.lz = levels_of(nz);
        g.dyadic = g.lxy == g.lz;
        g.bz = zband_of(nx, ny, nz, g.lz, g.dyadic);
        Dims a{nx, ny, nz};
        for (unsigned l = 0; l < 5; ++l) {
            g.dyad[l] = a;
            a = {half_len(a.x), half_len(a.y), half_len(a.z)};
        }
        a = {nx, ny, nz};
        for (unsigned l = 0; l < 5; ++l) {
            g.xyl[l] = a;
            a = {half_len(a.x), half_len(a.y), a.z};
        }
        a = {nx, ny, nz};
        for (unsigned l = 0; l < 5; ++l) {
            g.zl[l] = a;
            a = {a.x, a.y, half_len(a.z)};
        }
        return g;
    }
    uint8_t flags(unsigned width) const { return uint8_t((dyadic ? 1 : 0) | (width == 8 ? 4 : 0) | (3u << 3)); }
};

__host__ __device__ inline uint64_t vol(Dims d) { return uint64_t(d.x) * d.y * d.z; }
static inline Dims halve(Dims d, int mask) {
    return {(mask & AX) ? half_len(d.x) : d.x, (mask & AY) ? half_len(d.y) : d.y, (mask & AZ) ? half_len(d.z) : d.z};
}

// Tile shapes per schedule (UX, UY, UZ).
template <class T> struct Tiles;
template <> struct Tiles<float> {
    static constexpr int XYZ[3] = {32, 8, 16};
    static constexpr int XY[3] = {32, 16, 4};
    static constexpr int Z[3] = {32, 8, 16};
};
template <> struct Tiles<double> {
    static constexpr int XYZ[3] = {16, 8, 8};
    static constexpr int XY[3] = {32, 16, 4};
    static constexpr int Z[3] = {32, 8, 8};
};

// Tuning options of the calling thread (performance only: results do not
// depend on them; set through waltz_b200_set_option).
struct Options {
    bool stage_kernels = true; // plane schedule: whole-stage kernels where they fit
    uint32_t zmarch = 0;       // forward z-march planes per CTA: 0 = automatic
    uint64_t small_level = uint64_t(1) << 15; // inverse levels of at most this many samples: direct staging
    uint64_t small_fwd = uint64_t(1) << 20;   // forward levels of at most this many samples: direct staging,
                                              // short z ranges (measured on 128^3 .. 512^3 fields)
    uint32_t repair_scale = 0; // compact repair section (WPW1) with step eb / scale: 0 (off), 16 or 64
    uint32_t xy_march = 0;     // plane schedule: XY levels as the warp march instead of the staged kernels
                               // (bit 0: forward levels, bit 1: inverse levels)
    uint64_t small_march = 0;  // dyadic inverse levels of at most this many samples: Z march + XY march
    uint64_t small_march_fwd = 0; // dyadic forward levels of at most this many samples: XY march + Z march
};
static thread_local Options t_opt;

template <class T, bool Inverse, int Mask, int UX, int UY, int UZ, class Src, class Out>
static void launch_level(const Src& src, Dims a, const Out& out, Sink& sink) {
    using Op = LevelOp<T, Inverse, Mask, UX, UY, UZ, Src, Out>;
    constexpr size_t smem = level_smem<T, Inverse, Mask, UX, UY, UZ>();
    const Dims grid{(a.x + UX - 1) / UX, (a.y + UY - 1) / UY, (a.z + UZ - 1) / UZ};
    const uint64_t blocks = uint64_t(grid.x) * grid.y * grid.z;
    need(blocks < (1ull << 31), "Waltz: level grid too large");
    sink.run<Op>(typename Op::Params{src, a, grid, out}, uint32_t(blocks), smem);
}

template <class T, bool Inverse, int Mask, class Src, class Out>
static void level(const Src& src, Dims a, const Out& out, Sink& sink) {
    if constexpr (Mask == (AX | AY | AZ))
        launch_level<T, Inverse, Mask, Tiles<T>::XYZ[0], Tiles<T>::XYZ[1], Tiles<T>::XYZ[2]>(src, a, out, sink);
    else if constexpr (Mask == (AX | AY))
        launch_level<T, Inverse, Mask, Tiles<T>::XY[0], Tiles<T>::XY[1], Tiles<T>::XY[2]>(src, a, out, sink);
    else
        launch_level<T, Inverse, Mask, Tiles<T>::Z[0], Tiles<T>::Z[1], Tiles<T>::Z[2]>(src, a, out, sink);
}

// One Z level of the plane schedule as a per-column register march
// (ZMarchOp): a warp per 32 columns and run of windows. A single field's
// runs are halved until the level has about 32 warps per SM (a run's first
// window reloads the 4 pairs it shares with the run before); many fields fill
// the GPU together, so each keeps whole columns.
template <class T, bool Inverse, class Src, class Out>
static void level_z(const Src& src, Dims a, const Out& out, Sink& sink) {
    using Op = ZMarchOp<T, Inverse, Src, Out>;
    using Sh = ZMarchShape<T, Inverse>;
    const uint32_t wins = (a.z + Sh::W - 1) / Sh::W, tx = (a.x + 31) / 32;
    const uint64_t cols = uint64_t(tx) * a.y;
    uint32_t seg = wins;
    if (!sink.many)
        while (seg > 1 && cols * ((wins + seg - 1) / seg) < 148ull * 32) seg = (seg + 1) / 2;
    const uint64_t warps = cols * ((wins + seg - 1) / seg);
    const uint64_t blocks = (warps + Op::kThreads / 32 - 1) / (Op::kThreads / 32);
    need(blocks < (1ull << 31), "Waltz: level grid too large");
    sink.run<Op>(typename Op::Params{src, a, out, seg, tx}, uint32_t(blocks));
}

// One XY level of the plane schedule as a warp march (XYMarchOp, taken with
// WALTZ_B200_OPT_XY_MARCH): a warp per strip of 24 x, plane and run of Y
// windows; runs halved for a single field until the level has about 32
// warps per SM, as for the Z levels.
template <class T, bool Inverse, class Src, class Out>
static void level_xy(const Src& src, Dims a, const Out& out, Sink& sink) {
    using Op = XYMarchOp<T, Inverse, Src, Out>;
    using Sh = XYMarchShape<T, Inverse>;
    const uint32_t wins = (a.y + Sh::W - 1) / Sh::W, tx = (a.x + Sh::U - 1) / Sh::U;
    const uint64_t strips = uint64_t(tx) * a.z;
    uint32_t seg = wins;
    if (!sink.many)
        while (seg > 1 && strips * ((wins + seg - 1) / seg) < 148ull * 32) seg = (seg + 1) / 2;
    const uint64_t warps = strips * ((wins + seg - 1) / seg);
    const uint64_t blocks = (warps + Op::kThreads / 32 - 1) / (Op::kThreads / 32);
    need(blocks < (1ull << 31), "Waltz: level grid too large");
    sink.run<Op>(typename Op::Params{src, a, out, seg, tx}, uint32_t(blocks));
}

// Resident CTAs of a kernel per SM times the SM count, cached per device.
template <class K> static uint64_t resident_slots(K kernel, size_t smem, int threads = 256) {
    static thread_local int cached_dev = -1;
    static thread_local uint64_t slots = 0;
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (cached_dev != dev) {
        int sms = 0, occ = 0;
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem), "occupancy");
        slots = uint64_t(sms) * uint64_t(occ > 0 ? occ : 1);
        cached_dev = dev;
    }
    return slots;
}

// One dyadic forward level as a z-march: XY tiles, and the z axis split into
// ranges only as far as needed to give every resident CTA slot work (one
// range per column tile when many fields share the GPU). Planes are staged by
// TMA when the source rows meet the copy engine's alignment.
template <class T, bool Z, int NT>
static void level_fwd_stream_nt(const FwdSrc<T>& src, Dims a, const FwdOut<T>& out, uint32_t* status, Sink& sink) {
    constexpr int UX = StreamTile<T>::UX, UY = StreamTile<T>::UY, Q = StreamTile<T>::Q;
    using S = StreamShape<T, UX, UY, Q, NT>;
    using OpT = FwdStreamOp<T, UX, UY, Q, true, Z, NT>;
    using OpL = FwdStreamOp<T, UX, UY, Q, false, Z, NT>;
    typename OpT::Params p{};
    // small levels: almost every tile is an edge tile, whose reflected cells
    // the TMA path fixes up one by one; direct staging reflects on load
    const bool small = vol(a) <= t_opt.small_fwd;
    const bool tma = !small && make_map_3d<T>(&p.map, src.p, a.x, a.y, a.z, src.sy, src.sz, S::FX, S::FY, 1);
    const uint32_t tx = (a.x + UX - 1) / UX, ty = (a.y + UY - 1) / UY;
    const uint64_t tiles = uint64_t(tx) * ty;
    const uint32_t min_range = small || !Z ? 8 : 16;
    // planes a z range re-reads besides its own: the z halo of the pipeline
    // (none for an XY level, whose ranges only repeat the CTA's set-up)
    const double reread = Z ? 8.0 : 1.0;
    uint32_t zrange = a.z + (a.z & 1);
    if (Z && t_opt.zmarch) {
        zrange = std::min(zrange, std::max<uint32_t>(16, t_opt.zmarch + (t_opt.zmarch & 1)));
    } else if (!sink.many) {
        // maximise (filled share of the last wave) x (planes kept out of the
        // 8-plane halo a range re-reads), over up to 16 ranges of >= 16 planes
        // (>= 8 for small levels, which are latency-bound)
        static thread_local int device = -1;
        static thread_local size_t granted = 0;
        opt_in_smem(op_kernel_for<OpT>(), S::smem, device, granted);
        const uint64_t slots = resident_slots(op_kernel_for<OpT>(), S::smem);
        double best = -1;
        for (uint32_t k = 1; k <= 16; ++k) {
            uint32_t r = (a.z + k - 1) / k;
            r += r & 1;
            if (k > 1 && r < min_range) break;
            const uint64_t blocks = tiles * ((a.z + r - 1) / r);
            const double waves = double((blocks + slots - 1) / slots);
            const double score = double(blocks) / (waves * double(slots)) * double(r) / (double(r) + reread);
            if (score > best + 1e-9) {
                best = score;
                zrange = r;
            }
        }
    }
    if (!Z && sink.many) zrange = std::min<uint32_t>(zrange, 16); // many fields: XY ranges re-read no halo
    const uint64_t blocks = tiles * ((a.z + zrange - 1) / zrange);
    need(blocks < (1ull << 31), "Waltz: level grid too large");
    p.src = src;
    p.a = a;
    p.tiles_x = tx;
    p.tiles_y = ty;
    p.zrange = zrange;
    p.out = out;
    p.status = status;
    if (tma) {
        sink.run<OpT>(p, uint32_t(blocks), S::smem);
    } else {
        typename OpL::Params q{};
        q.src = src;
        q.a = a;
        q.tiles_x = tx;
        q.tiles_y = ty;
        q.zrange = zrange;
        q.out = out;
        q.status = status;
        sink.run<OpL>(q, uint32_t(blocks), S::smem);
    }
}

// Thread count of a z-march CTA: float dyadic levels of one field up to
// 2^24 samples run 512 threads per CTA, the rest 256.
template <class T, bool Z = true>
static void level_fwd_stream(const FwdSrc<T>& src, Dims a, const FwdOut<T>& out, uint32_t* status, Sink& sink) {
    if (sizeof(T) == 4 && Z && !sink.many && !sink.rec && vol(a) <= (uint64_t(1) << 24))
        level_fwd_stream_nt<T, Z, 512>(src, a, out, status, sink);
    else
        level_fwd_stream_nt<T, Z, 256>(src, a, out, status, sink);
}

// One dyadic inverse level from TMA-staged parity boxes when the coefficient
// rows meet the copy engine's alignment; the generic level kernel otherwise.
template <class T, class Out>
static void level_inv(const InvSrc<T>& src, Dims a, const Out& out, uint32_t* status, Sink& sink) {
    constexpr int UX = InvTile<T>::UX, UY = InvTile<T>::UY, UZ = InvTile<T>::UZ;
    using S = InvShape<T, UX, UY, UZ>;
    using Op = InvTileOp<T, UX, UY, UZ, Out>;
    typename Op::Params p{};
    bool tma = vol(a) > t_opt.small_level && half_len(a.x) % S::V == 0 &&
               make_map_3d<T>(&p.cmap, src.base, a.x, a.y, a.z, src.sy, src.sz, S::BX, S::HY, S::HZ);
    if (tma && src.low)
        tma = make_map_3d<T>(&p.lmap, src.low, src.lo.x, src.lo.y, src.lo.z, src.lo.x, uint64_t(src.lo.x) * src.lo.y,
                             S::BX, S::HY, S::HZ);
    if (!tma) {
        level<T, true, AX | AY | AZ>(src, a, out, sink);
        return;
    }
    const uint32_t tx = (a.x + UX - 1) / UX, ty = (a.y + UY - 1) / UY, tz = (a.z + UZ - 1) / UZ;
    const uint64_t blocks = uint64_t(tx) * ty * tz;
    need(blocks < (1ull << 31), "Waltz: level grid too large");
    p.lv = InvLevel<T>{src.base, src.sy, src.sz, src.low, src.lo, a};
    p.tiles_x = tx;
    p.tiles_y = ty;
    p.out = out;
    p.status = status;
    sink.run<Op>(p, uint32_t(blocks), S::smem);
}

// One small dyadic inverse level as two register marches: the Z synthesis
// (ZMarchOp, canonical folded windows) into `tmp` in the level's x/y split
// layout, then the X and Y synthesis (XYMarchOp, canonical Y windows of 8)
// to `out`. The passes are the tile inverse's Z, X and Y passes, sample for
// sample, so the bits are the same; a level whose tiles cannot fill the GPU
// takes thousands of short warps instead.
template <class T, class Out>
static void level_inv_march(const InvSrc<T>& src, Dims a, const Out& out, T* tmp, Sink& sink) {
    level_z<T, true>(src, a, StoreOut<T>{tmp, a.x, size_t(a.x) * a.y}, sink);
    level_xy<T, true>(InvSrc<T>{tmp, a.x, size_t(a.x) * a.y, nullptr, Dims{}}, a, out, sink);
}

// One inverse XY level of the plane schedule from TMA-staged parity boxes
// when the coefficient rows meet the copy engine's alignment; the generic
// level kernel otherwise.
template <class T, class Out>
static void level_inv_xy(const InvSrc<T>& src, Dims a, const Out& out, uint32_t* status, Sink& sink) {
    constexpr int UX = InvTileXY<T>::UX, UY = InvTileXY<T>::UY, UZ = InvTileXY<T>::UZ;
    using S = InvXYShape<T, UX, UY, UZ>;
    using Op = InvTileXYOp<T, UX, UY, UZ, Out>;
    typename Op::Params p{};
    bool tma = vol(a) > t_opt.small_level && half_len(a.x) % S::V == 0 &&
               make_map_3d<T>(&p.cmap, src.base, a.x, a.y, a.z, src.sy, src.sz, S::BX, S::HY, UZ);
    if (tma && src.low)
        tma = make_map_3d<T>(&p.lmap, src.low, src.lo.x, src.lo.y, src.lo.z, src.lo.x, uint64_t(src.lo.x) * src.lo.y,
                             S::BX, S::HY, UZ);
    if (!tma) {
        level<T, true, AX | AY>(src, a, out, sink);
        return;
    }
    const uint32_t tx = (a.x + UX - 1) / UX, ty = (a.y + UY - 1) / UY, tz = (a.z + UZ - 1) / UZ;
    const uint64_t blocks = uint64_t(tx) * ty * tz;
    need(blocks < (1ull << 31), "Waltz: level grid too large");
    p.lv = InvLevel<T>{src.base, src.sy, src.sz, src.low, src.lo, a};
    p.tiles_x = tx;
    p.tiles_y = ty;
    p.out = out;
    p.status = status;
    sink.run<Op>(p, uint32_t(blocks), S::smem);
}

// WZP encoder of one magnitude source: one CTA per 8192-sample chunk.
template <class Src>
static void launch_wzp_encode(const WzpEncodeArgs& wa, const Src& src, uint32_t chunks, Sink& sink) {
    sink.run<WzpEncodeOp<Src>>(typename WzpEncodeOp<Src>::Params{wa, src}, chunks, sizeof(WzpEncodeSmem));
}

template <class T, class Out> struct IdentityOp {
    static constexpr int kThreads = 256, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        const T* in;
        Dims d;
        Out out;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t block, uint32_t blocks) {
        const Dims d = P.d;
        const uint64_t n = vol(d);
        for (uint64_t i = block * uint64_t(kThreads) + threadIdx.x; i < n; i += uint64_t(blocks) * kThreads) {
            const uint32_t x = uint32_t(i % d.x), y = uint32_t((i / d.x) % d.y),
                           z = uint32_t(i / (uint64_t(d.x) * d.y));
            P.out(x, y, z, P.in[i]);
        }
    }
};

static unsigned grid_for(uint64_t n, unsigned threads = 256) {
    uint64_t b = (n + threads - 1) / threads;
    return unsigned(std::min<uint64_t>(std::max<uint64_t>(b, 1), 148ull * 64));
}

// ------------------------------------------------ whole-stage plane kernels
static StageLevels z_levels(const Geometry& g) {
    StageLevels lv{};
    lv.count = g.lz;
    for (unsigned l = 0; l < g.lz; ++l) lv.z[l] = g.zl[l].z;
    return lv;
}
static StageLevels xy_levels(const Geometry& g) {
    StageLevels lv{};
    lv.count = g.lxy;
    for (unsigned l = 0; l < g.lxy; ++l) {
        lv.x[l] = g.xyl[l].x;
        lv.y[l] = g.xyl[l].y;
    }
    return lv;
}
template <class T> static bool zstage_ok(const Geometry& g) {
    return t_opt.stage_kernels && g.lz && zstage_smem<T>(g.nz) <= kStageSmemCap;
}
template <class T> static bool xystage_ok(const Geometry& g) {
    return t_opt.stage_kernels && g.lxy && xystage_smem<T>(g.nx, g.ny) <= kStageSmemCap;
}

static unsigned zstage_grid(const Geometry& g, int cx, int cy) {
    return unsigned(((g.nx + cx - 1) / cx) * uint64_t((g.ny + cy - 1) / cy));
}

template <class T>
static void zstage_forward(const T* in, size_t sy, size_t sz, const Geometry& g, T* dst, uint32_t* status,
                           Sink& sink) {
    sink.run<ZStageFwdOp<T>>(typename ZStageFwdOp<T>::Params{in, sy, sz, g.nx, g.ny, g.nz, z_levels(g), dst, status},
                             zstage_grid(g, ZCols<T>::CX, ZCols<T>::CY), zstage_smem<T>(g.nz));
}

template <class T, class Out>
static void zstage_inverse(const T* coef, size_t sy, size_t sz, const Geometry& g, const Out& out, Sink& sink) {
    sink.run<ZStageInvOp<T, Out>>(typename ZStageInvOp<T, Out>::Params{coef, sy, sz, g.nx, g.ny, g.nz, z_levels(g), out},
                                  zstage_grid(g, ZCols<T>::CX, ZCols<T>::CY), zstage_smem<T>(g.nz));
}

template <class T>
static void xystage_forward(const T* in, size_t sy, size_t sz, const Geometry& g, T* dst, size_t dsy, size_t dsz,
                            uint32_t* status, Sink& sink) {
    sink.run<XYStageFwdOp<T>>(
        typename XYStageFwdOp<T>::Params{in, sy, sz, g.nx, g.ny, xy_levels(g), dst, dsy, dsz, status}, g.nz,
        xystage_smem<T>(g.nx, g.ny));
}

template <class T, class Out>
static void xystage_inverse(const T* coef, size_t sy, size_t sz, const Geometry& g, const Out& out, Sink& sink) {
    sink.run<XYStageInvOp<T, Out>>(typename XYStageInvOp<T, Out>::Params{coef, sy, sz, g.nx, g.ny, xy_levels(g), out},
                                   g.nz, xystage_smem<T>(g.nx, g.ny));
}

// Scratch element counts for the forward and inverse transforms.
struct TransformScratch {
    uint64_t low;   // each of two compact ping-pong buffers
    uint64_t inter; // full-size intermediate (plane schedule with both stages)
};
static TransformScratch scratch_need(const Geometry& g) {
    TransformScratch s{1, 0};
    if (g.dyadic) {
        for (unsigned l = 0; l < g.lxy; ++l) s.low = std::max(s.low, vol(halve(g.dyad[l], AX | AY | AZ)));
        for (unsigned l = 0; l < g.lxy; ++l) s.low = std::max(s.low, vol(g.dyad[l]) * (l > 0));
    } else {
        for (unsigned l = 0; l < g.lz; ++l) s.low = std::max(s.low, vol(halve(g.zl[l], AZ)));
        for (unsigned l = 0; l < g.lxy; ++l) s.low = std::max(s.low, vol(halve(g.xyl[l], AX | AY)));
        for (unsigned l = 1; l < g.lz; ++l) s.low = std::max(s.low, vol(g.zl[l]));
        for (unsigned l = 1; l < g.lxy; ++l) s.low = std::max(s.low, vol(g.xyl[l]));
        if (g.lz && g.lxy) s.inter = g.n;
    }
    return s;
}

template <class T, class Out>
static void zmatrix_apply(const T* x, uint32_t nx, uint32_t ny, uint32_t nz, bool inverse, int zsplit, const Out& out,
                          uint32_t* status, bool check_finite, Sink& sink);

// Forward all-level transform of `in` into the coefficient array C. With a
// split code `zsplit` (the precision form; plane schedule) the Z stage is the
// tensor-core matrix transform instead of Z lifting.
template <class T>
static void forward(const Geometry& g, const T* in, T* C, T* lowA, T* lowB, T* inter, uint32_t* status,
                    Sink& sink, int zsplit = 0) {
    const bool matrix = zsplit != 0;
    const size_t sy = g.nx, sz = size_t(g.nx) * g.ny;
    T* lows[2] = {lowA, lowB};
    if (g.lxy == 0 && g.lz == 0) {
        sink.run<CopyFiniteOp<T>>(typename CopyFiniteOp<T>::Params{in, C, g.n, status}, grid_for(g.n));
        return;
    }
    if (g.dyadic) {
        FwdSrc<T> src{in, sy, sz, status};
        for (unsigned l = 0; l < g.lxy; ++l) {
            const Dims a = g.dyad[l], lo = halve(a, AX | AY | AZ);
            const bool last = l + 1 == g.lxy;
            if (vol(a) <= t_opt.small_march_fwd) {
                // a small level as two marches: the Y and X analysis into
                // `inter` (x/y split, z spatial), then the Z analysis to C
                // and the compact low band (the z-march's Y, X, Z order)
                const size_t isy = a.x, isz = size_t(a.x) * a.y;
                level_xy<T, false>(src, a, FwdOut<T>{inter, isy, isz, nullptr, halve(a, AX | AY), a, AX | AY}, sink);
                level_z<T, false>(FwdSrc<T>{inter, isy, isz}, a,
                                  FwdOut<T>{C, sy, sz, last ? nullptr : lows[l & 1], lo, a, AZ}, sink);
            } else {
                FwdOut<T> out{C, sy, sz, last ? nullptr : lows[l & 1], lo, a, AX | AY | AZ};
                level_fwd_stream<T>(src, a, out, status, sink);
            }
            static const char* const kFwdNames[5] = {"fwd_l0", "fwd_l1", "fwd_l2", "fwd_l3", "fwd_l4"};
            sink.mark(kFwdNames[l]);
            src = FwdSrc<T>{lows[l & 1], lo.x, size_t(lo.x) * lo.y};
        }
        return;
    }
    FwdSrc<T> src{in, sy, sz, status};
    T* zdst = g.lxy ? inter : C;
    if (matrix) {
        zmatrix_apply<T>(in, g.nx, g.ny, g.nz, false, zsplit, ZmStore<T>{zdst}, status, true, sink);
        sink.mark("fwd_z_matrix");
    }
    const bool zstage = !matrix && zstage_ok<T>(g);
    if (zstage) zstage_forward<T>(in, sy, sz, g, zdst, status, sink);
    for (unsigned l = 0; l < (matrix || zstage ? 0u : g.lz); ++l) {
        const Dims a = g.zl[l], lo = halve(a, AZ);
        const bool last = l + 1 == g.lz;
        FwdOut<T> out{zdst, sy, sz, last ? nullptr : lows[l & 1], lo, a, AZ};
        level_z<T, false>(src, a, out, sink);
        src = FwdSrc<T>{lows[l & 1], lo.x, size_t(lo.x) * lo.y};
    }
    if (g.lz) sink.mark("fwd_z");
    if (g.lz) src = FwdSrc<T>{inter, sy, sz};
    if (xystage_ok<T>(g)) {
        xystage_forward<T>(src.p, sy, sz, g, C, sy, sz, g.lz ? nullptr : status, sink);
        sink.mark("fwd_xy");
        return;
    }
    for (unsigned l = 0; l < g.lxy; ++l) {
        const Dims a = g.xyl[l], lo = halve(a, AX | AY);
        const bool last = l + 1 == g.lxy;
        FwdOut<T> out{C, sy, sz, last ? nullptr : lows[l & 1], lo, a, AX | AY};
        if (t_opt.xy_march & 1u) level_xy<T, false>(src, a, out, sink);
        else level_fwd_stream<T, false>(src, a, out, status, sink);
        src = FwdSrc<T>{lows[l & 1], lo.x, size_t(lo.x) * lo.y};
    }
    if (g.lxy) sink.mark("fwd_xy");
}

// Largest compact low band the inverse keeps between two levels of one stage.
static uint64_t inverse_low_need(const Geometry& g) {
    uint64_t m = 0;
    if (g.dyadic) {
        for (unsigned l = 1; l < g.lxy; ++l) m = std::max(m, vol(g.dyad[l]));
    } else {
        for (unsigned l = 1; l < g.lxy; ++l) m = std::max(m, vol(g.xyl[l]));
    }
    return m;
}

// Inverse all-level transform within three banks of n samples: C (the
// coefficients, clobbered by the plane schedule once its XY stage is done),
// bank1 and bank2. Dyadic and XY-stage low bands ping-pong between the two
// halves of bank2; the plane schedule's XY output goes to bank1 and its Z
// stage ping-pongs between bank2 and the freed C (or bank1). The finest level
// hands every sample to `fin`.
template <class T, class Final>
static void inverse(const Geometry& g, T* C, T* bank1, T* bank2, const Final& fin, uint32_t* status,
                    Sink& sink, const char* final_stage = "inv_l0", int zsplit = 0) {
    const bool matrix = zsplit != 0;
    const size_t sy = g.nx, sz = size_t(g.nx) * g.ny;
    const uint64_t half_off = ((g.n + 1) / 2 + 63) & ~uint64_t(63);
    need(inverse_low_need(g) <= g.n - std::min(g.n, half_off), "Waltz: inverse scratch layout");
    T* halves[2] = {bank2, bank2 + half_off};
    if (g.lxy == 0 && g.lz == 0) {
        sink.run<IdentityOp<T, Final>>(typename IdentityOp<T, Final>::Params{C, Dims{g.nx, g.ny, g.nz}, fin},
                                       grid_for(g.n));
        return;
    }
    if (g.dyadic) {
        const T* low = nullptr;
        for (int l = int(g.lxy) - 1; l >= 0; --l) {
            const Dims a = g.dyad[l];
            InvSrc<T> src{C, sy, sz, low, halve(a, AX | AY | AZ)};
            // small levels: two marches through bank1 (unused by the dyadic
            // schedule) instead of the tile inverse
            const bool march = vol(a) <= t_opt.small_march;
            if (l > 0) {
                T* dst = halves[l & 1];
                const StoreOut<T> to{dst, a.x, size_t(a.x) * a.y};
                if (march) level_inv_march<T>(src, a, to, bank1, sink);
                else level_inv<T>(src, a, to, status, sink);
                low = dst;
                static const char* const kInvNames[5] = {"inv_l0", "inv_l1", "inv_l2", "inv_l3", "inv_l4"};
                sink.mark(kInvNames[l]);
            } else {
                if (march) level_inv_march<T>(src, a, fin, bank1, sink);
                else level_inv<T>(src, a, fin, status, sink);
                sink.mark(final_stage);
            }
        }
        return;
    }
    const T* zbase = C;
    T* zping[2] = {bank2, bank1};
    if (xystage_ok<T>(g)) {
        if (g.lz) {
            xystage_inverse<T>(C, sy, sz, g, StoreOut<T>{bank1, sy, sz}, sink);
            zbase = bank1;
            zping[1] = C;
        } else {
            xystage_inverse<T>(C, sy, sz, g, fin, sink);
        }
        sink.mark("inv_xy");
    } else if (g.lxy) {
        const T* low = nullptr;
        for (int l = int(g.lxy) - 1; l >= 0; --l) {
            const Dims a = g.xyl[l];
            InvSrc<T> src{C, sy, sz, low, halve(a, AX | AY)};
            if (l > 0) {
                T* dst = halves[l & 1];
                const StoreOut<T> to{dst, a.x, size_t(a.x) * a.y};
                if (t_opt.xy_march & 2u) level_xy<T, true>(src, a, to, sink);
                else level_inv_xy<T>(src, a, to, status, sink);
                low = dst;
            } else if (g.lz) {
                const StoreOut<T> to{bank1, sy, sz};
                if (t_opt.xy_march & 2u) level_xy<T, true>(src, a, to, sink);
                else level_inv_xy<T>(src, a, to, status, sink);
                zbase = bank1;
                zping[1] = C; // the coefficients are no longer read
            } else {
                if (t_opt.xy_march & 2u) level_xy<T, true>(src, a, fin, sink);
                else level_inv_xy<T>(src, a, fin, status, sink);
            }
        }
        sink.mark("inv_xy");
    }
    if (matrix && g.lz) {
        zmatrix_apply<T>(zbase, g.nx, g.ny, g.nz, true, zsplit, ZmEmit<T, Final>{fin, g.nx}, status, false, sink);
        sink.mark("inv_z_matrix");
        return;
    }
    if (zstage_ok<T>(g)) {
        zstage_inverse<T>(zbase, sy, sz, g, fin, sink);
        sink.mark("inv_z");
    } else if (g.lz) {
        const T* low = nullptr;
        for (int l = int(g.lz) - 1; l >= 0; --l) {
            const Dims a = g.zl[l];
            InvSrc<T> src{zbase, sy, sz, low, halve(a, AZ)};
            if (l > 0) {
                T* dst = zping[l & 1];
                level_z<T, true>(src, a, StoreOut<T>{dst, a.x, size_t(a.x) * a.y}, sink);
                low = dst;
            } else {
                level_z<T, true>(src, a, fin, sink);
            }
        }
        sink.mark("inv_z");
    }
}

// ------------------------------------------------ precision form: Z matrices
// Mz[n][k]: all Z levels of the forward transform of a unit column e_k, in
// double (the lifting of the symmetrically reflected line, the exact
// counterpart of the window lifting), coefficients in split-band order. Its
// inverse (the synthesis matrix) comes from Gauss-Jordan elimination.
static void lift_line_forward(std::vector<double>& v, uint32_t n) {
    constexpr int H = 8;
    const double A = -1.586134342059924, B = -0.052980118572961, G = 0.882911075530934, D = 0.443506852043971,
                 K = 1.1496043988602418;
    std::vector<double> x(n + 2 * H);
    for (int i = -H; i < int(n) + H; ++i) x[i + H] = v[mirror(i, n)];
    auto step = [&](int parity, double c) {
        for (int i = -H + 1; i < int(n) + H - 1; ++i)
            if (((i % 2) + 2) % 2 == parity) x[i + H] += c * (x[i + H - 1] + x[i + H + 1]);
    };
    step(1, A);
    step(0, B);
    step(1, G);
    step(0, D);
    const uint32_t h = half_len(n);
    for (uint32_t i = 0; i < n; ++i) {
        const double y = (i & 1) ? x[i + H] * (-1.0 / K) : x[i + H] * K;
        v[(i >> 1) + ((i & 1) ? h : 0)] = y;
    }
}

static std::vector<double> z_analysis_matrix(uint32_t nz) {
    const unsigned levels = levels_of(nz);
    std::vector<double> M(size_t(nz) * nz);
    for (uint32_t k = 0; k < nz; ++k) {
        std::vector<double> v(nz, 0.0);
        v[k] = 1.0;
        uint32_t len = nz;
        for (unsigned l = 0; l < levels; ++l) {
            std::vector<double> part(v.begin(), v.begin() + len);
            lift_line_forward(part, len);
            std::copy(part.begin(), part.end(), v.begin());
            len = half_len(len);
        }
        for (uint32_t r = 0; r < nz; ++r) M[size_t(r) * nz + k] = v[r];
    }
    return M;
}

static std::vector<double> invert_matrix(std::vector<double> a, uint32_t n) {
    std::vector<double> inv(size_t(n) * n, 0.0);
    for (uint32_t i = 0; i < n; ++i) inv[size_t(i) * n + i] = 1.0;
    for (uint32_t c = 0; c < n; ++c) {
        uint32_t piv = c;
        for (uint32_t r = c + 1; r < n; ++r)
            if (std::fabs(a[size_t(r) * n + c]) > std::fabs(a[size_t(piv) * n + c])) piv = r;
        need(std::fabs(a[size_t(piv) * n + c]) > 1e-12, "Waltz: singular Z transform matrix");
        for (uint32_t j = 0; j < n; ++j) {
            std::swap(a[size_t(c) * n + j], a[size_t(piv) * n + j]);
            std::swap(inv[size_t(c) * n + j], inv[size_t(piv) * n + j]);
        }
        const double d = a[size_t(c) * n + c];
        for (uint32_t j = 0; j < n; ++j) {
            a[size_t(c) * n + j] /= d;
            inv[size_t(c) * n + j] /= d;
        }
        for (uint32_t r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = a[size_t(r) * n + c];
            if (f == 0.0) continue;
            for (uint32_t j = 0; j < n; ++j) {
                a[size_t(r) * n + j] -= f * a[size_t(c) * n + j];
                inv[size_t(r) * n + j] -= f * inv[size_t(c) * n + j];
            }
        }
    }
    return inv;
}

// TF32 halves of a matrix in the K-major no-swizzle core layout of zmatrix_kernel.
static void pack_tf32_halves(const std::vector<double>& m, uint32_t nz, std::vector<float>& hi,
                             std::vector<float>& lo) {
    const ZmPlan P = ZmPlan::make(nz);
    hi.assign(size_t(P.np) * P.kp, 0.f);
    lo.assign(size_t(P.np) * P.kp, 0.f);
    for (uint32_t n = 0; n < P.np; ++n)
        for (uint32_t k = 0; k < P.kp; ++k) {
            const float v = (n < nz && k < nz) ? float(m[size_t(n) * nz + k]) : 0.f;
            uint32_t bits;
            std::memcpy(&bits, &v, 4);
            bits &= 0xffffe000u;
            float h;
            std::memcpy(&h, &bits, 4);
            const size_t at = (size_t(n / 8) * (P.kp / 4) + k / 4) * 32 + (n % 8) * 4 + (k % 4);
            hi[at] = h;
            lo[at] = v - h;
        }
}

// Bits of the bf16 nearest to v (round to nearest even; v finite).
static uint16_t host_bf16(double v) {
    const float f = float(v);
    uint32_t b;
    std::memcpy(&b, &f, 4);
    b += 0x7fffu + ((b >> 16) & 1u);
    return uint16_t(b >> 16);
}
static double host_bf16_value(uint16_t h) {
    const uint32_t b = uint32_t(h) << 16;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

// Slices of a matrix in the K-major no-swizzle core layouts of the slice
// kernels, slice after slice.
// BF16x3 (zmatrix_bf16_kernel): m = b0 + b1 + b2 (+ residual), each the bf16
//   of the remaining residual; core (n/8, k/8) at ((n/8) * kp/8 + k/8) * 64
//   elements, element (n%8, k%8) at (n%8) * 8 + k%8.
// Exact (zmatrix_exact_kernel): row n scaled by 2^-(f_n+1) (|m| < 2^f_n over
//   the row) and cut into five 7-bit integer slices (int8, |a| <= 64); core
//   (n/8, k/16) at ((n/8) * kp/16 + k/16) * 128 bytes, element (n%8, k%16) at
//   (n%8) * 16 + k%16; scale[n] = 2^(f_n + 1 - 14), the epilogue's row factor.
static void pack_bf16_slices(const std::vector<double>& m, uint32_t nz, std::vector<uint16_t>& out) {
    const ZsPlan P = ZsPlan::make(nz, false);
    const size_t per = size_t(P.np) * P.kp;
    out.assign(P.S * per, 0);
    for (uint32_t n = 0; n < P.np; ++n)
        for (uint32_t k = 0; k < P.kp; ++k) {
            const size_t at = (size_t(n / 8) * (P.kp / 8) + k / 8) * 64 + (n % 8) * 8 + (k % 8);
            double r = (n < nz && k < nz) ? m[size_t(n) * nz + k] : 0.0;
            for (uint32_t sl = 0; sl < P.S; ++sl) {
                const uint16_t h = host_bf16(r);
                out[sl * per + at] = h;
                r -= host_bf16_value(h);
            }
        }
}
static void pack_exact_slices(const std::vector<double>& m, uint32_t nz, std::vector<int8_t>& out,
                              std::vector<double>& scale) {
    const ZsPlan P = ZsPlan::make(nz, true);
    const size_t per = size_t(P.np) * P.kp;
    out.assign(P.S * per, 0);
    scale.assign(P.np, 0.0);
    for (uint32_t n = 0; n < nz; ++n) {
        double rmax = 0.0;
        for (uint32_t k = 0; k < nz; ++k) rmax = std::max(rmax, std::fabs(m[size_t(n) * nz + k]));
        int f = 0;
        if (rmax > 0) std::frexp(rmax, &f); // rmax < 2^f
        scale[n] = std::ldexp(1.0, f + 1 - 14);
        for (uint32_t k = 0; k < nz; ++k) {
            const size_t at = (size_t(n / 8) * (P.kp / 16) + k / 16) * 128 + (n % 8) * 16 + (k % 16);
            double u = std::ldexp(m[size_t(n) * nz + k], -(f + 1));
            for (uint32_t sl = 0; sl < P.S; ++sl) {
                const double a = std::nearbyint(u * 128.0);
                u = u * 128.0 - a;
                out[sl * per + at] = int8_t(a);
            }
        }
    }
}

// Device copies of the Z matrices per column length and split form, kept
// until exit: a captured graph may hold their addresses. TF32x3: the hi and
// lo halves of the analysis and synthesis matrices; bf16 forms: their slices
// (and row scales).
struct ZMatrixCache {
    struct Entry {
        uint32_t nz;
        int split;
        void* dev;
        size_t bytes[2];  // per direction: operand bytes, then scale bytes
        size_t off[2][2]; // [inverse][0 operand, 1 scales]
    };
    int device = -1;
    std::vector<Entry> entries;
    ~ZMatrixCache() {
        for (auto& e : entries) cudaFree(e.dev);
    }
    const Entry& get(uint32_t n, int split, cudaStream_t stream) {
        int d = 0;
        check(cudaGetDevice(&d), "cudaGetDevice");
        if (d != device) {
            entries.clear(); // matrices of another device's context stay allocated there
            device = d;
        }
        for (auto& e : entries)
            if (e.nz == n && e.split == split) return e;
        const std::vector<double> M = z_analysis_matrix(n), Sy = invert_matrix(M, n);
        std::vector<unsigned char> all;
        Entry e{n, split, nullptr, {0, 0}, {{0, 0}, {0, 0}}};
        auto append = [&](const void* p, size_t bytes) {
            const size_t at = (all.size() + 255) / 256 * 256;
            all.resize(at + bytes);
            std::memcpy(all.data() + at, p, bytes);
            return at;
        };
        for (int inv = 0; inv < 2; ++inv) {
            const std::vector<double>& mat = inv ? Sy : M;
            if (split == kZsTf32x3) {
                std::vector<float> hi, lo;
                pack_tf32_halves(mat, n, hi, lo);
                hi.insert(hi.end(), lo.begin(), lo.end());
                e.off[inv][0] = append(hi.data(), hi.size() * 4);
            } else if (split == kZsBf16x3) {
                std::vector<uint16_t> sl;
                pack_bf16_slices(mat, n, sl);
                e.off[inv][0] = append(sl.data(), sl.size() * 2);
            } else {
                std::vector<int8_t> sl;
                std::vector<double> sc;
                pack_exact_slices(mat, n, sl, sc);
                e.off[inv][0] = append(sl.data(), sl.size());
                e.off[inv][1] = append(sc.data(), sc.size() * 8);
            }
        }
        check(cudaMalloc(&e.dev, all.size()), "Waltz: cannot allocate Z matrices");
        check(cudaMemcpyAsync(e.dev, all.data(), all.size(), cudaMemcpyHostToDevice, stream), "Z matrix upload");
        check(cudaStreamSynchronize(stream), "Z matrix upload");
        entries.push_back(e);
        return entries.back();
    }
};
static thread_local ZMatrixCache t_zmat;

// Applies the all-levels Z analysis (or synthesis) matrix to a z-major float
// or double field of nx*ny columns on the tensor cores, in the arithmetic of
// split form `zsplit`; `out.group` takes every result. nz <= 128 (96 for the
// exact slices), nx*ny a multiple of 4.
template <class K>
static void zmatrix_launch(K kernel, uint32_t smem, uint32_t smem_max, uint64_t ncols, cudaStream_t stream,
                           unsigned& grid, uint32_t tmem_cols) {
    static thread_local std::vector<std::pair<const void*, int>> configured;
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    const void* key = reinterpret_cast<const void*>(kernel);
    bool seen = false;
    for (auto& c : configured)
        if (c.first == key && c.second == dev) seen = true;
    if (!seen) {
        check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_max)),
              "matrix kernel shared memory");
        // the whole unified L1 as shared memory, so that two CTAs of up to
        // ~113 KB share an SM
        check(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   int(cudaSharedmemCarveoutMaxShared)),
              "matrix kernel carveout");
        configured.emplace_back(key, dev);
    }
    const uint64_t tiles = (ncols + kZmCols - 1) / kZmCols;
    // resident CTAs at this column length's shared memory: the runtime's
    // answer, or the count the SM's shared memory and the two-CTA register
    // budget allow (__launch_bounds__(256, 2)), whichever is larger. A CTA
    // that does not fit waits for a free SM: the CTAs never wait on one
    // another, so a larger grid costs nothing but a second wave.
    int sms = 0, occ = 0, smem_sm = 0, reserved = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kZmThreads, smem), "occupancy");
    check(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev), "shared memory per SM");
    check(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev), "reserved shared memory");
    const int by_smem = smem_sm / int(smem + uint32_t(reserved));
    // ... and never more CTAs than the SM's 512 tensor-memory columns hold
    const int by_tmem = int(512 / std::max<uint32_t>(tmem_cols, 32));
    const int per_sm = std::min(std::max(occ, std::min(by_smem, 2)), std::max(by_tmem, 1));
    const uint64_t slots = uint64_t(sms) * uint64_t(per_sm > 0 ? per_sm : 1);
    grid = unsigned(std::min<uint64_t>(tiles, slots));
}

template <class T, class Out>
static void zmatrix_apply(const T* x, uint32_t nx, uint32_t ny, uint32_t nz, bool inverse, int zsplit, const Out& out,
                          uint32_t* status, bool check_finite, Sink& sink) {
    need(nz >= 1 && nz <= uint32_t(kZmMaxK), "Waltz: matrix form needs 1 <= nz <= 128");
    need(zsplit != kZsExact || nz <= uint32_t(kZsExactMaxK), "Waltz: the exact slice form needs nz <= 96");
    const uint64_t ncols = uint64_t(nx) * ny;
    const ZMatrixCache::Entry& e = t_zmat.get(nz, zsplit, sink.stream);
    const unsigned char* base = static_cast<const unsigned char*>(e.dev);
    const int dir = inverse ? 1 : 0;
    const uint32_t cf = check_finite ? 1u : 0u;
    // no batched form: every field keeps its own persistent launch
    if (zsplit == kZsTf32x3) {
        const ZmPlan P = ZmPlan::make(nz);
        const float* bhi = reinterpret_cast<const float*>(base + e.off[dir][0]);
        const float* blo = bhi + size_t(P.np) * P.kp;
        // float fields: planes staged by TMA (the plane stride meets the copy
        // engine's 16-byte rule because nx * ny is a multiple of 4)
        if constexpr (sizeof(T) == 4) {
            const ZmTmaPlan Q = ZmTmaPlan::make(nz);
            CUtensorMap xmap;
            if (make_map_3d<float>(&xmap, x, ncols, nz, 1, ncols, ncols * nz, kZmCols, Q.kc, 1)) {
                sink.direct([=](cudaStream_t stream) {
                    auto kernel = zmatrix_tma_kernel<Out>;
                    unsigned grid = 0;
                    zmatrix_launch(kernel, Q.smem(), ZmTmaPlan::make(kZmMaxK).smem(), ncols, stream, grid,
                                   Q.np <= 32 ? 32u : (Q.np <= 64 ? 64u : 128u));
                    kernel<<<grid, kZmThreads, Q.smem(), stream>>>(xmap, bhi, blo, nz, ncols, out, status, cf);
                    note_launch();
                    check(cudaGetLastError(), "matrix kernel launch");
                });
                return;
            }
        }
        sink.direct([=](cudaStream_t stream) {
            auto kernel = zmatrix_kernel<T, Out>;
            unsigned grid = 0;
            zmatrix_launch(kernel, P.smem(), ZmPlan::make(kZmMaxK).smem(), ncols, stream, grid,
                           P.np <= 32 ? 32u : (P.np <= 64 ? 64u : 128u));
            kernel<<<grid, kZmThreads, P.smem(), stream>>>(x, bhi, blo, nz, ncols, out, status, cf);
            note_launch();
            check(cudaGetLastError(), "matrix kernel launch");
        });
        return;
    }
    const bool exact = zsplit == kZsExact;
    need(zsplit == kZsBf16x3 || exact, "Waltz: unknown matrix split form");
    const ZsPlan P = ZsPlan::make(nz, exact);
    const unsigned char* bsl = base + e.off[dir][0];
    const double* bscale = reinterpret_cast<const double*>(base + e.off[dir][1]);
    sink.direct([=](cudaStream_t stream) {
        unsigned grid = 0;
        if (exact) {
            auto kernel = zmatrix_exact_kernel<T, Out>;
            zmatrix_launch(kernel, P.smem(), ZsPlan::make(kZsExactMaxK, true).smem(), ncols, stream, grid, 512u);
            kernel<<<grid, kZmThreads, P.smem(), stream>>>(x, reinterpret_cast<const int8_t*>(bsl), bscale, nz, ncols,
                                                           out, status, cf);
        } else {
            auto kernel = zmatrix_bf16_kernel<T, Out>;
            zmatrix_launch(kernel, P.smem(), ZsPlan::make(kZmMaxK, false).smem(), ncols, stream, grid,
                           P.np <= 32 ? 32u : (P.np <= 64 ? 64u : 128u));
            kernel<<<grid, kZmThreads, P.smem(), stream>>>(x, reinterpret_cast<const uint16_t*>(bsl), nz, ncols, out,
                                                           status, cf);
        }
        note_launch();
        check(cudaGetLastError(), "matrix kernel launch");
    });
}

size_t capacity_for(uint64_t n, unsigned width) {
    const uint64_t pwe = std::min<uint64_t>(n, 1ull << 22), qout = std::min<uint64_t>(n, 1ull << 20);
    return size_t(n * width + pwe * (4 + width) + qout * 8 + (1ull << 20));
}

static thread_local Arena t_arena;
static thread_local TableCache t_fwd_tables, t_inv_tables;
static thread_local uint64_t* t_pinned = nullptr; // small pinned readback slots

static uint64_t* pinned() {
    if (!t_pinned) check(cudaMallocHost(&t_pinned, 64 * sizeof(uint64_t)), "pinned readback");
    return t_pinned;
}

struct EncodeOptions {
    uint32_t spin_cap = 1u << 22;
    uint32_t skip_publish = 0xffffffffu;
    int zsplit = kZsNone; // precision form: tensor-core Z transform in this split form (header flag bits)
    uint32_t repair_scale = t_opt.repair_scale; // the calling thread's compact repair setting
};

// Header flag bit 6 (reserved in the reference header,
// include/utils/Blob.hpp:38-53, so the reference decoders reject such
// archives and the default bytes stay): the archive's Z stage is the
// tensor-core matrix form. Its split form (0 TF32x3, 1 BF16x3, 2 exact
// slices) is then stored in the two top bits of header byte 3, the z band,
// which needs six bits (1..32). Flag bit 5 keeps the reference's meaning (its
// CUDA fused plane-Z profile, which this decoder does not take).
constexpr uint8_t kMatrixFlag = 0x40;
static uint8_t split_flags(int zsplit) { return zsplit ? kMatrixFlag : uint8_t(0); }
static uint8_t split_band(int zsplit, uint32_t bz) {
    return uint8_t(bz | (zsplit ? uint32_t(zsplit - 1) << 6 : 0u));
}
// Split form of an archive (kZsNone for lifting; 4 for the undefined code).
static int split_of(uint8_t flags, uint8_t band) {
    if (!(flags & kMatrixFlag)) return kZsNone;
    return 1 + int(band >> 6);
}

// Fields the matrix form serves: float or double, plane schedule with Z
// levels, 1 <= nz <= 128 (96 for the exact slices) and nx*ny a multiple of 4.
static bool matrix_form_ok(const Geometry& g, size_t width, int zsplit = kZsTf32x3) {
    const uint32_t kmax = zsplit == kZsExact ? uint32_t(kZsExactMaxK) : uint32_t(kZmMaxK);
    return zsplit >= kZsTf32x3 && zsplit <= kZsExact && (width == 4 || width == 8) && !g.dyadic && g.lz >= 1 &&
           g.nz <= kmax && (uint64_t(g.nx) * g.ny) % 4 == 0;
}

// ------------------------------------------------------------------ encode
// One compression: validated arguments, its scratch plan, the enqueued
// kernels and the interpretation of the 9 result words (layout[0..7] and the
// status word) that the last kernels leave in scratch. Split so that a batch
// can enqueue many of them (inside one CUDA graph) and read all results once.
template <class T> struct CompressJob {
    const T* in;
    uint32_t nx, ny, nz;
    double eb;
    uint8_t* out;
    size_t capacity;
    EncodeOptions opt;
    Geometry g;
    uint64_t n;

    struct Plan {
        T *C, *lowA, *lowB, *inter, *bank2, *perr;
        uint16_t* mag;
        uint32_t *sign, *qbits, *qval, *pbits, *status, *ticket, *counts_p, *counts_q;
        uint64_t *state, *sizes, *wzp_total, *layout; // layout[8] = status copy
        uint32_t* wpw_groups;  // compact repairs: per group bytes, then offsets
        uint64_t* wpw_state;
        uint8_t* wpw_tail;     // the compact section and the moved q-outlier sections
    };
    // Compact repairs: record and group capacities of this field.
    uint64_t repair_cap() const { return std::min<uint64_t>(n, uint64_t(1) << 22); }
    uint64_t outlier_cap() const { return std::min<uint64_t>(n, uint64_t(1) << 20); }

    static CompressJob make(const T* d_in, uint32_t nx, uint32_t ny, uint32_t nz, double eb, uint8_t* d_out,
                            size_t capacity, const EncodeOptions& opt) {
        need(nx && ny && nz, "Waltz: nonzero dimensions required");
        const uint64_t n = uint64_t(nx) * ny * nz;
        need(n <= 0xffffffffull / sizeof(T), "Waltz: volume exceeds the archive section limits");
        need(d_in && d_out, "Waltz: null buffer");
        const double quantum = 1.5 * eb;
        const T q = T(quantum), inv = T(1.0 / quantum);
        need(eb > 0 && std::isfinite(eb) && std::isfinite(quantum) && q > T(0) && std::isfinite(q) &&
                 std::isfinite(inv),
             "Waltz: invalid bound (positive finite, representable quantum required)");
        {
            const uintptr_t a = reinterpret_cast<uintptr_t>(d_in), b = reinterpret_cast<uintptr_t>(d_out);
            need(!(a < b + capacity && b < a + n * sizeof(T)), "Waltz: input and output buffers overlap");
        }
        need(capacity >= 32 + wzp_header(uint32_t(n)), "Waltz: archive capacity too small");
        CompressJob j{d_in, nx, ny, nz, eb, d_out, capacity, opt, Geometry::make(nx, ny, nz), n};
        need(!opt.zsplit || matrix_form_ok(j.g, sizeof(T), opt.zsplit),
             "Waltz: the matrix form needs the plane schedule with 1 <= nz <= 128 (96 for the exact slices) and nx*ny "
             "a multiple of 4");
        return j;
    }

    Plan plan(Carver& c) const {
        const TransformScratch ts = scratch_need(g);
        const uint32_t chunks = wzp_chunks(uint32_t(n));
        const uint64_t words = (n + 31) / 32, cblocks = (words + kCompactWords - 1) / kCompactWords;
        Plan p;
        p.C = c.take<T>(n);
        p.lowA = c.take<T>(ts.low);
        p.lowB = c.take<T>(ts.low);
        p.inter = c.take<T>(n);
        p.bank2 = c.take<T>(n);
        p.perr = c.take<T>(n);
        p.mag = c.take<uint16_t>(n + 8);
        p.qval = c.take<uint32_t>(n);
        // zero-initialised block (one memset): bitmaps, status, ticket, lookback states
        p.sign = c.take<uint32_t>(words + 1);
        p.qbits = c.take<uint32_t>(words + 1);
        p.pbits = c.take<uint32_t>(words + 1);
        p.status = c.take<uint32_t>(1);
        p.ticket = c.take<uint32_t>(1);
        p.state = c.take<uint64_t>(chunks);
        p.counts_p = c.take<uint32_t>(cblocks);
        p.counts_q = c.take<uint32_t>(cblocks);
        p.sizes = c.take<uint64_t>(chunks);
        p.wzp_total = c.take<uint64_t>(1);
        p.layout = c.take<uint64_t>(9);
        p.wpw_groups = nullptr;
        p.wpw_state = nullptr;
        p.wpw_tail = nullptr;
        if (opt.repair_scale) {
            p.wpw_groups = c.take<uint32_t>((repair_cap() + 31) / 32 + 1);
            p.wpw_state = c.take<uint64_t>(8);
            p.wpw_tail = c.take<uint8_t>(repair_cap() * sizeof(T) + 2 * pad8(outlier_cap() * 4) + 64);
        }
        return p;
    }
    size_t scratch_bytes() const {
        Carver c{nullptr};
        plan(c);
        return c.used;
    }

    // Enqueues every kernel of the compression on `stream` (nothing syncs).
    // Enqueues every stage of the compression into `sink` (nothing syncs).
    // The 9 result words go to `results` (default: inside the scratch).
    void enqueue(char* scratch, const uint16_t* rank, Sink& sink, uint64_t* results = nullptr) const {
        Carver cv{scratch};
        const Plan P = plan(cv);
        uint64_t* const layout = results ? results : P.layout;
        const double quantum = 1.5 * eb;
        const T q = T(quantum), inv = T(1.0 / quantum);
        const uint32_t chunks = wzp_chunks(uint32_t(n));
        const uint64_t words = (n + 31) / 32, cblocks = (words + kCompactWords - 1) / kCompactWords;
        sink.phase(PH_INIT);
        sink.zero(P.sign, reinterpret_cast<char*>(P.state + chunks) - reinterpret_cast<char*>(P.sign));

        if (!sink.rec) stage_clock().begin(sink.stream);
        // 1. forward transform
        sink.phase(PH_FORWARD);
        forward<T>(g, in, P.C, P.lowA, P.lowB, P.inter, P.status, sink, opt.zsplit);
        // 2. quantisation + Morton reorder: a field made of whole bricks (2^k
        // samples each) is quantised inside the WZP encoder, chunk by chunk;
        // otherwise a separate pass writes the Morton-packed magnitudes and
        // signs first.
        const uint32_t bsz = 256 * g.bz;
        const bool fused = nx % 16 == 0 && ny % 16 == 0 && nz % g.bz == 0 && (bsz & (bsz - 1)) == 0 && bsz <= kChunk;
        if (!fused) {
            sink.phase(PH_QUANT);
            QuantArgs<T> qa{P.C, Bricks::make(nx, ny, nz, g.bz), rank, q, inv, P.mag, P.sign, P.qbits, P.qval, P.status};
            const uint64_t bricks = qa.b.count();
            need(bricks < (1ull << 31), "Waltz: brick grid too large");
            sink.run<QuantizeOp<T>>(qa, uint32_t(bricks));
            sink.mark("quantize");
        }
        // 3. WZP encode straight into the archive
        {
            sink.phase(PH_ENCODE);
            WzpEncodeArgs wa{uint32_t(n), out + 32, capacity - 32, P.ticket, P.state, P.sizes, P.status, opt.spin_cap,
                             opt.skip_publish};
            if (fused) {
                uint32_t lb = 0;
                while ((1u << lb) < bsz) ++lb;
                launch_wzp_encode(wa, QuantBricks<T>{P.C, nx, ny, g.bz, lb, rank, q, inv, P.qbits, P.qval, P.status},
                                  chunks, sink);
            } else {
                launch_wzp_encode(wa, MagArrays{P.mag, P.sign}, chunks, sink);
            }
            sink.phase(PH_DIRECTORY);
            const uint32_t groups = wzp_groups(uint32_t(n));
            sink.run<WzpDirectoryOp>(WzpDirectoryOp::Params{out + 32, uint32_t(n), P.state, P.sizes, P.wzp_total},
                                     (groups + 255) / 256);
        }
        sink.mark("wzp_encode");
        // 4. inverse transform + repairs; fast-accept threshold of the repair
        // check (float): eb * (1 - 2^-21), rounded down
        {
            sink.phase(PH_INVERSE);
            T safe = T(eb * (1.0 - std::ldexp(1.0, -21)));
            if (double(safe) > eb * (1.0 - std::ldexp(1.0, -21))) safe = std::nextafter(safe, T(0));
            RepairOut<T> fin{in, nx, size_t(nx) * ny, eb, T(eb), P.pbits, P.perr, P.status, safe};
            inverse<T>(g, P.C, P.inter, P.bank2, fin, P.status, sink, "inv_l0_repair", opt.zsplit);
        }
        // 5. ordered side records
        sink.phase(PH_SIDE);
        const uint32_t both = uint32_t(2 * cblocks);
        sink.run<CompactCountOp>(CompactCountOp::Params{P.pbits, P.qbits, words, P.counts_p, P.counts_q,
                                                        uint32_t(cblocks)},
                                 both);
        sink.run<ScanLayoutOp>(ScanLayoutOp::Params{P.counts_p, P.counts_q, uint32_t(cblocks), P.wzp_total, P.status,
                                                    out, capacity, uint32_t(sizeof(T)),
                                                    uint8_t(g.flags(sizeof(T)) | split_flags(opt.zsplit)),
                                                    uint8_t(g.lxy), uint8_t(g.lz), split_band(opt.zsplit, g.bz), quantum, layout},
                               1);
        sink.run<CompactWriteOp<T>>(typename CompactWriteOp<T>::Params{P.pbits, P.qbits, words, P.counts_p,
                                                                       P.counts_q, P.perr, P.qval, out, layout, n,
                                                                       uint32_t(cblocks)},
                                    both);
        // 6. compact repair section (opt-in WPW1 profile), from the ordered
        // native records just written; every grid is fixed by the field's
        // record capacity (the counts are on the device)
        if (opt.repair_scale) {
            const double step = eb / double(opt.repair_scale);
            const uint64_t groups = (repair_cap() + 31) / 32;
            const uint32_t gblocks = uint32_t(std::min<uint64_t>((groups + 7) / 8, 148 * 8));
            sink.run<WpwSizeOp<T>>(typename WpwSizeOp<T>::Params{layout, out, in, step, P.wpw_groups},
                                   std::max(gblocks, 1u));
            sink.run<WpwScanOp>(WpwScanOp::Params{layout, out, P.wpw_groups, P.wpw_state, uint32_t(sizeof(T)), step},
                                1);
            sink.run<WpwWriteOp<T>>(typename WpwWriteOp<T>::Params{layout, out, in, step, P.wpw_groups, P.wpw_state,
                                                                   P.wpw_tail},
                                    std::max(gblocks, 1u));
            const uint64_t tail = repair_cap() * sizeof(T) + 2 * pad8(outlier_cap() * 4);
            sink.run<WpwMoveOp>(WpwMoveOp::Params{layout, P.wpw_state, P.wpw_tail, out},
                                uint32_t(std::min<uint64_t>((tail / 8 + 255) / 256 + 1, 148 * 8)));
        }
        sink.mark("side_records");
    }

    // Device address of the 9 result words inside this job's scratch.
    uint64_t* result(char* scratch) const {
        Carver cv{scratch};
        return plan(cv).layout;
    }

    // Interprets the 9 result words; returns the archive size or throws.
    size_t finish(const uint64_t* h) const {
        const uint32_t status = uint32_t(h[8]);
        const uint64_t np = h[5], nq = h[6];
        if (status & ST_NONFINITE_INPUT) throw Error("nonfinite input is unsupported");
        if (status & ST_MATRIX_RANGE) throw Error("Waltz: the matrix form needs samples within the float range");
        if (status & ST_QUANT_DOMAIN) throw Error("coefficient exceeds portable integer conversion domain");
        if (status & ST_BOUND) throw Error("native repair cannot meet strict bound or nonfinite reconstruction");
        if (status & ST_LOOKBACK_TIMEOUT) throw Error("Waltz: WZP lookback wait exceeded its bound");
        if (status & ST_WAIT_TIMEOUT) throw Error("Waltz: asynchronous copy wait exceeded its bound");
        if (status & ST_CAPACITY) throw Error("archive capacity too small");
        if ((n > (1u << 20) && nq >= (1u << 20)) || (n > (1u << 22) && np >= (1u << 22)))
            throw Error("portable GPU side-channel capacity reached");
        if (h[7]) throw Error("archive capacity too small");
        return size_t(h[4]);
    }
};

template <class T>
static size_t compress(const T* d_in, uint32_t nx, uint32_t ny, uint32_t nz, double eb, uint8_t* d_out,
                       size_t capacity, cudaStream_t stream, const EncodeOptions& opt = EncodeOptions()) {
    const CompressJob<T> job = CompressJob<T>::make(d_in, nx, ny, nz, eb, d_out, capacity, opt);
    char* scratch = t_arena.reserve(job.scratch_bytes());
    const uint16_t* rank = t_fwd_tables.get(nx, ny, nz, job.g.bz, false, stream);
    Sink sink{stream};
    job.enqueue(scratch, rank, sink);
    uint64_t* h = pinned();
    check(cudaMemcpyAsync(h, job.result(scratch), 9 * 8, cudaMemcpyDeviceToHost, stream), "readback");
    check(cudaStreamSynchronize(stream), "compress");
    return job.finish(h);
}

// ------------------------------------------------------------------ decode
struct Header {
    uint8_t flags, lxy, lz, bz;
    int split;
    uint32_t pwe_bytes;
    double q;
    uint64_t wzp;
    uint32_t np, nq;
    static Header parse(const uint8_t* p) {
        Header h;
        h.flags = p[0]; h.lxy = p[1]; h.lz = p[2]; h.bz = p[3];
        // matrix-form archives keep their split code in the band's top bits
        h.split = split_of(h.flags, h.bz);
        if (h.split) h.bz &= 0x3f;
        std::memcpy(&h.pwe_bytes, p + 4, 4);
        std::memcpy(&h.q, p + 8, 8);
        std::memcpy(&h.wzp, p + 16, 8);
        std::memcpy(&h.np, p + 24, 4);
        std::memcpy(&h.nq, p + 28, 4);
        return h;
    }
};

struct Layout {
    uint64_t pi, pv, qi, qv, end;
};

// Archive length implied by the header's section sizes (BlobLayout of
// include/utils/Blob.hpp:62-90): header, WZP stream, repair indices and
// values, q-outlier indices and values, each padded to 8 bytes. Sizes beyond
// the format's limits give a length the header checks then reject.
static uint64_t archive_end(const Header& h) {
    if (h.wzp > (uint64_t(1) << 60)) return 0;
    return 32 + pad8(h.wzp) + pad8(uint64_t(h.np) * 4) + pad8(h.pwe_bytes) + 2 * pad8(uint64_t(h.nq) * 4);
}

// Header checks of the reference CPU decoder (cpu/src/codec.cpp:276-293);
// `canonical` adds the exact-profile checks of src/waltz.cu:631-646.
template <class T>
static Layout validate_header(const Header& h, const Geometry& g, size_t bytes, bool canonical) {
    const uint64_t n = g.n;
    need(bytes >= 32, "invalid Waltz archive header");
    const int zsplit = h.split;
    need(!(h.flags & 0xa0) && (h.flags & 0x18) && ((h.flags & 4) ? 8u : 4u) == sizeof(T),
         "invalid Waltz archive header");
    need(!zsplit || matrix_form_ok(g, sizeof(T), zsplit), "invalid Waltz archive header");
    need(((h.flags >> 3) & 3) == 3, "unsupported Waltz synthesis mode");
    const bool compact = (h.flags & 2) != 0; // WPW1 repair section (cpu/src/codec.cpp:280-293)
    const bool dyadic = h.flags & 1;
    need(h.lxy <= 5 && h.lz <= 5 && h.bz >= 1 && h.bz <= 32 && !(dyadic && h.lxy != h.lz), "invalid levels or z band");
    need(h.lxy == g.lxy && h.lz == g.lz, "dimensions/levels mismatch");
    const T q = T(h.q);
    need(h.q > 0 && std::isfinite(h.q) && q > T(0) && std::isfinite(q), "invalid quantum");
    need(h.np <= n && h.nq <= n, "invalid section counts");
    need(h.wzp <= (uint64_t(1) << 60), "Waltz archive size overflow");
    Layout L;
    L.pi = 32 + pad8(h.wzp);
    L.pv = L.pi + pad8(uint64_t(h.np) * 4);
    L.qi = L.pv + pad8(h.pwe_bytes);
    L.qv = L.qi + pad8(uint64_t(h.nq) * 4);
    L.end = L.qv + pad8(uint64_t(h.nq) * 4);
    need(L.end == bytes, "truncated archive or trailing data");
    if (compact)
        need(h.np > 0 && uint64_t(h.pwe_bytes) >= kWpwHeader + uint64_t(kWpwEntry) * ((uint64_t(h.np) + 31) / 32) &&
                 uint64_t(h.pwe_bytes) < uint64_t(h.np) * sizeof(T),
             "invalid compact correction section");
    else
        need(uint64_t(h.pwe_bytes) == uint64_t(h.np) * sizeof(T), "invalid native correction section");
    need(h.wzp >= wzp_header(uint32_t(n)) && h.wzp <= wzp_max_bytes(uint32_t(n)), "WZP archive size is outside its valid bounds");
    need(h.bz == g.bz, "invalid Waltz reorder z-band");
    if (canonical) {
        need(h.flags == g.flags(sizeof(T)) && dyadic == g.dyadic, "invalid canonical Waltz chunk shape, header or length");
    }
    need(dyadic == g.dyadic, "dimensions/levels mismatch");
    return L;
}

// Directory check: group spans must tile the payload exactly. The fast path
// verifies canonical (increasing) order on the device; anything else is
// checked on the host like cpu/src/wzp_cpu.cpp:720-761.
struct DirectoryCheckOp {
    static constexpr int kThreads = 1024, kMinBlocks = 0; // no occupancy floor: the compiler picks the register budget
    struct Params {
        JobRef job;
        uint32_t n;
        uint32_t* status;
    };
    static __device__ __forceinline__ void run(const Params P, uint32_t, uint32_t);
};

__device__ __forceinline__ void DirectoryCheckOp::run(const Params P, uint32_t, uint32_t) {
    const uint32_t n = P.n;
    uint32_t* const status = P.status;
    const JobRef& job = P.job;
    __shared__ uint32_t tmp[40];
    const DecodeJob J = job.get();
    const uint8_t* in = J.base + 32;
    const uint64_t payload = J.wzp - wzp_header(n);
    const uint32_t chunks = wzp_chunks(n), groups = wzp_groups(n);
    const uint8_t* meta = in + size_t(groups) * 4;
    uint64_t carry = 0;
    uint32_t st = 0;
    for (uint32_t base = 0; base < groups; base += kThreads) {
        const uint32_t g = base + threadIdx.x;
        uint32_t len = 0, off = 0;
        if (g < groups) {
            // the group's 16 metadata words are independent loads: all in flight at once
#pragma unroll
            for (uint32_t k = 0; k < kGroup; ++k) {
                const uint32_t c = g * kGroup + k;
                if (c >= chunks) break;
                const WzpChunkInfo ci = wzp_meta(load_u24(meta + size_t(c) * 3), min(kChunk, n - c * kChunk));
                if (!ci.ok) st |= ST_BAD_STREAM;
                len += ci.mbytes + ci.sbytes;
            }
            off = load_u32(in + size_t(g) * 4);
            if (off > payload || len > payload - off || (!len && off)) st |= ST_BAD_STREAM;
        }
        uint32_t sum;
        const uint32_t ex = block_excl_scan<kThreads>(len, tmp, sum);
        if (g < groups && len && uint64_t(off) != carry + ex) st |= ST_DIRECTORY;
        carry += sum;
    }
    if (threadIdx.x == 0 && carry != payload) st |= ST_DIRECTORY;
    if (st) atomicOr(status, st);
}

static void host_directory_check(const uint8_t* in, uint32_t n, uint64_t payload) {
    const uint32_t chunks = wzp_chunks(n), groups = wzp_groups(n);
    std::vector<std::pair<uint32_t, uint32_t>> spans;
    for (uint32_t g = 0; g < groups; ++g) {
        uint32_t len = 0;
        for (uint32_t c = g * kGroup; c < std::min(chunks, (g + 1) * kGroup); ++c) {
            const uint8_t* m = in + size_t(groups) * 4 + size_t(c) * 3;
            const uint32_t meta = m[0] | (m[1] << 8) | (m[2] << 16);
            const uint32_t count = std::min(kChunk, n - c * kChunk), code = meta & kRawCode, sc = meta >> 14;
            if (!code) {
                need(!sc, "WZP zero chunk carries sign metadata");
                continue;
            }
            const bool raw = code == kRawCode;
            need(raw || (code >= 4 && code + 2 < 2 * count), "WZP invalid compressed magnitude length");
            const uint32_t sb = sc ? sc : 1024;
            need(sb <= (count + 7) / 8, "WZP sign stream exceeds the chunk size");
            len += (raw ? 2 * count : code) + sb;
        }
        uint32_t off;
        std::memcpy(&off, in + size_t(g) * 4, 4);
        need(off <= payload && len <= payload - off && (len || !off), "WZP directory range is outside the payload");
        if (len) spans.push_back({off, len});
    }
    std::sort(spans.begin(), spans.end());
    uint64_t cursor = 0;
    for (auto& s : spans) {
        need(s.first == cursor, "WZP payload groups overlap or leave a gap");
        cursor += s.second;
    }
    need(cursor == payload, "WZP trailing or missing payload bytes");
}

static DecodeJob decode_job(const uint8_t* d_in, const Header& h, const Layout& L, void* out = nullptr) {
    return DecodeJob{d_in, h.wzp, L.pi, L.pv, L.qi, L.qv, h.q, h.np, h.nq, out, h.pwe_bytes, (h.flags & 2u) != 0 ? 1u : 0u};
}

// Decoder kernels of one archive, launched without synchronising. Scratch:
// C, bank1, bank2 of n samples each and the inverse Morton table. With
// `job.ptr` set (graph capture) the side-record kernels are always launched
// on a fixed grid, as the counts are only known on the device.
template <class T, class Final, class Patch>
static void decode_launch(const JobRef& job, int zsplit, const Geometry& g, const uint16_t* irank,
                          const uint16_t* frank, T* C, T* bank1,
                          T* bank2, const Final& fin, const Patch& patch, uint32_t* status, Sink& sink) {
    const uint32_t n = uint32_t(g.n);
    if (!sink.rec) stage_clock().begin(sink.stream);
    sink.phase(PH_DCHECK);
    sink.run<DirectoryCheckOp>(DirectoryCheckOp::Params{job, n, status}, 1);
    {
        sink.phase(PH_DECODE);
        BrickMap map{g.nx, g.ny, g.nz, g.bz, irank, frank, false, 0};
        const uint32_t bsz = 256 * g.bz;
        if (g.nx % 16 == 0 && g.ny % 16 == 0 && g.nz % g.bz == 0 && (bsz & (bsz - 1)) == 0 && bsz <= kChunk &&
            kChunk / bsz <= 32) {
            map.fast = true;
            while ((1u << map.lb) < bsz) ++map.lb;
        }
        sink.run<WzpDecodeOp<T>>(WzpDecodeArgs<T>{job, n, map, C, status}, wzp_chunks(n), sizeof(WzpDecodeSmem));
    }
    sink.mark("wzp_decode");
    const uint32_t fixed = uint32_t(std::min<uint64_t>((g.n + 255) / 256, 32));
    if (job.ptr || job.val.nq) {
        sink.phase(PH_QPATCH);
        sink.run<QPatchOp<T>>(typename QPatchOp<T>::Params{job, g.n, C, status},
                              job.ptr ? fixed : (job.val.nq + 255) / 256);
    }
    sink.mark("qpatch");
    sink.phase(PH_DINVERSE);
    inverse<T>(g, C, bank1, bank2, fin, status, sink, "inv_l0", zsplit);
    if (job.ptr || job.val.np) {
        sink.phase(PH_RPATCH);
        sink.run<RPatchOp<T, Patch>>(typename RPatchOp<T, Patch>::Params{job, g.n, patch, status},
                                     job.ptr ? fixed : (job.val.np + 255) / 256);
    }
    sink.mark("rpatch");
}

// Status word -> exception, with the exact checks that need the host: a
// non-canonical WZP directory order and unordered side-record lists.
template <class T>
static void decode_finish(uint32_t status, const uint8_t* d_in, const Header& h, const Layout& L, const Geometry& g,
                          uint32_t* d_status, uint32_t* seen, cudaStream_t stream) {
    uint64_t* pin = pinned();
    const uint64_t header = wzp_header(uint32_t(g.n));
    if (status & ST_DIRECTORY) {
        std::vector<uint8_t> dir(header);
        check(cudaMemcpy(dir.data(), d_in + 32, header, cudaMemcpyDeviceToHost), "directory readback");
        host_directory_check(dir.data(), uint32_t(g.n), h.wzp - header);
        status &= ~ST_DIRECTORY;
    }
    if (status & ST_UNORDERED) {
        // Unsorted side records are valid when their indices are distinct.
        const uint64_t words = (g.n + 31) / 32;
        check(cudaMemsetAsync(d_status, 0, 4, stream), "memset");
        for (int k = 0; k < 2; ++k) {
            const uint32_t cnt = k ? h.nq : h.np;
            if (cnt < 2) continue;
            check(cudaMemsetAsync(seen, 0, (words + 1) * 4, stream), "memset");
            duplicate_kernel<<<(cnt + 255) / 256, 256, 0, stream>>>(d_in + (k ? L.qi : L.pi), cnt, seen, d_status); note_launch();
        }
        check(cudaMemcpyAsync(pin + 9, d_status, 4, cudaMemcpyDeviceToHost, stream), "readback");
        check(cudaStreamSynchronize(stream), "duplicate check");
        status = (status & ~ST_UNORDERED) | uint32_t(pin[9]);
    }
    if (status & ST_BAD_STREAM) throw Error("malformed WZP stream");
    if (status & ST_BAD_INDEX) throw Error("invalid or duplicate outlier index");
    if (status & ST_BAD_QOUT) throw Error("invalid quantization outlier");
    if (status & ST_BAD_REPAIR) throw Error("nonfinite correction");
    if (status & ST_NONFINITE_INPUT) throw Error("nonfinite reconstruction");
    if (status & ST_WAIT_TIMEOUT) throw Error("Waltz: asynchronous copy wait exceeded its bound");
}

template <class T>
static void decompress(const uint8_t* d_in, size_t bytes, uint32_t nx, uint32_t ny, uint32_t nz, T* d_out,
                       size_t out_bytes, cudaStream_t stream, bool canonical, const uint8_t* host_copy) {
    need(nx && ny && nz, "Waltz: nonzero dimensions required");
    const uint64_t n = uint64_t(nx) * ny * nz;
    need(n <= 0xffffffffull / sizeof(T), "Waltz: volume exceeds the archive section limits");
    need(d_in && d_out, "Waltz: null buffer");
    need(out_bytes >= n * sizeof(T), "output capacity too small");
    need(bytes >= 32 || (bytes == 0 && !canonical), "invalid Waltz archive header");
    const Geometry g = Geometry::make(nx, ny, nz);
    Header h;
    uint64_t* pin = pinned();
    if (host_copy) {
        h = Header::parse(host_copy);
    } else {
        check(cudaMemcpyAsync(pin, d_in, 32, cudaMemcpyDeviceToHost, stream), "header readback");
        check(cudaStreamSynchronize(stream), "header readback");
        h = Header::parse(reinterpret_cast<const uint8_t*>(pin));
    }
    // bytes == 0: the caller does not know the archive length (the reference's
    // d_decompress takes none, src/waltz.cu:612-626); the header's section
    // sizes give it, and every later check runs against that length.
    if (bytes == 0) bytes = size_t(archive_end(h));
    {
        const uintptr_t a = reinterpret_cast<uintptr_t>(d_in), b = reinterpret_cast<uintptr_t>(d_out);
        need(!(a < b + n * sizeof(T) && b < a + bytes), "Waltz: input and output buffers overlap");
    }
    const Layout L = validate_header<T>(h, g, bytes, canonical);
    const uint64_t words = (n + 31) / 32;
    Carver cv{nullptr};
    auto plan = [&](Carver& c) {
        struct P {
            T *C, *bank1, *bank2;
            uint32_t *status, *seen;
        } p;
        p.C = c.take<T>(n);
        p.bank1 = c.take<T>(n);
        p.bank2 = c.take<T>(n);
        p.status = c.take<uint32_t>(1);
        p.seen = c.take<uint32_t>(words + 1);
        return p;
    };
    plan(cv);
    Carver real{t_arena.reserve(cv.used)};
    auto P = plan(real);
    const uint16_t* irank = t_inv_tables.get(nx, ny, nz, g.bz, true, stream);
    const uint16_t* frank = t_fwd_tables.get(nx, ny, nz, g.bz, false, stream);
    check(cudaMemsetAsync(P.status, 0, 4, stream), "memset");
    FinalOut<T> fin{d_out, nx, size_t(nx) * ny, P.status};
    Sink sink{stream};
    decode_launch<T>(JobRef{nullptr, decode_job(d_in, h, L)}, h.split, g, irank, frank, P.C, P.bank1,
                     P.bank2, fin, RowPatch<T>{d_out}, P.status, sink);
    check(cudaMemcpyAsync(pin + 8, P.status, 4, cudaMemcpyDeviceToHost, stream), "readback");
    check(cudaStreamSynchronize(stream), "decompress");
    decode_finish<T>(uint32_t(pin[8]), d_in, h, L, g, P.status, P.seen, stream);
}

template <class T>
static void extrema(const T* d_in, uint64_t n, double* mn, double* mx, cudaStream_t stream) {
    need(d_in && n, "extrema requires at least one element");
    Carver cv{t_arena.reserve(256)};
    auto* keys = cv.take<unsigned long long>(2);
    const unsigned long long init[2] = {~0ull, 0ull};
    uint64_t* pin = pinned();
    std::memcpy(pin, init, 16);
    check(cudaMemcpyAsync(keys, pin, 16, cudaMemcpyHostToDevice, stream), "extrema init");
    extrema_kernel<T><<<grid_for(n, 256), 256, 0, stream>>>(d_in, n, keys); note_launch();
    check(cudaGetLastError(), "extrema launch");
    check(cudaMemcpyAsync(pin + 2, keys, 16, cudaMemcpyDeviceToHost, stream), "extrema readback");
    check(cudaStreamSynchronize(stream), "extrema");
    auto value = [](unsigned long long k) {
        const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
        double d;
        std::memcpy(&d, &b, 8);
        return d;
    };
    *mn = value(pin[2]);
    *mx = value(pin[3]);
}

// ------------------------------------------------------------ batched compress
// Many independent fields (uneven shapes) compressed by one CUDA graph: each
// field's kernel chain is captured on one of several parallel branches,
// so fields run concurrently and one graph launch replaces thousands of
// kernel launches. The instantiated graph is kept and replayed while the
// batch description (pointers, shapes, bounds) stays the same; all results
// come back in one copy.
// Batch execution of the calling thread's next captured batch graphs:
// stage-batched (fields split round-robin into `width` groups, each group one
// graph branch on which every stage is one batched launch per op type over
// the group's fields), or field chains (each field's own launches, fields
// round-robin on `width` branches).
constexpr int kMaxBranches = 64;
struct BatchConfig {
    int mode = WALTZ_B200_BATCH_FIELDS;
    int width = 32;
};
static thread_local BatchConfig t_batch_cfg;

struct BatchTables {
    struct Entry {
        uint32_t nx, ny, nz, bz;
        bool inverse;
        uint16_t* ptr;
    };
    int device = -1;
    std::vector<Entry> entries;
    ~BatchTables() {
        for (auto& e : entries) cudaFree(e.ptr);
    }
    const uint16_t* get(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t bz, bool inverse, cudaStream_t stream) {
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        if (dev != device) {
            entries.clear(); // tables of another device's context stay allocated there
            device = dev;
        }
        for (auto& e : entries)
            if (e.nx == nx && e.ny == ny && e.nz == nz && e.bz == bz && e.inverse == inverse) return e.ptr;
        const auto host = morton_tables(nx, ny, nz, bz, inverse);
        uint16_t* p = nullptr;
        check(cudaMalloc(&p, host.size() * 2), "Waltz: cannot allocate Morton table");
        check(cudaMemcpyAsync(p, host.data(), host.size() * 2, cudaMemcpyHostToDevice, stream), "table upload");
        check(cudaStreamSynchronize(stream), "table upload");
        entries.push_back({nx, ny, nz, bz, inverse, p});
        return p;
    }
};

// The capture stream, the parallel branches and their fork/join events.
struct BatchStreams {
    int device = -1;
    cudaStream_t cap = nullptr;
    cudaStream_t work[kMaxBranches] = {};
    cudaEvent_t fork = nullptr, join[kMaxBranches] = {};
    void ensure() {
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        if (cap && dev == device) return;
        check(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "stream");
        for (auto& w : work) check(cudaStreamCreateWithFlags(&w, cudaStreamNonBlocking), "stream");
        check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");
        for (auto& e : join) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        device = dev;
    }
};
static thread_local BatchStreams t_batch_streams;

// One instantiated batch graph and the description it was captured for.
struct CachedGraph {
    int device = -1;
    std::vector<unsigned char> key;
    cudaGraphExec_t exec = nullptr;
    bool valid(const std::vector<unsigned char>& k) const {
        int dev = 0;
        return exec && cudaGetDevice(&dev) == cudaSuccess && dev == device && k == key;
    }
};

// Captures `body(work streams)` between a fork and a join of `branches`
// parallel streams (or, with no branches, on the capture stream alone) and
// replaces the cached graph with its instantiation.
template <class Body>
static void capture_batch(BatchStreams& bs, int branches, CachedGraph& cg, std::vector<unsigned char>&& key,
                          Body body) {
    StageClock& clock = stage_clock();
    const bool profiling = clock.enabled;
    clock.enabled = false;
    cudaGraph_t graph = nullptr;
    check(cudaStreamBeginCapture(bs.cap, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        if (branches == 0) {
            body(&bs.cap); // one chain on the capture stream
        } else {
            check(cudaEventRecord(bs.fork, bs.cap), "fork");
            for (int k = 0; k < branches; ++k) check(cudaStreamWaitEvent(bs.work[k], bs.fork, 0), "fork wait");
            body(bs.work);
            for (int k = 0; k < branches; ++k) {
                check(cudaEventRecord(bs.join[k], bs.work[k]), "join");
                check(cudaStreamWaitEvent(bs.cap, bs.join[k], 0), "join wait");
            }
        }
    } catch (...) {
        cudaStreamEndCapture(bs.cap, &graph);
        if (graph) cudaGraphDestroy(graph);
        clock.enabled = profiling;
        throw;
    }
    clock.enabled = profiling;
    check(cudaStreamEndCapture(bs.cap, &graph), "end capture");
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    check(ie, "graph instantiate");
    graph_counter().fetch_add(1, std::memory_order_relaxed);
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (cg.exec && cg.device == dev) cudaGraphExecDestroy(cg.exec);
    cg.exec = exec;
    cg.device = dev;
    cg.key = std::move(key);
}

// Pinned host staging that grows on demand.
struct PinnedBuffer {
    void* ptr = nullptr;
    size_t cap = 0;
    ~PinnedBuffer() {
        if (ptr) cudaFreeHost(ptr);
    }
    template <class V> V* get(size_t count) {
        if (cap < count * sizeof(V)) {
            if (ptr) cudaFreeHost(ptr);
            ptr = nullptr;
            cap = 0;
            check(cudaMallocHost(&ptr, count * sizeof(V)), "pinned staging");
            cap = count * sizeof(V);
        }
        return static_cast<V*>(ptr);
    }
};

template <class V> static void append_key(std::vector<unsigned char>& key, const V& v) {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    key.insert(key.end(), p, p + sizeof(V));
}

struct BatchCompressState {
    CachedGraph graph;
    Arena scratch, table;
    PinnedBuffer results;
    BatchTables tables;
};

// Records every field's stages and captures their stage-batched replay on
// the capture stream; the parameter table is uploaded first and kept.
template <class Enqueue>
static void capture_stage_batched(BatchStreams& bs, int groups, CachedGraph& cg, Arena& table_arena,
                                  std::vector<unsigned char>&& key, uint32_t count, Enqueue enqueue,
                                  bool queue = false) {
    groups = int(std::min<uint32_t>(uint32_t(groups), count));
    std::vector<Recorder> recs(groups);
    for (uint32_t i = 0; i < count; ++i) {
        Recorder& rec = recs[i % uint32_t(groups)];
        rec.begin_field();
        Sink sink{bs.cap, &rec, true};
        enqueue(i, sink);
    }
    std::vector<BatchPlan> plans;
    std::vector<size_t> at;
    size_t total = 0;
    for (const Recorder& rec : recs) {
        plans.push_back(BatchPlan::make(rec));
        at.push_back(total);
        total += (plans.back().bytes() + 255) & ~size_t(255);
    }
    unsigned char* table = reinterpret_cast<unsigned char*>(table_arena.reserve(total));
    for (size_t g = 0; g < plans.size(); ++g)
        check(cudaMemcpy(table + at[g], plans[g].host.data(), plans[g].bytes(), cudaMemcpyHostToDevice),
              "batch table upload");
    capture_batch(bs, groups == 1 ? 0 : groups, cg, std::move(key), [&](cudaStream_t* s) {
        for (size_t g = 0; g < plans.size(); ++g) plans[g].execute(table + at[g], s[g], queue, uint32_t(plans.size()));
    });
}
static thread_local BatchCompressState t_bc;

template <class T>
static void compress_batch(const waltz_b200_chunk* items, uint32_t count, uint64_t* written, cudaStream_t stream) {
    need(count > 0 && items && written, "invalid batch arguments");
    std::vector<CompressJob<T>> jobs;
    jobs.reserve(count);
    std::vector<size_t> offset(count);
    size_t total = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const waltz_b200_chunk& c = items[i];
        try {
            jobs.push_back(CompressJob<T>::make(static_cast<const T*>(c.input), c.nx, c.ny, c.nz, c.abs_error,
                                                static_cast<uint8_t*>(c.archive), c.capacity, EncodeOptions()));
        } catch (const std::exception& e) {
            throw Error("batch item " + std::to_string(i) + ": " + e.what());
        }
        total = (total + 255) & ~size_t(255);
        offset[i] = total;
        total += jobs.back().scratch_bytes();
    }
    total = (total + 255) & ~size_t(255);
    const size_t results_at = total;
    total += size_t(count) * 9 * 8;

    BatchCompressState& st = t_bc;
    BatchStreams& bs = t_batch_streams;
    bs.ensure();
    std::vector<unsigned char> key(reinterpret_cast<const unsigned char*>(items),
                                   reinterpret_cast<const unsigned char*>(items + count));
    key.push_back(uint8_t(sizeof(T)));
    const BatchConfig cfg = t_batch_cfg;
    append_key(key, cfg.mode);
    append_key(key, cfg.width);
    append_key(key, t_opt.stage_kernels);
    append_key(key, t_opt.zmarch);
    append_key(key, t_opt.small_level);
    append_key(key, t_opt.small_fwd);
    append_key(key, t_opt.xy_march);
    append_key(key, t_opt.small_march);
    append_key(key, t_opt.small_march_fwd);
    char* base = st.scratch.reserve(total);
    append_key(key, base); // the scratch must not have moved since the graph was captured
    uint64_t* results = reinterpret_cast<uint64_t*>(base + results_at);
    if (!st.graph.valid(key)) {
        std::vector<const uint16_t*> rank(count);
        for (uint32_t i = 0; i < count; ++i)
            rank[i] = st.tables.get(jobs[i].nx, jobs[i].ny, jobs[i].nz, jobs[i].g.bz, false, bs.cap);
        if (cfg.mode == WALTZ_B200_BATCH_STAGES || cfg.mode == WALTZ_B200_BATCH_QUEUE) {
            capture_stage_batched(bs, cfg.width, st.graph, st.table, std::move(key), count,
                                  [&](uint32_t i, Sink& sink) {
                                      jobs[i].enqueue(base + offset[i], rank[i], sink, results + 9 * size_t(i));
                                  },
                                  cfg.mode == WALTZ_B200_BATCH_QUEUE);
        } else {
            capture_batch(bs, cfg.width, st.graph, std::move(key), [&](cudaStream_t* work) {
                for (uint32_t i = 0; i < count; ++i) {
                    Sink sink{work[i % uint32_t(cfg.width)]};
                    jobs[i].enqueue(base + offset[i], rank[i], sink, results + 9 * size_t(i));
                }
            });
        }
    }
    check(cudaGraphLaunch(st.graph.exec, stream), "graph launch");
    uint64_t* host = st.results.get<uint64_t>(size_t(count) * 9);
    check(cudaMemcpyAsync(host, results, size_t(count) * 9 * 8, cudaMemcpyDeviceToHost, stream), "readback");
    check(cudaStreamSynchronize(stream), "batch compress");
    for (uint32_t i = 0; i < count; ++i) {
        try {
            written[i] = jobs[i].finish(host + 9 * size_t(i));
        } catch (const std::exception& e) {
            throw Error("batch item " + std::to_string(i) + ": " + e.what());
        }
    }
}

// ---------------------------------------------------------- batched decode
// Many archives (uneven shapes, either form) decoded by one CUDA graph into
// caller buffers: views of one preallocated tensor, or boxes of a larger
// frame (output strides). Archive and output addresses live in a device job
// table rewritten before every launch, so the graph is captured once per
// (shapes, forms, output strides) and replayed for every later batch with
// that description — the data-loader pattern, where every batch brings other
// archives and a fresh output tensor.
__global__ void gather_headers_kernel(const uint8_t* const* archives, uint8_t* headers) {
    headers[size_t(blockIdx.x) * 32 + threadIdx.x] = archives[blockIdx.x][threadIdx.x];
}

struct BatchDecodeState {
    CachedGraph graph;
    Arena scratch, table;
    PinnedBuffer stage; // job table, then archive pointers / headers / status words
    BatchTables tables;
};
static thread_local BatchDecodeState t_bd;

template <class T>
static void decompress_batch(const waltz_b200_archive* items, uint32_t count, cudaStream_t stream) {
    need(count > 0 && items, "invalid batch arguments");
    struct Item {
        Geometry g;
        Header h;
        Layout L;
        uint64_t sy, sz; // output strides (elements)
    };
    std::vector<Item> list(count);
    auto item_error = [](uint32_t i, const char* what) {
        return Error("batch item " + std::to_string(i) + ": " + what);
    };
    uint64_t max_n = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const waltz_b200_archive& a = items[i];
        try {
            need(a.nx && a.ny && a.nz, "Waltz: nonzero dimensions required");
            const uint64_t n = uint64_t(a.nx) * a.ny * a.nz;
            need(n <= 0xffffffffull / sizeof(T), "Waltz: volume exceeds the archive section limits");
            need(a.archive && a.output, "Waltz: null buffer");
            const uint64_t sy = a.stride_y ? a.stride_y : a.nx, sz = a.stride_z ? a.stride_z : sy * a.ny;
            need(sy >= a.nx && sz >= sy * a.ny, "Waltz: output strides smaller than the chunk");
            const uint64_t extent = ((a.nz - 1) * sz + (a.ny - 1) * sy + a.nx) * sizeof(T);
            need(a.output_bytes >= extent, "output capacity too small");
            need(a.bytes >= 32, "invalid Waltz archive header");
            const uintptr_t p = reinterpret_cast<uintptr_t>(a.archive), q = reinterpret_cast<uintptr_t>(a.output);
            need(!(p < q + extent && q < p + a.bytes), "Waltz: input and output buffers overlap");
            need(!(q % sizeof(T)), "Waltz: misaligned output");
            list[i].sy = sy;
            list[i].sz = sz;
            list[i].g = Geometry::make(a.nx, a.ny, a.nz);
            max_n = std::max(max_n, n);
        } catch (const std::exception& e) {
            throw item_error(i, e.what());
        }
    }
    // Scratch: job table, status words, archive pointers, gathered headers,
    // the duplicate-check bitmap, then C / bank1 / bank2 per lane: one lane
    // per field when stage-batched (all fields run at once), else one per
    // branch sized by the largest field on it.
    const BatchConfig cfg = t_batch_cfg;
    const bool staged = cfg.mode == WALTZ_B200_BATCH_STAGES || cfg.mode == WALTZ_B200_BATCH_QUEUE;
    const uint32_t lanes = staged ? count : uint32_t(cfg.width);
    auto lane_of = [&](uint32_t i) { return staged ? i : i % uint32_t(cfg.width); };
    std::vector<uint64_t> lane_n(lanes, 0);
    for (uint32_t i = 0; i < count; ++i) lane_n[lane_of(i)] = std::max<uint64_t>(lane_n[lane_of(i)], list[i].g.n);
    Carver plan{nullptr};
    auto carve = [&](Carver& c) {
        struct P {
            DecodeJob* jobs;
            uint32_t* status;
            const uint8_t** ptrs;
            uint8_t* headers;
            uint32_t* seen;
            std::vector<T*> C, b1, b2;
        } p;
        p.jobs = c.take<DecodeJob>(count);
        p.status = c.take<uint32_t>(count);
        p.ptrs = c.take<const uint8_t*>(count);
        p.headers = c.take<uint8_t>(size_t(count) * 32);
        p.seen = c.take<uint32_t>((max_n + 31) / 32 + 1);
        for (uint32_t k = 0; k < lanes; ++k) {
            p.C.push_back(c.take<T>(lane_n[k]));
            p.b1.push_back(c.take<T>(lane_n[k]));
            p.b2.push_back(c.take<T>(lane_n[k]));
        }
        return p;
    };
    carve(plan);
    BatchDecodeState& st = t_bd;
    BatchStreams& bs = t_batch_streams;
    bs.ensure();
    Carver real{st.scratch.reserve(plan.used)};
    auto P = carve(real);
    // Pinned words: job table (8 per archive), archive pointers (1), gathered
    // headers (4), status words (1/2).
    uint64_t* pin = st.stage.get<uint64_t>(size_t(count) * 14 + 1);
    DecodeJob* jobs = reinterpret_cast<DecodeJob*>(pin);
    uint64_t* ptrs = pin + size_t(count) * 8;
    uint8_t* gathered = reinterpret_cast<uint8_t*>(pin + size_t(count) * 9);
    uint32_t* status = reinterpret_cast<uint32_t*>(pin + size_t(count) * 13);

    // Headers: from the caller's host copies, else gathered on the device.
    std::vector<const uint8_t*> hdr(count, nullptr);
    bool gather = false;
    for (uint32_t i = 0; i < count; ++i) {
        hdr[i] = static_cast<const uint8_t*>(items[i].header);
        gather |= !hdr[i];
    }
    if (gather) {
        for (uint32_t i = 0; i < count; ++i) ptrs[i] = reinterpret_cast<uint64_t>(items[i].archive);
        check(cudaMemcpyAsync(P.ptrs, ptrs, size_t(count) * 8, cudaMemcpyHostToDevice, stream), "pointer upload");
        gather_headers_kernel<<<count, 32, 0, stream>>>(P.ptrs, P.headers); note_launch();
        check(cudaGetLastError(), "header gather");
        check(cudaMemcpyAsync(gathered, P.headers, size_t(count) * 32, cudaMemcpyDeviceToHost, stream),
              "header readback");
        check(cudaStreamSynchronize(stream), "header readback");
    }
    for (uint32_t i = 0; i < count; ++i) {
        Item& it = list[i];
        it.h = Header::parse(hdr[i] ? hdr[i] : gathered + size_t(i) * 32);
        try {
            it.L = validate_header<T>(it.h, it.g, items[i].bytes, false);
        } catch (const std::exception& e) {
            throw item_error(i, e.what());
        }
    }
    for (uint32_t i = 0; i < count; ++i)
        jobs[i] = decode_job(static_cast<const uint8_t*>(items[i].archive), list[i].h, list[i].L, items[i].output);
    check(cudaMemcpyAsync(P.jobs, jobs, size_t(count) * sizeof(DecodeJob), cudaMemcpyHostToDevice, stream),
          "job table upload");
    check(cudaMemsetAsync(P.status, 0, size_t(count) * 4, stream), "memset");

    std::vector<unsigned char> key;
    key.push_back(uint8_t(sizeof(T)));
    append_key(key, cfg.mode);
    append_key(key, cfg.width);
    append_key(key, t_opt.stage_kernels);
    append_key(key, t_opt.zmarch);
    append_key(key, t_opt.small_level);
    append_key(key, t_opt.small_fwd);
    append_key(key, t_opt.xy_march);
    append_key(key, t_opt.small_march);
    append_key(key, t_opt.small_march_fwd);
    append_key(key, count);
    append_key(key, static_cast<const void*>(P.jobs));
    for (uint32_t i = 0; i < count; ++i) {
        append_key(key, items[i].nx);
        append_key(key, items[i].ny);
        append_key(key, items[i].nz);
        append_key(key, list[i].sy);
        append_key(key, list[i].sz);
        key.push_back(list[i].h.split);
    }
    if (!st.graph.valid(key)) {
        std::vector<const uint16_t*> irank(count), frank(count);
        for (uint32_t i = 0; i < count; ++i) {
            const Geometry& g = list[i].g;
            irank[i] = st.tables.get(g.nx, g.ny, g.nz, g.bz, true, bs.cap);
            frank[i] = st.tables.get(g.nx, g.ny, g.nz, g.bz, false, bs.cap);
            if (list[i].h.split) t_zmat.get(g.nz, list[i].h.split, bs.cap); // upload before capture
        }
        auto enqueue = [&](uint32_t i, Sink& sink) {
            const uint32_t k = lane_of(i);
            const Geometry& g = list[i].g;
            const DecodeJob* job = P.jobs + i;
            JobOut<T> fin{job, list[i].sy, list[i].sz, P.status + i};
            JobPatch<T> patch{job, g.nx, g.ny, list[i].sy, list[i].sz};
            decode_launch<T>(JobRef{job, {}}, list[i].h.split, g, irank[i], frank[i], P.C[k], P.b1[k],
                             P.b2[k], fin, patch, P.status + i, sink);
        };
        if (staged) {
            capture_stage_batched(bs, cfg.width, st.graph, st.table, std::move(key), count, enqueue,
                                  cfg.mode == WALTZ_B200_BATCH_QUEUE);
        } else {
            capture_batch(bs, cfg.width, st.graph, std::move(key), [&](cudaStream_t* work) {
                for (uint32_t i = 0; i < count; ++i) {
                    Sink sink{work[i % uint32_t(cfg.width)]};
                    enqueue(i, sink);
                }
            });
        }
    }
    check(cudaGraphLaunch(st.graph.exec, stream), "graph launch");
    check(cudaMemcpyAsync(status, P.status, size_t(count) * 4, cudaMemcpyDeviceToHost, stream), "readback");
    check(cudaStreamSynchronize(stream), "batch decompress");
    for (uint32_t i = 0; i < count; ++i) {
        if (!status[i]) continue;
        try {
            decode_finish<T>(status[i], static_cast<const uint8_t*>(items[i].archive), list[i].h, list[i].L,
                             list[i].g, P.status + i, P.seen, stream);
        } catch (const std::exception& e) {
            throw item_error(i, e.what());
        }
    }
}

static thread_local char t_error[256];
static int fail(const std::exception& e) {
    std::snprintf(t_error, sizeof(t_error), "%s", e.what());
    return -1;
}

} // namespace wb

using namespace wb;

extern "C" {

const char* waltz_b200_last_error(void) { return t_error; }

size_t waltz_b200_compressed_capacity(uint64_t n, int width) {
    if ((width != 4 && width != 8) || n > 0xffffffffull) return 0;
    return capacity_for(n, unsigned(width));
}

int waltz_b200_compress(const void* d_input, int width, uint32_t nx, uint32_t ny, uint32_t nz, double abs_error,
                        void* d_archive, size_t capacity, size_t* written, void* stream) {
    try {
        need(written != nullptr, "null argument");
        *written = 0;
        need(width == 4 || width == 8, "type must be FP32 or FP64");
        auto s = reinterpret_cast<cudaStream_t>(stream);
        auto* out = static_cast<uint8_t*>(d_archive);
        *written = width == 4 ? compress(static_cast<const float*>(d_input), nx, ny, nz, abs_error, out, capacity, s)
                              : compress(static_cast<const double*>(d_input), nx, ny, nz, abs_error, out, capacity, s);
        t_error[0] = 0;
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int waltz_b200_compress_form(const void* d_input, int width, uint32_t nx, uint32_t ny, uint32_t nz,
                             double abs_error, int form, void* d_archive, size_t capacity, size_t* written,
                             void* stream) {
    try {
        need(written != nullptr, "null argument");
        *written = 0;
        need(width == 4 || width == 8, "type must be FP32 or FP64");
        need(form >= WALTZ_B200_FORM_PLAIN && form <= WALTZ_B200_FORM_MATRIX_EXACT, "unknown transform form");
        EncodeOptions opt;
        opt.zsplit = form; // the form values are the split codes
        auto s = reinterpret_cast<cudaStream_t>(stream);
        auto* out = static_cast<uint8_t*>(d_archive);
        *written = width == 4
                       ? compress(static_cast<const float*>(d_input), nx, ny, nz, abs_error, out, capacity, s, opt)
                       : compress(static_cast<const double*>(d_input), nx, ny, nz, abs_error, out, capacity, s, opt);
        t_error[0] = 0;
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int waltz_b200_compress_batch(const waltz_b200_chunk* chunks, uint32_t count, int width, uint64_t* written,
                              void* stream) {
    try {
        need(width == 4 || width == 8, "type must be FP32 or FP64");
        if (written)
            for (uint32_t i = 0; i < count; ++i) written[i] = 0;
        auto s = reinterpret_cast<cudaStream_t>(stream);
        if (width == 4) compress_batch<float>(chunks, count, written, s);
        else compress_batch<double>(chunks, count, written, s);
        t_error[0] = 0;
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int waltz_b200_set_option(int option, int value) {
    using namespace wb;
    switch (option) {
    case WALTZ_B200_OPT_STAGE_KERNELS:
        if (value != 0 && value != 1) break;
        t_opt.stage_kernels = value != 0;
        return 0;
    case WALTZ_B200_OPT_ZMARCH_PLANES:
        if (value < 0 || value > 65536) break;
        t_opt.zmarch = uint32_t(value);
        return 0;
    case WALTZ_B200_OPT_SMALL_LEVEL:
        if (value < 0) break;
        t_opt.small_level = uint64_t(value);
        return 0;
    case WALTZ_B200_OPT_SMALL_FWD:
        if (value < 0) break;
        t_opt.small_fwd = uint64_t(value);
        return 0;
    case WALTZ_B200_OPT_COMPACT_REPAIRS:
        if (value != 0 && value != 16 && value != 64) break;
        t_opt.repair_scale = uint32_t(value);
        return 0;
    case WALTZ_B200_OPT_XY_MARCH:
        if (value < 0 || value > 3) break;
        t_opt.xy_march = uint32_t(value);
        return 0;
    case WALTZ_B200_OPT_SMALL_MARCH:
        if (value < 0) break;
        t_opt.small_march = uint64_t(value);
        return 0;
    case WALTZ_B200_OPT_SMALL_MARCH_FWD:
        if (value < 0) break;
        t_opt.small_march_fwd = uint64_t(value);
        return 0;
    default:
        break;
    }
    std::snprintf(t_error, sizeof(t_error), "invalid option %d or value %d", option, value);
    return -1;
}

int waltz_b200_batch_config(int mode, int width) {
    using namespace wb;
    if ((mode != WALTZ_B200_BATCH_STAGES && mode != WALTZ_B200_BATCH_FIELDS && mode != WALTZ_B200_BATCH_QUEUE) ||
        width < 1 || width > kMaxBranches) {
        std::snprintf(t_error, sizeof(t_error), "invalid batch configuration (mode %d, width %d)", mode, width);
        return -1;
    }
    t_batch_cfg = BatchConfig{mode, width};
    return 0;
}

int waltz_b200_decompress_batch(const waltz_b200_archive* archives, uint32_t count, int width, void* stream) {
    using namespace wb;
    try {
        need(width == 4 || width == 8, "Waltz: width must be 4 or 8");
        if (width == 4) decompress_batch<float>(archives, count, reinterpret_cast<cudaStream_t>(stream));
        else decompress_batch<double>(archives, count, reinterpret_cast<cudaStream_t>(stream));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int waltz_b200_decompress(const void* d_archive, size_t bytes, int width, uint32_t nx, uint32_t ny, uint32_t nz,
                          void* d_output, size_t output_bytes, void* stream) {
    try {
        need(width == 4 || width == 8, "type must be FP32 or FP64");
        auto s = reinterpret_cast<cudaStream_t>(stream);
        auto* in = static_cast<const uint8_t*>(d_archive);
        if (width == 4) decompress(in, bytes, nx, ny, nz, static_cast<float*>(d_output), output_bytes, s, false, nullptr);
        else decompress(in, bytes, nx, ny, nz, static_cast<double*>(d_output), output_bytes, s, false, nullptr);
        t_error[0] = 0;
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int waltz_b200_extrema(const void* d_input, int width, uint64_t n, double* min_out, double* max_out, void* stream) {
    try {
        need(min_out && max_out, "null argument");
        need(width == 4 || width == 8, "type must be FP32 or FP64");
        auto s = reinterpret_cast<cudaStream_t>(stream);
        if (width == 4) extrema(static_cast<const float*>(d_input), n, min_out, max_out, s);
        else extrema(static_cast<const double*>(d_input), n, min_out, max_out, s);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

const char* waltz_cuda_decode_chunk(uint32_t nx, uint32_t ny, uint32_t nz, int width, const void* archive,
                                    size_t bytes, void* output, size_t out_bytes, void* stream) {
    static std::mutex lock;
    static thread_local char error[256];
    try {
        std::lock_guard<std::mutex> guard(lock);
        need((width == 4 || width == 8) && nx && ny && nz && archive && output && bytes >= 32 &&
                 uint64_t(nx) * ny <= 0xffffffffull / unsigned(width) / nz &&
                 out_bytes == uint64_t(nx) * ny * nz * unsigned(width),
             "invalid chunk dimensions or buffer sizes");
        auto s = reinterpret_cast<cudaStream_t>(stream);
        auto* in = static_cast<const uint8_t*>(archive);
        if (width == 4) decompress(in, bytes, nx, ny, nz, static_cast<float*>(output), out_bytes, s, true, nullptr);
        else decompress(in, bytes, nx, ny, nz, static_cast<double*>(output), out_bytes, s, true, nullptr);
        return nullptr;
    } catch (const std::exception& e) {
        std::snprintf(error, sizeof(error), "%s", e.what());
    }
    (void)cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream));
    return error;
}

} // extern "C"

namespace wb {
// Status word of a standalone WZP encode -> diagnostic (capacity, a
// lookback wait that hit its bound, anything else).
static void wzp_encode_status(uint32_t st) {
    if (st & ST_CAPACITY) throw Error("WZP output capacity is too small");
    if (st & ST_LOOKBACK_TIMEOUT) throw Error("Waltz: WZP lookback wait exceeded its bound");
    if (st & ST_WAIT_TIMEOUT) throw Error("Waltz: asynchronous copy wait exceeded its bound");
    if (st) throw Error("WZP encode failed");
}
} // namespace wb

// Diagnostic stage entry points (declared in include/waltz_b200.h).
extern "C" int waltz_b200_transform(void* d_data, int width, uint32_t nx, uint32_t ny, uint32_t nz, int inverse,
                                    void* stream) {
    try {
        need(width == 4 || width == 8, "type must be FP32 or FP64");
        need(nx && ny && nz && d_data, "invalid transform arguments");
        auto s = reinterpret_cast<cudaStream_t>(stream);
        const Geometry g = Geometry::make(nx, ny, nz);
        const TransformScratch ts = scratch_need(g);
        auto run = [&](auto* data) {
            using T = std::remove_pointer_t<decltype(data)>;
            Carver cv{nullptr};
            auto plan = [&](Carver& c) {
                struct P { T *C, *a, *b, *inter, *bank2; uint32_t* status; } p;
                p.C = c.take<T>(g.n); p.a = c.take<T>(ts.low); p.b = c.take<T>(ts.low);
                p.inter = c.take<T>(g.n); p.bank2 = c.take<T>(g.n); p.status = c.take<uint32_t>(1);
                return p;
            };
            plan(cv);
            Carver real{t_arena.reserve(cv.used)};
            auto P = plan(real);
            check(cudaMemsetAsync(P.status, 0, 4, s), "memset");
            if (!inverse) {
                Sink sink{s};
                forward<T>(g, data, P.C, P.a, P.b, P.inter, P.status, sink);
                check(cudaMemcpyAsync(data, P.C, g.n * sizeof(T), cudaMemcpyDeviceToDevice, s), "copy");
            } else {
                check(cudaMemcpyAsync(P.C, data, g.n * sizeof(T), cudaMemcpyDeviceToDevice, s), "copy");
                Sink sink{s};
                wb::inverse<T>(g, P.C, P.inter, P.bank2, StoreOut<T>{data, nx, size_t(nx) * ny}, P.status, sink);
            }
            uint32_t st = 0;
            check(cudaMemcpyAsync(&st, P.status, 4, cudaMemcpyDeviceToHost, s), "readback");
            check(cudaStreamSynchronize(s), "transform");
            if (st & ST_WAIT_TIMEOUT) throw Error("Waltz: asynchronous copy wait exceeded its bound");
        };
        if (width == 4) run(static_cast<float*>(d_data));
        else run(static_cast<double*>(d_data));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

extern "C" int waltz_b200_wzp_encode(const uint16_t* d_mag, const uint32_t* d_sign, uint32_t n, void* d_out,
                                     size_t capacity, size_t* written, void* stream) {
    try {
        need(written && d_mag && d_sign && d_out, "null argument");
        need(n && n <= 0x7fffffffu, "WZP element count outside (0, 2^31)");
        need(!(reinterpret_cast<uintptr_t>(d_mag) & 15), "WZP magnitudes must be 16-byte aligned");
        need(capacity >= wzp_header(n), "WZP output capacity is too small");
        auto s = reinterpret_cast<cudaStream_t>(stream);
        const uint32_t chunks = wzp_chunks(n);
        Carver cv{nullptr};
        auto plan = [&](Carver& c) {
            struct P { uint32_t *status, *ticket; uint64_t *state, *sizes, *total; } p;
            p.status = c.take<uint32_t>(1); p.ticket = c.take<uint32_t>(1);
            p.state = c.take<uint64_t>(chunks); p.sizes = c.take<uint64_t>(chunks); p.total = c.take<uint64_t>(1);
            return p;
        };
        plan(cv);
        Carver real{t_arena.reserve(cv.used)};
        auto P = plan(real);
        check(cudaMemsetAsync(P.status, 0, 4, s), "memset");
        check(cudaMemsetAsync(P.ticket, 0, 4, s), "memset");
        check(cudaMemsetAsync(P.state, 0, size_t(chunks) * 8, s), "memset");
        WzpEncodeArgs wa{n, static_cast<uint8_t*>(d_out), capacity, P.ticket, P.state, P.sizes, P.status, 1u << 22,
                         0xffffffffu};
        Sink sink{s};
        launch_wzp_encode(wa, MagArrays{d_mag, d_sign}, chunks, sink);
        const uint32_t groups = wzp_groups(n);
        sink.run<WzpDirectoryOp>(WzpDirectoryOp::Params{static_cast<uint8_t*>(d_out), n, P.state, P.sizes, P.total},
                                 (groups + 255) / 256);
        uint64_t* h = pinned();
        check(cudaMemcpyAsync(h, P.total, 8, cudaMemcpyDeviceToHost, s), "readback");
        check(cudaMemcpyAsync(h + 1, P.status, 4, cudaMemcpyDeviceToHost, s), "readback");
        check(cudaStreamSynchronize(s), "wzp encode");
        wzp_encode_status(uint32_t(h[1]));
        *written = size_t(h[0]);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// ------------------------------------------------ allocation-free WZP encode
// Some callers cannot allocate device memory at the point of call: a host
// framework whose caching allocator owns the whole device budget, a plugin or
// filter callback with no device-memory lifetime of its own, or a hot loop
// that cannot afford the device-wide synchronisation of cudaMalloc/cudaFree.
// For them the WZP encoder keeps its working state (ticket, status, total and
// the per-chunk lookback states and sizes) in one file-scope device array,
// loaded with the library on every GPU that uses it and held until exit.
namespace wb {
constexpr uint32_t kNoAllocMaxChunks = 16384; // 134,217,728 magnitudes
constexpr size_t kNoAllocWords = 32 + 2 * size_t(kNoAllocMaxChunks); // u64 words: header, states, sizes
static __device__ __align__(256) uint64_t g_wzp_noalloc_scratch[kNoAllocWords];

// Device address of the array for the current device. The first call on a
// device resolves it with cudaGetSymbolAddress (with that device current);
// later calls reuse it. The host-side name of the array is only a stand-in
// and must never reach a kernel.
static uint64_t* noalloc_scratch() {
    constexpr int kMaxDevices = 64;
    static std::mutex lock;
    static uint64_t* addr[kMaxDevices] = {};
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    need(dev >= 0 && dev < kMaxDevices, "Waltz: device ordinal outside the scratch table");
    std::lock_guard<std::mutex> guard(lock);
    if (!addr[dev]) {
        void* p = nullptr;
        check(cudaGetSymbolAddress(&p, g_wzp_noalloc_scratch), "Waltz: scratch symbol address");
        addr[dev] = static_cast<uint64_t*>(p);
    }
    return addr[dev];
}
} // namespace wb

extern "C" int waltz_b200_wzp_encode_noalloc(const uint16_t* d_mag, const uint32_t* d_sign, uint32_t n, void* d_out,
                                             size_t capacity, size_t* written, void* stream) {
    try {
        need(written && d_mag && d_sign && d_out, "null argument");
        *written = 0;
        need(n > 0, "WZP element count must be positive");
        need(!(reinterpret_cast<uintptr_t>(d_mag) & 15), "WZP magnitudes must be 16-byte aligned");
        need(wzp_chunks(n) <= kNoAllocMaxChunks,
             "WZP element count exceeds the allocation-free limit of 134217728 magnitudes");
        need(capacity >= wzp_header(n), "WZP output capacity is too small");
        auto s = reinterpret_cast<cudaStream_t>(stream);
        const uint32_t chunks = wzp_chunks(n), groups = wzp_groups(n);
        uint64_t* base = noalloc_scratch();
        auto* ticket = reinterpret_cast<uint32_t*>(base);      // word 0, low half
        auto* status = reinterpret_cast<uint32_t*>(base) + 1;  // word 0, high half
        uint64_t* total = base + 1;
        uint64_t* state = base + 32;
        uint64_t* sizes = state + kNoAllocMaxChunks;
        // The array keeps the previous call's contents: clear what must start at zero.
        check(cudaMemsetAsync(base, 0, 16, s), "memset");
        check(cudaMemsetAsync(state, 0, size_t(chunks) * 8, s), "memset");
        WzpEncodeArgs wa{n, static_cast<uint8_t*>(d_out), capacity, ticket, state, sizes, status, 1u << 22,
                         0xffffffffu};
        Sink sink{s};
        launch_wzp_encode(wa, MagArrays{d_mag, d_sign}, chunks, sink);
        sink.run<WzpDirectoryOp>(WzpDirectoryOp::Params{static_cast<uint8_t*>(d_out), n, state, sizes, total},
                                 (groups + 255) / 256);
        uint64_t host[2] = {0, 0}; // pageable: the copy completes before cudaMemcpyAsync returns
        check(cudaMemcpyAsync(host, base, 16, cudaMemcpyDeviceToHost, s), "readback");
        check(cudaStreamSynchronize(s), "wzp encode");
        const uint32_t st = uint32_t(host[0] >> 32);
        wzp_encode_status(st);
        *written = size_t(host[1]);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// Diagnostic entries of the tensor-core Z transform (declared in include/waltz_b200.h).
template <class T>
static void zmatrix_in_place(T* d_data, uint32_t nx, uint32_t ny, uint32_t nz, int inverse, int zsplit, void* stream) {
    need(d_data && nx && ny && nz, "invalid matrix transform arguments");
    need(zsplit >= kZsTf32x3 && zsplit <= kZsExact, "unknown matrix split form");
    auto s = reinterpret_cast<cudaStream_t>(stream);
    const uint64_t n = uint64_t(nx) * ny * nz;
    Carver cv{nullptr};
    auto plan = [&](Carver& c) {
        struct P { T* out; uint32_t* status; } p;
        p.out = c.take<T>(n);
        p.status = c.take<uint32_t>(1);
        return p;
    };
    plan(cv);
    Carver real{t_arena.reserve(cv.used)};
    auto P = plan(real);
    check(cudaMemsetAsync(P.status, 0, 4, s), "memset");
    Sink sink{s};
    zmatrix_apply<T>(d_data, nx, ny, nz, inverse != 0, zsplit, ZmStore<T>{P.out}, P.status, false, sink);
    check(cudaMemcpyAsync(d_data, P.out, n * sizeof(T), cudaMemcpyDeviceToDevice, s), "copy");
    uint32_t st = 0;
    check(cudaMemcpyAsync(&st, P.status, 4, cudaMemcpyDeviceToHost, s), "readback");
    check(cudaStreamSynchronize(s), "matrix transform");
    if (st & ST_WAIT_TIMEOUT) throw Error("Waltz: asynchronous copy wait exceeded its bound");
}

extern "C" int waltz_b200_zmatrix(float* d_data, uint32_t nx, uint32_t ny, uint32_t nz, int inverse, void* stream) {
    try {
        zmatrix_in_place<float>(d_data, nx, ny, nz, inverse, kZsTf32x3, stream);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

extern "C" int waltz_b200_zmatrix_f64(double* d_data, uint32_t nx, uint32_t ny, uint32_t nz, int inverse,
                                      void* stream) {
    try {
        zmatrix_in_place<double>(d_data, nx, ny, nz, inverse, kZsTf32x3, stream);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

extern "C" int waltz_b200_zmatrix_split(void* d_data, int width, uint32_t nx, uint32_t ny, uint32_t nz, int inverse,
                                        int form, void* stream) {
    try {
        need(width == 4 || width == 8, "type must be FP32 or FP64");
        need(form >= WALTZ_B200_FORM_MATRIX && form <= WALTZ_B200_FORM_MATRIX_EXACT, "unknown matrix form");
        if (width == 4) zmatrix_in_place<float>(static_cast<float*>(d_data), nx, ny, nz, inverse, form, stream);
        else zmatrix_in_place<double>(static_cast<double*>(d_data), nx, ny, nz, inverse, form, stream);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

extern "C" unsigned long long waltz_b200_launch_count(void) { return launch_counter().load(); }

extern "C" unsigned long long waltz_b200_graph_count(void) { return graph_counter().load(); }

extern "C" void waltz_b200_profile(int enable) { stage_clock().enabled = enable != 0; }

extern "C" int waltz_b200_stage_times(double* ms, const char** names, int cap) {
    const StageClock& c = stage_clock();
    const int n = c.read(ms, cap);
    for (int i = 0; i < n; ++i) names[i] = c.names[i];
    return n;
}

// Test hook: compress with a bounded lookback cap and a chunk that never
// publishes its state, to exercise the wait bound without a GPU fault.
extern "C" int waltz_b200_test_lookback_timeout(const void* d_input, int width, uint32_t nx, uint32_t ny,
                                                uint32_t nz, double abs_error, void* d_archive, size_t capacity,
                                                uint32_t skip_chunk, uint32_t spin_cap, void* stream) {
    try {
        EncodeOptions opt;
        opt.spin_cap = spin_cap;
        opt.skip_publish = skip_chunk;
        auto s = reinterpret_cast<cudaStream_t>(stream);
        auto* out = static_cast<uint8_t*>(d_archive);
        if (width == 4) compress(static_cast<const float*>(d_input), nx, ny, nz, abs_error, out, capacity, s, opt);
        else compress(static_cast<const double*>(d_input), nx, ny, nz, abs_error, out, capacity, s, opt);
        t_error[0] = 0;
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

#include "batch.cuh"

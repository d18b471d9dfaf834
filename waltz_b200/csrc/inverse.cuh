// Inverse dyadic level (synthesis Z, X, Y) from TMA-staged parity boxes.
//
// The coefficients of one level live in the reference's split-band layout:
// along each axis the even spatial positions are the low half [0, ceil(n/2))
// and the odd positions the high half. The footprint of a spatial tile
// (UX x UY x UZ outputs plus a 4-sample halo per side) therefore maps to eight
// coefficient boxes, one per parity combination (x, y, z even or odd), each
// (UX/2+4) x (UY/2+4) x (UZ/2+4). A CTA loads the eight boxes with tensor-map
// copies (the all-even box from the separately reconstructed low band when
// there is one), so every lifting pass reads its even samples from one box
// and its odd samples from the other, and writes its outputs back in place.
//
// Inverse windows fold their endpoint normalisations along Y and Z, so those
// results depend on the window (cpu/src/transform.cpp:110-147): the tile's Z
// extent is exactly one canonical Z window (16 f32 / 8 f64 outputs at a
// multiple of it) and its Y extent two canonical Y windows of 8. X does not
// fold and takes the tile's whole row as one window.
//
// Edge tiles (footprint crossing the array) first fix every out-of-range cell
// from its reflected position, coefficient-mapped like
// include/transformers/halo3d.cuh:23-28 of the reference: copied from inside
// the staged footprint when the reflected cell is there, else loaded.
#pragma once
#include "common.cuh"
#include "tma.cuh"
#include "transform.cuh"

namespace wb {

template <class T> struct InvTile;
template <> struct InvTile<float> {
    static constexpr int UX = 32, UY = 16, UZ = 16;
};
template <> struct InvTile<double> {
    static constexpr int UX = 16, UY = 16, UZ = 8;
};

template <class T, int UX, int UY, int UZ> struct InvShape {
    static constexpr int V = 16 / int(sizeof(T));       // elements per 16 bytes
    static constexpr int HX = UX / 2 + 4, HY = UY / 2 + 4, HZ = UZ / 2 + 4;
    static constexpr int PADX = (V - 2 % V) % V;         // box x origin = ox/2 - 2 - PADX (16-byte aligned)
    static constexpr int BX = (HX + PADX + V - 1) / V * V;
    static constexpr int BOX = HZ * HY * BX;             // elements per parity box
    static constexpr int FX = UX + 8, FY = UY + 8, FZ = UZ + 8;
    static constexpr size_t smem = size_t(8) * BOX * sizeof(T) + 128 + 32; // + alignment + four barriers
    static_assert((BOX * sizeof(T)) % 128 == 0, "parity boxes must stay 128-byte aligned");
    static_assert(UX % (2 * V) == 0 && UZ == (sizeof(T) == 4 ? 16 : 8) && UY % 8 == 0, "tile shape");
};

// Emission and source description of one inverse level.
template <class T> struct InvLevel {
    const T* base;  // coefficients (split layout), strides sy, sz
    size_t sy, sz;
    const T* low;   // reconstructed low band (compact, dims lo) or null
    Dims lo;
    Dims a;         // level dims
};

template <class T, int UX, int UY, int UZ, class Out> struct InvTileOp {
    // float tiles: 16 warps per CTA, two CTAs per SM (the passes have 512 to
    // 960 items); double tiles are half as wide and keep 8 warps
    static constexpr int kThreads = sizeof(T) == 4 ? 512 : 256, kMinBlocks = 2;
    static constexpr bool kGridConstant = true;
    struct Params {
        CUtensorMap cmap, lmap;
        InvLevel<T> lv;
        uint32_t tiles_x, tiles_y;
        Out out;
        uint32_t* status;
    };
    static __device__ __forceinline__ void run(const Params& P, uint32_t block, uint32_t);
    static __device__ __forceinline__ void acquire_maps(const Params& P) {
        tensormap_acquire(&P.cmap);
        if (P.lv.low) tensormap_acquire(&P.lmap);
    }
};

template <class T, int UX, int UY, int UZ, class Out>
__device__ __forceinline__ void InvTileOp<T, UX, UY, UZ, Out>::run(const Params& P, uint32_t block, uint32_t) {
    const InvLevel<T> lv = P.lv;
    const uint32_t tiles_x = P.tiles_x, tiles_y = P.tiles_y;
    const Out out = P.out;
    uint32_t* const status = P.status;
    using S = InvShape<T, UX, UY, UZ>;
    extern __shared__ __align__(128) unsigned char inv_smem[];
    T* Bx = reinterpret_cast<T*>(inv_smem + ((128 - (smem_u32(inv_smem) & 127)) & 127));
    uint64_t* bar = reinterpret_cast<uint64_t*>(Bx + 8 * S::BOX);
    const int tid = threadIdx.x, warp = tid >> 5;
    const Dims a = lv.a;
    const uint32_t bx = block % tiles_x, by = (block / tiles_x) % tiles_y, bz = block / (tiles_x * tiles_y);
    const uint32_t ox = bx * UX, oy = by * UY, oz = bz * UZ;
    const uint32_t hx = half_len(a.x), hy = half_len(a.y), hz = half_len(a.z);

    // staged cell of spatial footprint position (fx, fy, fz)
    auto cell = [&](int fx, int fy, int fz) -> T* {
        return Bx + ((fz & 1) * 4 + (fy & 1) * 2 + (fx & 1)) * S::BOX + ((fz >> 1) * S::HY + (fy >> 1)) * S::BX +
               (fx >> 1) + S::PADX;
    };

    // ---- stage the eight parity boxes, the z-even and z-odd box of one x/y
    // parity on one barrier each (bar[par], par = x parity + 2 * y parity),
    // so the Z pass of a parity starts as soon as its two boxes have landed
    if (tid == 0) {
#pragma unroll 1
        for (int p = 0; p < 4; ++p) mbar_init(bar + p, 1);
        fence_barrier_init();
        const int x0 = int(ox / 2) - 2 - S::PADX, y0 = int(oy / 2) - 2, z0 = int(oz / 2) - 2;
#pragma unroll 1
        for (int p = 0; p < 4; ++p) {
            mbar_expect_tx(bar + p, uint32_t(2 * S::BOX * sizeof(T)));
            const int xp = p & 1, yp = p >> 1;
#pragma unroll 1
            for (int zp = 0; zp < 2; ++zp) {
                const int b = p + 4 * zp;
                const bool from_low = b == 0 && lv.low != nullptr;
                tma_load_3d(Bx + b * S::BOX, from_low ? &P.lmap : &P.cmap, x0 + (xp ? int(hx) : 0),
                            y0 + (yp ? int(hy) : 0), z0 + (zp ? int(hz) : 0), bar + p);
            }
        }
    }
    __syncthreads(); // the barriers are initialised before any thread polls them
    // the emitter's own operands (the originals, for repairs): one thread per
    // tile row of UX samples (one 128-byte line) asks L2 for it now, so the
    // Y pass's fetches find it there
    if constexpr (Out::kPrefetch) {
        static_assert(UZ * UY <= kThreads && UX * sizeof(T) == 128, "one line per tile row and thread");
        if (tid < UZ * UY) {
            const uint32_t gy = oy + tid % UY, gz = oz + tid / UY;
            if (gy < a.y && gz < a.z) out.warm(ox, gy, gz);
        }
    }
    // ---- edge tiles: every box first, then the out-of-range cells from
    // their reflections
    const bool edge = ox < 4 || ox + UX + 4 > a.x || oy < 4 || oy + UY + 4 > a.y || oz < 4 || oz + UZ + 4 > a.z;
    if (edge) {
        {
            bool landed = true;
            if (warp == 0) {
#pragma unroll 1
                for (int p = 0; p < 4; ++p) landed = landed && mbar_wait(bar + p, 0, kWaitBound);
            }
            if (!__syncthreads_and(landed)) {
                if (tid == 0) atomicOr(status, ST_WAIT_TIMEOUT);
                return;
            }
        }
        // only the cells outside the array: the in-range footprint is the box
        // [f*_lo, f*_hi); cells of in-range rows left or right of it (A), and
        // whole rows outside it in y or z (B), as one flat list
        const int fx_lo = ox < 4 ? int(4 - ox) : 0, fx_hi = min(S::FX, int(a.x - ox) + 4);
        const int fy_lo = oy < 4 ? int(4 - oy) : 0, fy_hi = min(S::FY, int(a.y - oy) + 4);
        const int fz_lo = oz < 4 ? int(4 - oz) : 0, fz_hi = min(S::FZ, int(a.z - oz) + 4);
        const int nx_out = fx_lo + (S::FX - fx_hi), ny_in = fy_hi - fy_lo, nz_in = fz_hi - fz_lo;
        const int ny_out = S::FY - ny_in, nz_out = S::FZ - nz_in;
        const int na = ny_in * nz_in * nx_out;
        const int nb = (nz_out * S::FY + nz_in * ny_out) * S::FX;
        for (int i = tid; i < na + nb; i += kThreads) {
            int fx, fy, fz;
            if (i < na) {
                const int k = i % nx_out, row = i / nx_out;
                fy = fy_lo + row % ny_in;
                fz = fz_lo + row / ny_in;
                fx = k < fx_lo ? k : fx_hi + (k - fx_lo);
            } else {
                const int j = i - na;
                fx = j % S::FX;
                const int rr = j / S::FX;
                if (rr < nz_out * S::FY) {
                    const int zs = rr / S::FY;
                    fy = rr % S::FY;
                    fz = zs < fz_lo ? zs : fz_hi + (zs - fz_lo);
                } else {
                    const int r2 = rr - nz_out * S::FY, ks = r2 % ny_out;
                    fz = fz_lo + r2 / ny_out;
                    fy = ks < fy_lo ? ks : fy_hi + (ks - fy_lo);
                }
            }
            const int64_t px = int64_t(ox) + fx - 4, py = int64_t(oy) + fy - 4, pz = int64_t(oz) + fz - 4;
            const uint32_t mx = mirror(px, a.x), my = mirror(py, a.y), mz = mirror(pz, a.z);
            const int64_t gx = int64_t(mx) - (int64_t(ox) - 4), gy = int64_t(my) - (int64_t(oy) - 4),
                          gz = int64_t(mz) - (int64_t(oz) - 4);
            T v;
            if (gx >= 0 && gx < S::FX && gy >= 0 && gy < S::FY && gz >= 0 && gz < S::FZ) {
                v = *cell(int(gx), int(gy), int(gz));
            } else {
                const uint32_t cx = split_of(mx, a.x), cy = split_of(my, a.y), cz = split_of(mz, a.z);
                if (lv.low && cx < lv.lo.x && cy < lv.lo.y && cz < lv.lo.z)
                    v = lv.low[(size_t(cz) * lv.lo.y + cy) * lv.lo.x + cx];
                else
                    v = lv.base[size_t(cz) * lv.sz + size_t(cy) * lv.sy + cx];
            }
            *cell(fx, fy, fz) = v;
        }
        __syncthreads();
    }

    // ---- Z: every (x, y) footprint column, one canonical window, in place.
    // Pair j of a line sits at slot j of the z-even and z-odd boxes, and the
    // outputs of pair j overwrite exactly those two slots.
    constexpr int ZS = S::HY * S::BX; // z-slot stride inside a box
    {
        constexpr int P = UZ / 2 + 4;
        bool failed = false; // a copy that never landed: skip the work, the status fails the call
        for (int L = tid; L < S::FX * S::FY; L += kThreads) {
            // x index fastest inside one (x parity, y parity) box
            const int i = L % (S::FX / 2), k = (L / (S::FX / 2)) % (S::FY / 2);
            const int par = L / ((S::FX / 2) * (S::FY / 2)); // x parity + 2 * y parity
            if (!edge && !failed && !mbar_wait(bar + par, 0, kWaitBound)) { // edge tiles waited above
                failed = true;
                atomicOr(status, ST_WAIT_TIMEOUT);
            }
            if (failed) continue;
            T* pe = Bx + par * S::BOX + k * S::BX + i + S::PADX;
            T* po = pe + 4 * S::BOX;
            T e[P], o[P];
#pragma unroll
            for (int j = 0; j < P; ++j) {
                e[j] = pe[j * ZS];
                o[j] = po[j * ZS];
            }
            lift_inverse<T, P, true>(e, o);
#pragma unroll
            for (int j = 2; j < P - 2; ++j) {
                pe[j * ZS] = e[j];
                po[j * ZS] = o[j];
            }
        }
    }
    __syncthreads();
    // ---- X: every (y, z) row of the Z outputs, one window over the row; the
    // x-even and x-odd halves of a row are read and written as 16-byte vectors
    {
        constexpr int P = UX / 2 + 4;
        constexpr int NV = S::BX / S::V; // 16-byte vectors per box row
        for (int L = tid; L < S::FY * UZ; L += kThreads) {
            const int fy = L % S::FY, fz = 4 + L / S::FY;
            T* re = Bx + ((fz & 1) * 4 + (fy & 1) * 2) * S::BOX + ((fz >> 1) * S::HY + (fy >> 1)) * S::BX;
            T* ro = re + S::BOX;
            T ve[S::BX], vo[S::BX];
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                *reinterpret_cast<uint4*>(ve + q * S::V) = reinterpret_cast<const uint4*>(re)[q];
                *reinterpret_cast<uint4*>(vo + q * S::V) = reinterpret_cast<const uint4*>(ro)[q];
            }
            T e[P], o[P];
#pragma unroll
            for (int j = 0; j < P; ++j) {
                e[j] = ve[S::PADX + j];
                o[j] = vo[S::PADX + j];
            }
            lift_inverse<T, P, false>(e, o);
#pragma unroll
            for (int j = 2; j < P - 2; ++j) {
                ve[S::PADX + j] = e[j];
                vo[S::PADX + j] = o[j];
            }
            // slots PADX+2 .. PADX+P-3 changed: whole vectors from (PADX+2)/V on
            static_assert((S::PADX + 2) % S::V == 0, "X outputs start on a vector");
#pragma unroll
            for (int q = (S::PADX + 2) / S::V; q < (S::PADX + P - 2 + S::V - 1) / S::V; ++q) {
                reinterpret_cast<uint4*>(re)[q] = *reinterpret_cast<const uint4*>(ve + q * S::V);
                reinterpret_cast<uint4*>(ro)[q] = *reinterpret_cast<const uint4*>(vo + q * S::V);
            }
        }
    }
    __syncthreads();
    // ---- Y: every (x, z) column of the tile, two canonical windows of 8,
    // emitted from registers. Lanes 0-15 take even x, 16-31 odd x, so a warp
    // covers 32 consecutive x.
    {
        constexpr int P = 8 / 2 + 4;
        constexpr int WIN = UY / 8;
        constexpr int K = S::HY; // y slots per parity
        for (int L = tid; L < UX * UZ; L += kThreads) {
            const int zrow = L / UX, xr = L % UX;
            const int u_x = 2 * (xr % (UX / 2)) + xr / (UX / 2); // first half of a row: even x
            const int fx = u_x + 4, fz = zrow + 4;
            const T* pe = Bx + ((fz & 1) * 4 + (fx & 1)) * S::BOX + (fz >> 1) * ZS + (fx >> 1) + S::PADX;
            const T* po = pe + 2 * S::BOX;
            T ye[K], yo[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                ye[k] = pe[k * S::BX];
                yo[k] = po[k * S::BX];
            }
            const uint32_t gx = ox + u_x, gz = oz + zrow;
            const bool live = gx < a.x && gz < a.z;
            // operands the emitter needs (the originals, for repairs) are
            // fetched before the synthesis so their latency overlaps it
            T pre[UY];
            if constexpr (Out::kPrefetch) {
#pragma unroll
                for (int k = 0; k < UY; ++k) pre[k] = (live && oy + k < a.y) ? out.fetch(gx, oy + k, gz) : T(0);
            }
#pragma unroll
            for (int win = 0; win < WIN; ++win) {
                T e[P], o[P];
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    e[j] = ye[4 * win + j];
                    o[j] = yo[4 * win + j];
                }
                lift_inverse<T, P, true>(e, o);
                if (live) {
#pragma unroll
                    for (int j = 2; j < P - 2; ++j) {
                        const uint32_t gy = oy + win * 8 + 2 * (j - 2);
                        if constexpr (Out::kPrefetch) {
                            if (gy < a.y) out.emit(gx, gy, gz, e[j], pre[win * 8 + 2 * (j - 2)]);
                            if (gy + 1 < a.y) out.emit(gx, gy + 1, gz, o[j], pre[win * 8 + 2 * (j - 2) + 1]);
                        } else {
                            if (gy < a.y) out(gx, gy, gz, e[j]);
                            if (gy + 1 < a.y) out(gx, gy + 1, gz, o[j]);
                        }
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Inverse XY level of the plane schedule from TMA-staged parity boxes: the
// same scheme with the z axis untouched. A tile is UX x UY outputs on UZ
// consecutive planes; its footprint maps to four boxes (x and y parity), each
// (UX/2+4) x (UY/2+4) x UZ, the all-even box from the reconstructed low band
// when there is one. X is lifted over each footprint row in place (one
// window per row), then Y over each tile column in two canonical windows of
// 8 from registers, emitted to `Out`.
template <class T> struct InvTileXY;
template <> struct InvTileXY<float> {
    static constexpr int UX = 32, UY = 16, UZ = 8;
};
template <> struct InvTileXY<double> {
    static constexpr int UX = 16, UY = 16, UZ = 8;
};

template <class T, int UX, int UY, int UZ> struct InvXYShape {
    static constexpr int V = 16 / int(sizeof(T));
    static constexpr int HX = UX / 2 + 4, HY = UY / 2 + 4;
    static constexpr int PADX = (V - 2 % V) % V;          // box x origin = ox/2 - 2 - PADX (16-byte aligned)
    static constexpr int BX = (HX + PADX + V - 1) / V * V;
    static constexpr int BOX = UZ * HY * BX;               // elements per parity box
    static constexpr int FX = UX + 8, FY = UY + 8;
    static constexpr size_t smem = size_t(4) * BOX * sizeof(T) + 128 + 16;
    static_assert((BOX * sizeof(T)) % 128 == 0, "parity boxes must stay 128-byte aligned");
    static_assert(UX % (2 * V) == 0 && UY % 8 == 0 && UZ >= 1 && UZ <= 256, "tile shape");
};

template <class T, int UX, int UY, int UZ, class Out> struct InvTileXYOp {
    static constexpr int kThreads = 256, kMinBlocks = 3;
    static constexpr bool kGridConstant = true;
    struct Params {
        CUtensorMap cmap, lmap;
        InvLevel<T> lv;
        uint32_t tiles_x, tiles_y;
        Out out;
        uint32_t* status;
    };
    static __device__ __forceinline__ void run(const Params& P, uint32_t block, uint32_t);
    static __device__ __forceinline__ void acquire_maps(const Params& P) {
        tensormap_acquire(&P.cmap);
        if (P.lv.low) tensormap_acquire(&P.lmap);
    }
};

template <class T, int UX, int UY, int UZ, class Out>
__device__ __forceinline__ void InvTileXYOp<T, UX, UY, UZ, Out>::run(const Params& P, uint32_t block, uint32_t) {
    const InvLevel<T> lv = P.lv;
    const uint32_t tiles_x = P.tiles_x, tiles_y = P.tiles_y;
    const Out out = P.out;
    uint32_t* const status = P.status;
    using S = InvXYShape<T, UX, UY, UZ>;
    extern __shared__ __align__(128) unsigned char inv_smem[];
    T* Bx = reinterpret_cast<T*>(inv_smem + ((128 - (smem_u32(inv_smem) & 127)) & 127));
    uint64_t* bar = reinterpret_cast<uint64_t*>(Bx + 4 * S::BOX);
    const int tid = threadIdx.x, warp = tid >> 5;
    const Dims a = lv.a;
    const uint32_t bx = block % tiles_x, by = (block / tiles_x) % tiles_y, bz = block / (tiles_x * tiles_y);
    const uint32_t ox = bx * UX, oy = by * UY, oz = bz * UZ;
    const uint32_t hx = half_len(a.x), hy = half_len(a.y);
    const int nz = int(min(uint32_t(UZ), a.z - oz)); // planes of this tile inside the array

    // staged cell of footprint position (fx, fy) on tile plane z
    auto cell = [&](int fx, int fy, int z) -> T* {
        return Bx + ((fy & 1) * 2 + (fx & 1)) * S::BOX + (z * S::HY + (fy >> 1)) * S::BX + (fx >> 1) + S::PADX;
    };

    // ---- stage the four parity boxes
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
        mbar_expect_tx(bar, uint32_t(4 * S::BOX * sizeof(T)));
        const int x0 = int(ox / 2) - 2 - S::PADX, y0 = int(oy / 2) - 2;
#pragma unroll 1
        for (int b = 0; b < 4; ++b) {
            const int xp = b & 1, yp = b >> 1;
            const bool from_low = b == 0 && lv.low != nullptr;
            tma_load_3d(Bx + b * S::BOX, from_low ? &P.lmap : &P.cmap, x0 + (xp ? int(hx) : 0),
                        y0 + (yp ? int(hy) : 0), int(oz), bar);
        }
    }
    {
        const bool ok = __syncthreads_and(warp != 0 || mbar_wait(bar, 0, kWaitBound));
        if (!ok) {
            if (tid == 0) atomicOr(status, ST_WAIT_TIMEOUT);
            return;
        }
    }
    // ---- edge tiles: out-of-range cells of the in-array planes from their
    // reflections (cells of in-range rows left or right of the in-range box,
    // then whole out-of-range rows, as one flat list per plane)
    const bool edge = ox < 4 || ox + UX + 4 > a.x || oy < 4 || oy + UY + 4 > a.y;
    if (edge) {
        const int fx_lo = ox < 4 ? int(4 - ox) : 0, fx_hi = min(S::FX, int(a.x - ox) + 4);
        const int fy_lo = oy < 4 ? int(4 - oy) : 0, fy_hi = min(S::FY, int(a.y - oy) + 4);
        const int nx_out = fx_lo + (S::FX - fx_hi), ny_in = fy_hi - fy_lo, ny_out = S::FY - ny_in;
        const int na = ny_in * nx_out, per = na + ny_out * S::FX;
        for (int i = tid; i < per * nz; i += kThreads) {
            const int z = i / per, r = i - z * per;
            int fx, fy;
            if (r < na) {
                const int k = r % nx_out;
                fy = fy_lo + r / nx_out;
                fx = k < fx_lo ? k : fx_hi + (k - fx_lo);
            } else {
                const int j = r - na, ks = j / S::FX;
                fx = j % S::FX;
                fy = ks < fy_lo ? ks : fy_hi + (ks - fy_lo);
            }
            const uint32_t mx = mirror(int64_t(ox) + fx - 4, a.x), my = mirror(int64_t(oy) + fy - 4, a.y);
            const int64_t gx = int64_t(mx) - (int64_t(ox) - 4), gy = int64_t(my) - (int64_t(oy) - 4);
            T v;
            if (gx >= 0 && gx < S::FX && gy >= 0 && gy < S::FY) {
                v = *cell(int(gx), int(gy), z);
            } else {
                const uint32_t cx = split_of(mx, a.x), cy = split_of(my, a.y), pz = oz + uint32_t(z);
                if (lv.low && cx < lv.lo.x && cy < lv.lo.y)
                    v = lv.low[(size_t(pz) * lv.lo.y + cy) * lv.lo.x + cx];
                else
                    v = lv.base[size_t(pz) * lv.sz + size_t(cy) * lv.sy + cx];
            }
            *cell(fx, fy, z) = v;
        }
        __syncthreads();
    }
    // ---- X: every footprint row of the in-array planes, one window over the
    // row; the x-even and x-odd halves are read and written as 16-byte vectors
    {
        constexpr int P = UX / 2 + 4;
        constexpr int NV = S::BX / S::V;
        for (int L = tid; L < S::FY * nz; L += kThreads) {
            const int fy = L % S::FY, z = L / S::FY;
            T* re = Bx + ((fy & 1) * 2) * S::BOX + (z * S::HY + (fy >> 1)) * S::BX;
            T* ro = re + S::BOX;
            T ve[S::BX], vo[S::BX];
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                *reinterpret_cast<uint4*>(ve + q * S::V) = reinterpret_cast<const uint4*>(re)[q];
                *reinterpret_cast<uint4*>(vo + q * S::V) = reinterpret_cast<const uint4*>(ro)[q];
            }
            T e[P], o[P];
#pragma unroll
            for (int j = 0; j < P; ++j) {
                e[j] = ve[S::PADX + j];
                o[j] = vo[S::PADX + j];
            }
            lift_inverse<T, P, false>(e, o);
#pragma unroll
            for (int j = 2; j < P - 2; ++j) {
                ve[S::PADX + j] = e[j];
                vo[S::PADX + j] = o[j];
            }
            static_assert((S::PADX + 2) % S::V == 0, "X outputs start on a vector");
#pragma unroll
            for (int q = (S::PADX + 2) / S::V; q < (S::PADX + P - 2 + S::V - 1) / S::V; ++q) {
                reinterpret_cast<uint4*>(re)[q] = *reinterpret_cast<const uint4*>(ve + q * S::V);
                reinterpret_cast<uint4*>(ro)[q] = *reinterpret_cast<const uint4*>(vo + q * S::V);
            }
        }
    }
    __syncthreads();
    // ---- Y: every (x, plane) column of the tile, two canonical windows of 8,
    // emitted from registers; lanes 0-15 take even x, 16-31 odd x
    {
        constexpr int P = 8 / 2 + 4;
        constexpr int WIN = UY / 8;
        constexpr int K = S::HY;
        for (int L = tid; L < UX * nz; L += kThreads) {
            const int zrow = L / UX, xr = L % UX;
            const int u_x = 2 * (xr % (UX / 2)) + xr / (UX / 2);
            const int fx = u_x + 4;
            const T* pe = Bx + (fx & 1) * S::BOX + zrow * S::HY * S::BX + (fx >> 1) + S::PADX;
            const T* po = pe + 2 * S::BOX;
            T ye[K], yo[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                ye[k] = pe[k * S::BX];
                yo[k] = po[k * S::BX];
            }
            const uint32_t gx = ox + u_x, gz = oz + zrow;
            const bool live = gx < a.x;
            T pre[UY];
            if constexpr (Out::kPrefetch) {
#pragma unroll
                for (int k = 0; k < UY; ++k) pre[k] = (live && oy + k < a.y) ? out.fetch(gx, oy + k, gz) : T(0);
            }
#pragma unroll
            for (int win = 0; win < WIN; ++win) {
                T e[P], o[P];
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    e[j] = ye[4 * win + j];
                    o[j] = yo[4 * win + j];
                }
                lift_inverse<T, P, true>(e, o);
                if (live) {
#pragma unroll
                    for (int j = 2; j < P - 2; ++j) {
                        const uint32_t gy = oy + win * 8 + 2 * (j - 2);
                        if constexpr (Out::kPrefetch) {
                            if (gy < a.y) out.emit(gx, gy, gz, e[j], pre[win * 8 + 2 * (j - 2)]);
                            if (gy + 1 < a.y) out.emit(gx, gy + 1, gz, o[j], pre[win * 8 + 2 * (j - 2) + 1]);
                        } else {
                            if (gy < a.y) out(gx, gy, gz, e[j]);
                            if (gy + 1 < a.y) out(gx, gy + 1, gz, o[j]);
                        }
                    }
                }
            }
        }
    }
}

} // namespace wb

// Device code of the B200 wave stepper: one time step of WaveSolver::run
// (cpp/include/acoustic_spaces/fdtd.hpp:786-904 of naelolaiz/acoustic-spaces) as four kernels.
//
// A step reads the current pressure b and branch velocities wb, and writes the next pressure over
// the previous one in a, the branch velocities over wa and the matched layer's state in place.
// Each cell's new value depends only on b, wb and its own a, wa and layer state, so the four kinds
// of work (interior air, special rows, matched-layer cells, probe records) write disjoint memory.
//
// Fields live on the device in a pitched layout: cell (x, y, z) at x + pitch * (y + ny * z), with
// pitch = nx rounded up to 16 cells, so that every row starts 64-byte aligned and the tensor maps
// of the bulk sweep meet TMA's 16-byte rules. The cells x >= nx of a row are solid and hold 0.
//
// Arithmetic: built with --fmad=false and -ftz=true; every expression keeps the reference's
// operands in the reference's order, so with T = float each operation rounds as the reference's
// -ffp-contract=off build does, subnormal results flushed to zero as its MXCSR flush does
// (fdtd.hpp:316-336). T = double steps the same layout with every stored coefficient promoted.
//
// COMP (compensated single precision, float only) steps the same scheme on the pressure p_n and
// its increment d_n = p_n - p_(n-1), kept in place of the previous level: with p_(n-1) = p_n - d_n
// written into the updates, every neighbour enters as a difference (p_m - p_n) and the constant
// mode's residual (fdtd_compensated.h) times p_n; then p_(n+1) = p_n + d_(n+1). The increment is
// rounded relative to itself, not to the pressure, so that rounding no longer drives a long run's
// slow modes. A matched-layer cell carries its pressure on from its own rather than summing its
// split parts, which grow far beyond the pressure under a net mass.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace fdtd {

constexpr int kSolid = 0, kInterior = 1, kSpecial = 2, kLayer = 3;
constexpr int kBlock = 128;  // threads per block of every kernel
// A matched-layer cell's state — its three pressure parts and the velocities on its three + faces —
// sits together, six values a cell in a pitched array (two such arrays, the state a step before and
// the new one): one stream of memory for the state in place of nine.
constexpr int kLayerSlots = 6;

// ---- the bulk sweep's tiles ------------------------------------------------------------------
constexpr int kHX = 4;                          // x halo of the pressure tile: 16 bytes of floats
constexpr uint32_t kSpinLimit = 1u << 24;       // bounded waits: then the block gives up
constexpr int kLayerPerSm = 8;                  // blocks an SM of the matched-layer kernel
constexpr int kSpecialPerSm = 4;                // blocks an SM of the special rows' kernel

// A tile shape of the bulk sweep: TX x TY cells a plane, a ring of STAGES plane stages (the three
// in use and STAGES - 3 loaded ahead), THREADS threads a block. Each thread updates ROWS rows of
// one column.
template <int TX_, int TY_, int STAGES_, int THREADS_ = kBlock, int COLS_ = 1>
struct Shape {
    static constexpr int TX = TX_, TY = TY_, STAGES = STAGES_, THREADS = THREADS_;
    static constexpr int COLS = COLS_;       // adjacent columns a thread (2: pairs of cells, vector loads)
    static constexpr int XT = TX / COLS;     // threads across a row
    static constexpr int BX = TX + 2 * kHX;  // pressure tile width (x halo each side)
    static constexpr int BY = TY + 2;        // pressure tile rows (one halo row each side)
    static constexpr int ROWS = TX * TY / (THREADS * COLS);
    static constexpr int AHEAD = STAGES - 3;
    static_assert(TX % 16 == 0 && (COLS == 1 || COLS == 2) && THREADS % XT == 0 && THREADS % 32 == 0 &&
                      (TX * TY) % (THREADS * COLS) == 0 && STAGES >= 4,
                  "tile shape");
};

// The shapes the library is built with (fdtd_autotune picks one per grid; shape 0 by default):
// 64 x 16 with 5 stages (4 blocks of 52 KB an SM in FP32), 128 x 16 and 64 x 32 with 4 stages (2
// blocks of 80 KB: fewer halo cells a cell, 1.19x against 1.27x), and 32 x 32 with 5 (4 blocks);
// then the first three again with 256 threads a block (4 rows a thread, or 8), twice the warps an
// SM in the same shared memory, for a sweep whose issue waits on its own latencies.
using Shape0 = Shape<64, 16, 5>;
using Shape1 = Shape<128, 16, 4>;
using Shape2 = Shape<64, 32, 4>;
using Shape3 = Shape<32, 32, 5>;
using Shape4 = Shape<64, 16, 5, 256>;
using Shape5 = Shape<128, 16, 4, 256>;
using Shape6 = Shape<64, 32, 4, 256>;
// Pairs of cells a thread (the 7-point stencil's loads and stores two cells wide): 64 x 16 with 128
// threads, 128 x 16 with 256, 64 x 16 with 256.
using Shape7 = Shape<64, 16, 5, 128, 2>;
using Shape8 = Shape<128, 16, 4, 256, 2>;
using Shape9 = Shape<64, 16, 5, 256, 2>;
constexpr int kShapes = 10;
struct ShapeInfo {
    int tx, ty, stages, threads, cols;
};
#define FDTD_SHAPE_INFO(SH) {SH::TX, SH::TY, SH::STAGES, SH::THREADS, SH::COLS}
constexpr ShapeInfo kShapeInfo[kShapes] = {FDTD_SHAPE_INFO(Shape0), FDTD_SHAPE_INFO(Shape1), FDTD_SHAPE_INFO(Shape2),
                                           FDTD_SHAPE_INFO(Shape3), FDTD_SHAPE_INFO(Shape4), FDTD_SHAPE_INFO(Shape5),
                                           FDTD_SHAPE_INFO(Shape6), FDTD_SHAPE_INFO(Shape7), FDTD_SHAPE_INFO(Shape8),
                                           FDTD_SHAPE_INFO(Shape9)};
#undef FDTD_SHAPE_INFO
// The default shape's sizes (the adjoint's sweep keeps them).
constexpr int kTX = Shape0::TX, kTY = Shape0::TY, kBX = Shape0::BX, kBY = Shape0::BY;

constexpr uint32_t align128(uint32_t v) { return (v + 127u) & ~127u; }

// Two adjacent values of T as one vector (8 bytes of float, 16 of double).
template <typename T>
struct Pair;
template <>
struct Pair<float> {
    using type = float2;
};
template <>
struct Pair<double> {
    using type = double2;
};

// One stage of the ring: plane k's pressure tile with halos, and its previous pressure, cell
// types and (with a speed field) scales over the tile's own cells.
template <typename T, bool SCALED, class SH = Shape0>
struct Stage {
    static constexpr uint32_t b_bytes = align128(SH::BY * SH::BX * sizeof(T));
    static constexpr uint32_t a_bytes = align128(SH::TY * SH::TX * sizeof(T));
    static constexpr uint32_t t_bytes = align128(SH::TY * SH::TX);
    static constexpr uint32_t s_bytes = SCALED ? align128(SH::TY * SH::TX * 4) : 0;
    static constexpr uint32_t b_off = 0;
    static constexpr uint32_t a_off = b_off + b_bytes;
    static constexpr uint32_t t_off = a_off + a_bytes;
    static constexpr uint32_t s_off = t_off + t_bytes;
    static constexpr uint32_t bytes = s_off + s_bytes;
    // What the copies of a stage write (the boxes, zero-filled where they leave the grid); a tile
    // whose cells are all interior loads no types (kFullTile).
    static constexpr uint32_t tx_bytes =
        SH::BY * SH::BX * sizeof(T) + SH::TY * SH::TX * sizeof(T) + SH::TY * SH::TX + (SCALED ? SH::TY * SH::TX * 4 : 0);
    static constexpr uint32_t tx_bytes_full = tx_bytes - SH::TY * SH::TX;
    // A tile's first and last stages (planes z0 - 1 and z_end) serve only as the pressure above or
    // below: they carry the pressure tile alone.
    static constexpr uint32_t tx_bytes_halo = SH::BY * SH::BX * sizeof(T);
    static constexpr uint32_t smem = SH::STAGES * bytes + 8 * SH::STAGES;  // + the stages' mbarriers
};

// (The adjoint's sweep steps the forward's list of shape 0 with shape 7's pairs: the same tile.)
static_assert(Shape7::TX == Shape0::TX && Shape7::TY == Shape0::TY && Shape7::STAGES == Shape0::STAGES &&
                  Shape7::THREADS == Shape0::THREADS,
              "shapes 0 and 7 share their tiles and stages");

// A tile list entry's w holds z_end, with this bit set when every cell of the tile, in every one
// of its planes, is interior: its planes' stages then carry no cell types.
constexpr int kFullTile = 1 << 30;

struct BulkArgs {
    void *a;  // the previous pressure, overwritten with the next (T)
    void *d;  // COMP: each cell's increment, updated in place
    float residual;  // COMP: the constant mode's residual (with a speed field, per unit scale)
    uint32_t pitch, ny;
    uint32_t xa, y0, z0, x1, y1, z1;  // tiles start at xa (16-aligned), y0, z0; the box ends x1, y1, z1
    // The tiles that hold interior cells: {x, y, z0, z_end | kFullTile if all interior} each, x
    // 16-aligned; a tile spans the shape's TX x TY cells from (x, y) and the planes z0 .. z_end-1.
    const int4 *tile_list;
    uint32_t tiles;
    float axial, diagonal, centre, total;
    unsigned int *error;  // set to 1 when a wait gives up
};

// ---- PTX helpers (mbarrier, TMA) ---------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_address(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// Waits for the phase of parity `parity` of the barrier, at most kSpinLimit tries.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t spin = 0; spin < kSpinLimit; ++spin) {
        if (mbar_try_wait(bar, parity)) return true;
    }
    return false;
}

// A 3-D tile of the tensor `map` at element coordinates (x, y, z) into shared memory at `dst`,
// completing `bytes` of the barrier's expected transactions.
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int x, int y, int z,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

// The error flag's bits: 1 an interior sweep's wait gave up; kWaitTestBit fdtd_test_wait's.
constexpr unsigned int kWaitTestBit = 2u;

// The failure path of a bounded wait, on its own (fdtd_test_wait): lane 0 polls a flag that
// nothing sets, at most `spins` times, then sets the error flag and returns, as a kernel whose
// wait gave up does; the host reads the flag as a status.
__global__ void wait_test_kernel(const unsigned int *flag, uint32_t spins, unsigned int *error) {
    if (threadIdx.x != 0) return;
    const volatile unsigned int *f = flag;
    for (uint32_t i = 0; i < spins; ++i)
        if (*f) return;
    atomicOr(error, kWaitTestBit);
}

// ---- interior air ------------------------------------------------------------------------------

// Interior air (fdtd.hpp:242-288). The interior cells are covered by tiles of SH::TX x SH::TY cells
// by a chunk of planes along z (a list, only tiles that hold interior cells); each block takes tiles
// blockIdx.x, + gridDim.x, ... and marches each along z. Its planes' stages — plane k's pressure
// tile with halos, previous pressure, types and scales — form one sequence over all its tiles:
// tile m's stages are planes z0-1 .. z_end. Thread 0 issues the sequence with TMA, SH::AHEAD stages
// ahead of the three in use (across tile boundaries too), into a ring of SH::STAGES slots in shared
// memory, each completed on its slot's mbarrier; the block updates plane z from the stages of
// planes z-1, z and z+1, each thread SH::ROWS rows of one column, and stores the new pressure of the
// interior cells. A tile whose cells are all interior (kFullTile) loads no cell types and checks
// none. Every wait is bounded: a block that gives up sets the error flag, lets its copies in flight
// land, and stops.
// The reference's sums in its order: x-1, x+1, y-1, y+1, z-1, z+1, then the twelve edges.
struct TileSpan {
    int xt, yt, z0, z_end;  // the tile's corner and its planes z0 .. z_end-1
    bool full;              // every cell of the tile interior
};

__device__ __forceinline__ TileSpan tile_span(const BulkArgs &p, uint32_t tile) {
    const int4 t = p.tile_list[tile];
    return TileSpan{t.x, t.y, t.z, t.w & (kFullTile - 1), (t.w & kFullTile) != 0};
}

template <typename T, bool WIDE, bool SCALED, bool COMP = false, class SH = Shape0>
__global__ void __launch_bounds__(SH::THREADS) bulk_kernel(const __grid_constant__ CUtensorMap map_b,
                                                      const __grid_constant__ CUtensorMap map_a,
                                                      const __grid_constant__ CUtensorMap map_t,
                                                      const __grid_constant__ CUtensorMap map_s,
                                                      const BulkArgs p) {
    using S = Stage<T, SCALED, SH>;
    constexpr int kStages = SH::STAGES, TX = SH::TX, BX = SH::BX;
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t base = smem_address(smem);
    const uint32_t bars = base + kStages * S::bytes;
    const uint32_t tiles = p.tiles;
    if (blockIdx.x >= tiles) return;  // the whole block alike

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(bars + 8 * s, 1);
        fence_barrier_init();
    }
    __syncthreads();

    // The producer's place in the sequence (thread 0 only): its tile, the next plane to issue,
    // and the count of stages issued.
    uint32_t p_tile = blockIdx.x;
    TileSpan p_span = tile_span(p, p_tile);
    int p_k = p_span.z0 - 1;
    int issued = 0;
    const T axial = (T)p.axial, centre = (T)p.centre, diagonal = (T)p.diagonal, total = (T)p.total;
    const int xl = (threadIdx.x % SH::XT) * SH::COLS;
    const int r0 = (threadIdx.x / SH::XT) * SH::ROWS;
    T *__restrict__ a = static_cast<T *>(p.a);
    T *__restrict__ dd = static_cast<T *>(p.d);
    const T residual = (T)p.residual;
    const uint64_t plane = (uint64_t)p.pitch * p.ny;
    bool ok = true, failed = false;
    int waited = 0;    // stages 0 .. waited-1 complete (this thread's view)
    int position = 0;  // the sequence position of the current tile's stage z0-1

    for (uint32_t tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x) {
        const TileSpan t = tile_span(p, tile);
        const int x = t.xt + xl;
        for (int z = t.z0; z < t.z_end; ++z) {
            const int centre_at = position + (z - t.z0 + 1);  // plane z's stage
            // Refill the slots whose stages are over (up to plane z-2's) with the stages up to
            // SH::AHEAD beyond plane z+1's.
            if (threadIdx.x == 0) {
                fence_proxy_async();
                const int target = centre_at + 2 + SH::AHEAD;  // issue stages .. target-1
                while (issued < target && p_tile < tiles) {
                    const int slot = issued % kStages;
                    const uint32_t stage = base + slot * S::bytes, bar = bars + 8 * slot;
                    const bool halo = p_k < p_span.z0 || p_k >= p_span.z_end;
                    mbar_expect_tx(bar, halo ? S::tx_bytes_halo : (p_span.full ? S::tx_bytes_full : S::tx_bytes));
                    tma_load_3d(stage + S::b_off, &map_b, p_span.xt - kHX, p_span.yt - 1, p_k, bar);
                    if (!halo) {
                        tma_load_3d(stage + S::a_off, &map_a, p_span.xt, p_span.yt, p_k, bar);
                        if (!p_span.full) tma_load_3d(stage + S::t_off, &map_t, p_span.xt, p_span.yt, p_k, bar);
                        if (SCALED) tma_load_3d(stage + S::s_off, &map_s, p_span.xt, p_span.yt, p_k, bar);
                    }
                    ++issued;
                    if (++p_k > p_span.z_end) {
                        p_tile += gridDim.x;
                        if (p_tile < tiles) {
                            p_span = tile_span(p, p_tile);
                            p_k = p_span.z0 - 1;
                        }
                    }
                }
            }
            for (; waited <= centre_at + 1 && ok; ++waited)
                ok = mbar_wait(bars + 8 * (waited % kStages), (waited / kStages) & 1);
            if (ok) {
                const unsigned char *s0 = smem + (centre_at % kStages) * S::bytes;
                const T *bm = reinterpret_cast<const T *>(smem + ((centre_at - 1) % kStages) * S::bytes + S::b_off);
                const T *b0 = reinterpret_cast<const T *>(s0 + S::b_off);
                const T *bp = reinterpret_cast<const T *>(smem + ((centre_at + 1) % kStages) * S::bytes + S::b_off);
                const T *pa = reinterpret_cast<const T *>(s0 + S::a_off);
                const uint8_t *pt = reinterpret_cast<const uint8_t *>(s0 + S::t_off);
                const float *ps = reinterpret_cast<const float *>(s0 + S::s_off);
                // (the thread's first row in the level; row r lies r pitches on)
                const uint64_t row0 = (uint64_t)x + (uint64_t)(t.yt + r0) * p.pitch + (uint64_t)z * plane;
#pragma unroll
                for (int r = 0; r < SH::ROWS; ++r) {
                    const int yl = r0 + r;
                    if constexpr (SH::COLS == 2 && !WIDE) {
                        // Two cells side by side: the pair's pressures, previous pressures, scales
                        // and neighbours above, below, z-1 and z+1 each as one vector load (even
                        // offsets: the tile's x start, the halo and the pitch are even), and the
                        // pair's new pressures as one vector store where both are interior.
                        using V2 = typename Pair<T>::type;
                        const int c = yl * TX + xl;
                        const bool in0 = t.full || pt[c] == kInterior, in1 = t.full || pt[c + 1] == kInterior;
                        if (!in0 && !in1) continue;
                        const int q = (yl + 1) * BX + (xl + kHX);
                        const V2 h = *reinterpret_cast<const V2 *>(b0 + q);
                        const T left = b0[q - 1], right = b0[q + 2];
                        const V2 up = *reinterpret_cast<const V2 *>(b0 + q - BX);
                        const V2 dn = *reinterpret_cast<const V2 *>(b0 + q + BX);
                        const V2 zm = *reinterpret_cast<const V2 *>(bm + q);
                        const V2 zp = *reinterpret_cast<const V2 *>(bp + q);
                        const V2 pv = *reinterpret_cast<const V2 *>(pa + c);
                        T *out = a + (row0 + (uint32_t)r * p.pitch);
                        if constexpr (COMP) {
                            // pv holds the pair's increments; the neighbours as differences, in the
                            // sum's order; the new pressures and increments as one vector store each.
                            const T sum0 = (left - h.x) + (h.y - h.x) + (up.x - h.x) + (dn.x - h.x) + (zm.x - h.x) +
                                           (zp.x - h.x);
                            const T sum1 = (h.x - h.y) + (right - h.y) + (up.y - h.y) + (dn.y - h.y) + (zm.y - h.y) +
                                           (zp.y - h.y);
                            T d0, d1;
                            if (SCALED) {
                                const float2 sv = *reinterpret_cast<const float2 *>(ps + c);
                                const T s0 = (T)sv.x, s1 = (T)sv.y;
                                d0 = pv.x + (s0 * axial) * sum0 + (s0 * residual) * h.x;
                                d1 = pv.y + (s1 * axial) * sum1 + (s1 * residual) * h.y;
                            } else {
                                d0 = pv.x + axial * sum0 + residual * h.x;
                                d1 = pv.y + axial * sum1 + residual * h.y;
                            }
                            T *dout = dd + (row0 + (uint32_t)r * p.pitch);
                            if (in0 && in1) {
                                V2 v, w;
                                v.x = h.x + d0, v.y = h.y + d1, w.x = d0, w.y = d1;
                                *reinterpret_cast<V2 *>(out) = v;
                                *reinterpret_cast<V2 *>(dout) = w;
                            } else if (in0) {
                                out[0] = h.x + d0, dout[0] = d0;
                            } else {
                                out[1] = h.y + d1, dout[1] = d1;
                            }
                            continue;
                        }
                        const T sum0 = left + h.y + up.x + dn.x + zm.x + zp.x;
                        const T sum1 = h.x + right + up.y + dn.y + zm.y + zp.y;
                        T n0, n1;
                        if (SCALED) {
                            const float2 sv = *reinterpret_cast<const float2 *>(ps + c);
                            const T s0 = (T)sv.x, s1 = (T)sv.y;
                            n0 = ((T)2 - total * s0) * h.x + (s0 * axial) * sum0 - pv.x;
                            n1 = ((T)2 - total * s1) * h.y + (s1 * axial) * sum1 - pv.y;
                        } else {
                            n0 = centre * h.x + axial * sum0 - pv.x;
                            n1 = centre * h.y + axial * sum1 - pv.y;
                        }
                        if (in0 && in1) {
                            V2 v;
                            v.x = n0, v.y = n1;
                            *reinterpret_cast<V2 *>(out) = v;
                        } else if (in0) {
                            out[0] = n0;
                        } else {
                            out[1] = n1;
                        }
                    } else {
#pragma unroll
                    for (int k = 0; k < SH::COLS; ++k) {
                        const int c = yl * TX + xl + k;
                        // Outside the interior cells' box, and outside the grid (zero fill), no cell
                        // is interior.
                        if (!t.full && pt[c] != kInterior) continue;
                        const int q = (yl + 1) * BX + (xl + k + kHX);
                        const T here = b0[q];
                        const uint64_t at = row0 + (uint32_t)r * p.pitch + k;
                        if (COMP) {
                            // pa holds the increment; the neighbours as differences, in the sum's order.
                            const T sum = (b0[q - 1] - here) + (b0[q + 1] - here) + (b0[q - BX] - here) +
                                          (b0[q + BX] - here) + (bm[q] - here) + (bp[q] - here);
                            T edges = (T)0;
                            if (WIDE)
                                edges = (b0[q - 1 - BX] - here) + (b0[q + 1 - BX] - here) + (b0[q - 1 + BX] - here) +
                                        (b0[q + 1 + BX] - here) + (bm[q - 1] - here) + (bm[q + 1] - here) +
                                        (bp[q - 1] - here) + (bp[q + 1] - here) + (bm[q - BX] - here) +
                                        (bm[q + BX] - here) + (bp[q - BX] - here) + (bp[q + BX] - here);
                            T step;
                            if (SCALED) {
                                const T sc = (T)ps[c];
                                step = WIDE ? pa[c] + (sc * axial) * sum + (sc * diagonal) * edges + (sc * residual) * here
                                            : pa[c] + (sc * axial) * sum + (sc * residual) * here;
                            } else {
                                step = WIDE ? pa[c] + axial * sum + diagonal * edges + residual * here
                                            : pa[c] + axial * sum + residual * here;
                            }
                            a[at] = here + step;
                            dd[at] = step;
                            continue;
                        }
                        const T sum = b0[q - 1] + b0[q + 1] + b0[q - BX] + b0[q + BX] + bm[q] + bp[q];
                        T next;
                        if (WIDE) {
                            const T edges = b0[q - 1 - BX] + b0[q + 1 - BX] + b0[q - 1 + BX] + b0[q + 1 + BX] +
                                            bm[q - 1] + bm[q + 1] + bp[q - 1] + bp[q + 1] +
                                            bm[q - BX] + bm[q + BX] + bp[q - BX] + bp[q + BX];
                            if (SCALED) {
                                const T sc = (T)ps[c];
                                next = ((T)2 - total * sc) * here + (sc * axial) * sum + (sc * diagonal) * edges - pa[c];
                            } else {
                                next = centre * here + axial * sum + diagonal * edges - pa[c];
                            }
                        } else {
                            if (SCALED) {
                                const T sc = (T)ps[c];
                                next = ((T)2 - total * sc) * here + (sc * axial) * sum - pa[c];
                            } else {
                                next = centre * here + axial * sum - pa[c];
                            }
                        }
                        a[at] = next;
                    }
                    }
                }
            }
            // Every thread is done with plane z-1's stage; stop the block alike if a wait gave up.
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
        }
        position += t.z_end - t.z0 + 2;
    }
    if (failed) {  // the same in every thread of the block
        // Give up: report it, and let the copies in flight land before the block's shared
        // memory is released (each wait bounded again).
        if (threadIdx.x == 0) {
            atomicOr(p.error, 1u);
            for (int k = waited; k < issued; ++k) mbar_wait(bars + 8 * (k % kStages), (k / kStages) & 1);
        }
        __syncthreads();
    }
}

// ---- special rows, matched layer, probes -------------------------------------------------------

// Division of 32-bit indices by a divisor fixed at set-up (a row's pitch, a plane's cells) by one
// multiply-high and two shifts, Granlund and Montgomery's method for run-time invariant unsigned
// divisors ("Division by invariant integers using multiplication", 1994, figure 4.1): with
// l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1, t = mulhi(m, n) gives
// n / d = (t + ((n - t) >> 1)) >> (l - 1) for every 32-bit n (d >= 2).
struct FastDiv {
    uint32_t m = 0, shift = 0;
    FastDiv() = default;
    explicit FastDiv(uint32_t d) {
        uint32_t l = 0;
        while ((1ull << l) < d) ++l;
        m = (uint32_t)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
        shift = l - 1;
    }
    __host__ __device__ __forceinline__ uint32_t operator()(uint32_t n) const {
#ifdef __CUDA_ARCH__
        const uint32_t t = __umulhi(m, n);
#else
        const uint32_t t = (uint32_t)(((uint64_t)m * n) >> 32);
#endif
        return (t + ((n - t) >> 1)) >> shift;
    }
};

struct Tables {
    uint32_t pitch, ny, nz, sz;
    // Special rows (fdtd.hpp:860-881), as structure of arrays.
    uint32_t specials;
    const uint32_t *special, *state_start;
    // Each row's links as a slot-major table (slot l of row k at l * specials + k), in the
    // layout's order, and each row's count of links.
    uint32_t link_slots;
    const uint8_t *link_count, *link_direction;
    const float *link_weight, *coef_a, *coef_b, *coef_inv, *source;
    // Where every row's links are axial, in the directions' order, each of the axial weight (walls
    // on cell faces without a speed field), each row's links as a mask of the six directions
    // instead (special_kernel<T, 0>): one byte a row in place of five a link.
    const uint8_t *link_mask;
    float link_axial;
    const float *row_residual;  // COMP: each row's constant-mode residual
    const float *state_weight, *state_now, *state_before, *state_gain;
    int32_t offset[18];
    // Matched layer (fdtd.hpp:2242-2264): cells, and per axis and grid coordinate x (0..n_axis)
    // {keep of the centre, push of the centre, keep of the face below, push of the face below}
    // (layer_coefficients, fdtd.hpp:2219-2238); with a speed field each cell's scale.
    uint32_t layers;
    const uint32_t *layer_cells;
    const float *layer_scale;
    const float4 *layer_coef[3];
    const uint8_t *layer_below;  // bit a: the cell below along axis a is in the layer too
    uint32_t plane;  // pitch * ny
    FastDiv by_plane, by_pitch;  // a pitched index's plane, and its row within the plane
    // With a tangent of the layer's tables (fdtd_set_layer_tangent): per axis and coordinate the
    // tangent of the centre's {keep, push} and of the face's {keep, push}; each layer cell's axes
    // along which the tangent touches it (bit a: at its coordinate or the one after), and the place
    // of its first factor among a step's (three per such axis, axis by axis).
    const double2 *tangent_centre[3], *tangent_face[3];
    const uint8_t *tangent_axes;
    const uint32_t *tangent_start;
    // Probes (fdtd.hpp:3525-3533).
    uint32_t probes;
    const uint32_t *probe_start, *probe_cells;
    const double *probe_weights;
};

template <typename T>
struct Fields {
    T *a;              // the pressure a step before, overwritten with the next
    T *d;              // COMP: each cell's increment p_n - p_(n-1), updated in place
    const T *b;        // the current pressure
    T *wa;             // branch velocities a step before, overwritten with the next
    const T *wb;       // current branch velocities
    // The matched layer's state, kLayerSlots values a (pitched) cell: at kLayerSlots i + axis the
    // layer cell's pressure part along that axis, at kLayerSlots i + 3 + axis the velocity on its
    // + face along it (also kept at a cell outside the layer whose + face is a layer cell's - face).
    const T *cell_old;  // a step before
    T *cell_new;        // this step
    const float *signal;  // the step's drive at signal[0]
    double *out;       // probe p's record at out[p * out_stride]
    uint64_t out_stride;
    T *traj_u;         // when not null: each special row's new pressure at traj_u[k] (the gradient's
    T *traj_w;         // recomputation), and each branch state's new velocity at traj_w[j]
    // When not null (the gradient's recomputation of a grid with a matched layer): each layer
    // cell's six factors per axis of the tables' gradient, at traj_layer[f * layers + c]
    // (fdtd_adjoint.cuh: q, hi' - lo', hi, b_(i+st) - b_i, lo, b_i - b_(i-st) per axis).
    T *traj_layer;
    // When not null (a run recording for a gradient along a tangent of the layer's tables): each
    // layer cell's tangent factors of the step at traj_tangent[tangent_start[c] + 3 j + f], j its
    // j-th axis of tangent_axes (fdtd_adjoint.cuh: the centre's, the + face's, the - face's).
    T *traj_tangent;
};

// Special rows (fdtd.hpp:860-881), one a thread: its links, its branch states' flow, the update,
// then the branch velocities. The links' table is slot-major, so that a warp's loads of a slot
// are coalesced; all of a row's link loads are issued before the sum, which then adds them in
// the layout's order. A state's term now * wb - before * wa is worked out again for the
// velocities' update rather than kept: wa has not changed in between, so it is the same value.
// The links' tables are read once a step and the new pressure by no kernel of the same step, so
// those go through the caches as streaming (evict-first) accesses, leaving L2 to the pressures
// that the sweep and the layer share with the rows (measured: the concurrent step 2 % shorter).
template <typename T, int SLOTS, bool COMP>
__device__ __forceinline__ void special_row(const Tables &g, const Fields<T> &f, const uint32_t k, const uint32_t i,
                                            const uint32_t links, const uint32_t s0, const uint32_t s1) {
    const uint32_t K = g.specials;
    const T *__restrict__ b = f.b;
    T sum = 0;
    T here;
    if constexpr (SLOTS == 0) {
        // The links as a mask of the axial directions, in their order, each of the axial weight.
        const uint32_t mask = g.link_mask[k];
        T value[6];
#pragma unroll
        for (int d = 0; d < 6; ++d) value[d] = (mask >> d) & 1u ? b[(uint32_t)((int64_t)i + g.offset[d])] : (T)0;
        here = b[i];
        const T w = (T)g.link_axial;
#pragma unroll
        for (int d = 0; d < 6; ++d)
            if ((mask >> d) & 1u) sum += COMP ? w * (value[d] - here) : w * value[d];
    } else {
        T value[SLOTS];
        float weight[SLOTS];
#pragma unroll
        for (int l = 0; l < SLOTS; ++l) {
            value[l] = (T)0;
            weight[l] = 0.0f;
            if ((uint32_t)l < links) {
                const uint32_t at = l * K + k;
                weight[l] = __ldcs(g.link_weight + at);
                value[l] = b[(uint32_t)((int64_t)i + g.offset[__ldcs(g.link_direction + at)])];
            }
        }
        here = b[i];
#pragma unroll
        for (int l = 0; l < SLOTS; ++l)
            if ((uint32_t)l < links) sum += COMP ? (T)weight[l] * (value[l] - here) : (T)weight[l] * value[l];
    }
    T flow = 0;
    for (uint32_t j = s0; j < s1; ++j) {
        const T own = (T)g.state_now[j] * f.wb[j] - (T)g.state_before[j] * f.wa[j];
        flow += (T)g.state_weight[j] * own;
    }
    if (COMP) {
        const T before = f.d[i];
        const T step = (sum + (T)g.coef_b[k] * before - flow + (T)g.source[k] * (T)f.signal[0]) * (T)g.coef_inv[k] +
                       (T)g.row_residual[k] * here;
        f.a[i] = here + step;
        f.d[i] = step;
        for (uint32_t j = s0; j < s1; ++j) {
            const T own = (T)g.state_now[j] * f.wb[j] - (T)g.state_before[j] * f.wa[j];
            f.wa[j] = f.wa[j] + ((step + before) * (T)g.state_gain[j] + own);
        }
        return;
    }
    const T previous = f.a[i];
    const T next = ((T)g.coef_a[k] * here + sum - (T)g.coef_b[k] * previous - flow +
                    (T)g.source[k] * (T)f.signal[0]) * (T)g.coef_inv[k];
    __stcs(f.a + i, next);
    if (f.traj_u) f.traj_u[k] = next;
    for (uint32_t j = s0; j < s1; ++j) {
        const T own = (T)g.state_now[j] * f.wb[j] - (T)g.state_before[j] * f.wa[j];
        const T w = f.wa[j] + ((next - previous) * (T)g.state_gain[j] + own);
        f.wa[j] = w;
        if (f.traj_w) f.traj_w[j] = w;
    }
}

// Rows k, k + the grid's threads, ... a thread, the next row's cell index, link count and branch
// states' bounds loaded while this row's loads are in flight, so that a row's link loads wait on
// no load of its own (measured: the kernel 10 % shorter on the fitted rows).
template <typename T, int SLOTS, bool COMP = false>
__global__ void __launch_bounds__(kBlock) special_kernel(const Tables g, const Fields<T> f) {
    const uint32_t K = g.specials;
    const uint32_t step = gridDim.x * kBlock;
    uint32_t k = blockIdx.x * kBlock + threadIdx.x;
    if (k >= K) return;
    uint32_t next = g.special[k];
    uint32_t next_links = SLOTS ? (uint32_t)__ldcs(g.link_count + k) : 0u;
    uint32_t next_s0 = g.state_start[k], next_s1 = g.state_start[k + 1];
    for (; k < K; k += step) {
        const uint32_t i = next, links = next_links, s0 = next_s0, s1 = next_s1;
        if (k + step < K) {
            next = g.special[k + step];
            if (SLOTS) next_links = __ldcs(g.link_count + k + step);
            next_s0 = g.state_start[k + step], next_s1 = g.state_start[k + step + 1];
        }
        special_row<T, SLOTS, COMP>(g, f, k, i, links, s0, s1);
    }
}

// Matched-layer cells (fdtd.hpp:2242-2264), one a thread: per axis the cell's two face
// velocities, then its pressure part; the cell's pressure is the parts' sum.
//
// The reference keeps, per layer cell, its own copy of the velocity on each of its six faces
// (fdtd.hpp:2245), and both cells of a face update their copies alike: cell i's + face along an
// axis of stride s and cell i+s's - face take keep_face[x+1] * u - push_face[x+1] * (b[i+s] -
// b[i]) from the same value, so that, both starting at 0, the two copies stay equal to the bit.
// Here each face is kept once, on the cell below it (face[i] is cell i's + face), in two buffers
// that alternate with the steps: every cell reads the old values of its two faces and works both
// out again, and writes the new value of its + face, and of its - face too where the cell below
// is not in the layer (no one else writes that face). The pressure parts stay per cell.
template <typename T, bool SCALED, bool COMP>
__device__ __forceinline__ void layer_cell(const Tables &g, const Fields<T> &f, const uint32_t c, const uint32_t i) {
    const uint32_t L = g.layers;
    // Every load of the cell first — its parts, its pressure and its six neighbours', its faces'
    // old velocities and the coefficients — so that they are in flight together; then the
    // reference's arithmetic, axis by axis; then the stores, as streaming (evict-first) stores:
    // the new state and pressure are read by no kernel of the same step.
    const uint32_t z = g.by_plane(i), r = i - z * g.plane, y = g.by_pitch(r);
    const uint32_t at[3] = {r - y * g.pitch, y, z};
    const uint32_t strides[3] = {1u, g.pitch, g.plane};
    const T *__restrict__ b = f.b;
    using V2 = typename Pair<T>::type;
    T part[3], lo[3], hi[3], old_below[3], old_above[3];
    float4 c0[3], c1[3];
    {
        // the cell's own state in three vector loads: parts x, y; part z, face x; faces y, z
        const V2 *own = reinterpret_cast<const V2 *>(f.cell_old + (uint64_t)kLayerSlots * i);
        const V2 s0 = own[0], s1 = own[1], s2 = own[2];
        part[0] = s0.x, part[1] = s0.y, part[2] = s1.x;
        old_above[0] = s1.y, old_above[1] = s2.x, old_above[2] = s2.y;
    }
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const uint32_t stride = strides[axis];
        lo[axis] = b[i - stride];
        hi[axis] = b[i + stride];
        old_below[axis] = f.cell_old[(uint64_t)kLayerSlots * (i - stride) + 3 + axis];
        c0[axis] = __ldg(g.layer_coef[axis] + at[axis]);
        c1[axis] = __ldg(g.layer_coef[axis] + at[axis] + 1);
    }
    const T here = b[i];
    const T scale = SCALED ? (T)g.layer_scale[c] : (T)1;
    const uint32_t shared_below = g.layer_below[c];
    const uint32_t tangent_axes = f.traj_tangent ? g.tangent_axes[c] : 0u;
    uint32_t tangent_slot = f.traj_tangent ? g.tangent_start[c] : 0u;
    T below[3], above[3];
    T total = 0;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        below[axis] = (T)c0[axis].z * old_below[axis] - (T)c0[axis].w * (here - lo[axis]);
        above[axis] = (T)c1[axis].z * old_above[axis] - (T)c1[axis].w * (hi[axis] - here);
        if (COMP) {
            // The parts' sum carried on from the pressure: p + (keep - 1) * part - flux per axis.
            const T keep = (T)c0[axis].x;
            const T push = SCALED ? (T)c0[axis].y * scale : (T)c0[axis].y;
            const T flux = push * (above[axis] - below[axis]);
            total += (keep - (T)1) * part[axis] - flux;
            part[axis] = keep * part[axis] - flux;
            continue;
        }
        if (f.traj_tangent && (tangent_axes & (1u << axis))) {
            // The step's factors along the tangent: its products with the adjoints of the new part
            // and faces give the gradient's step (fdtd_adjoint.cuh), in double.
            const double2 tc = g.tangent_centre[axis][at[axis]];
            const double2 t0 = g.tangent_face[axis][at[axis]], t1 = g.tangent_face[axis][at[axis] + 1];
            T *o = f.traj_tangent + tangent_slot;
            tangent_slot += 3;
            o[0] = (T)((double)part[axis] * tc.x - (double)scale * (double)(above[axis] - below[axis]) * tc.y);
            o[1] = (T)((double)old_above[axis] * t1.x - (double)(hi[axis] - here) * t1.y);
            o[2] = (T)((double)old_below[axis] * t0.x - (double)(here - lo[axis]) * t0.y);
        }
        if (f.traj_layer) {
            T *o = f.traj_layer + (uint64_t)(6 * axis) * L + c;
            o[0] = part[axis];
            o[(uint64_t)1 * L] = above[axis] - below[axis];
            o[(uint64_t)2 * L] = old_above[axis];
            o[(uint64_t)3 * L] = hi[axis] - here;
            o[(uint64_t)4 * L] = old_below[axis];
            o[(uint64_t)5 * L] = here - lo[axis];
        }
        if (SCALED) {
            part[axis] = (T)c0[axis].x * part[axis] - ((T)c0[axis].y * scale) * (above[axis] - below[axis]);
        } else {
            part[axis] = (T)c0[axis].x * part[axis] - (T)c0[axis].y * (above[axis] - below[axis]);
        }
        total += part[axis];
    }
    {
        V2 *own = reinterpret_cast<V2 *>(f.cell_new + (uint64_t)kLayerSlots * i);
        V2 s0, s1, s2;
        s0.x = part[0], s0.y = part[1], s1.x = part[2], s1.y = above[0], s2.x = above[1], s2.y = above[2];
        __stcs(own, s0), __stcs(own + 1, s1), __stcs(own + 2, s2);
    }
    // The cell below owns the face when it is in the layer; else this cell keeps it there.
#pragma unroll
    for (int axis = 0; axis < 3; ++axis)
        if (!(shared_below & (1u << axis))) __stcs(f.cell_new + (uint64_t)kLayerSlots * (i - strides[axis]) + 3 + axis, below[axis]);
    if (COMP) {
        f.a[i] = here + total;
        f.d[i] = total;  // (read by no update; it keeps the state's level before readable)
    } else {
        __stcs(f.a + i, total);
    }
}

// A grid of a few blocks an SM (the sweep's blocks keep their places beside it), each thread taking
// cells c, c + the grid's threads, ...; the next cell's index is loaded while this cell's loads are
// in flight, so that a cell costs one round trip to memory rather than two.
template <typename T, bool SCALED, bool COMP = false>
__global__ void __launch_bounds__(kBlock) layer_kernel(const Tables g, const Fields<T> f) {
    const uint32_t L = g.layers;
    const uint32_t step = gridDim.x * kBlock;
    uint32_t c = blockIdx.x * kBlock + threadIdx.x;
    if (c >= L) return;
    uint32_t next = g.layer_cells[c];
    for (; c < L; c += step) {
        const uint32_t i = next;
        if (c + step < L) next = g.layer_cells[c + step];
        layer_cell<T, SCALED, COMP>(g, f, c, i);
    }
}

// Probe p's pressure before the step (fdtd.hpp:3525-3533): its cells' weighted sum in double, in
// the layout's order. A warp per probe: the lanes load the cells and form the products (each
// product is the reference's own), then lane 0 adds them up in the layout's order, so that the
// sum rounds as the reference's sequential one.
constexpr int kProbeWarps = kBlock / 32;

template <typename T>
__global__ void __launch_bounds__(kBlock) probe_kernel(const Tables g, const Fields<T> f) {
    const uint32_t p = blockIdx.x * kProbeWarps + threadIdx.x / 32;
    const uint32_t lane = threadIdx.x % 32;
    if (p >= g.probes) return;  // the whole warp alike
    const uint32_t start = g.probe_start[p], end = g.probe_start[p + 1];
    double value = 0.0;
    for (uint32_t base = start; base < end; base += 32) {
        const uint32_t k = base + lane;
        const double product = k < end ? g.probe_weights[k] * (double)f.b[g.probe_cells[k]] : 0.0;
        const uint32_t count = min(32u, end - base);
        for (uint32_t l = 0; l < count; ++l) {
            const double term = __shfl_sync(0xffffffffu, product, l);
            if (lane == 0) value += term;
        }
    }
    if (lane == 0) f.out[(uint64_t)p * f.out_stride] = value;
}

}  // namespace fdtd

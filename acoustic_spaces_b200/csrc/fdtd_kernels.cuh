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
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace fdtd {

constexpr int kSolid = 0, kInterior = 1, kSpecial = 2, kLayer = 3;
constexpr int kBlock = 128;  // threads per block of every kernel

// ---- the bulk sweep's tiles ------------------------------------------------------------------
constexpr int kTX = 64;                         // cells of a tile along x
constexpr int kTY = 16;                         // rows of a tile along y
constexpr int kHX = 4;                          // x halo of the pressure tile: 16 bytes of floats
constexpr int kBX = kTX + 2 * kHX;              // 72: pressure tile width
constexpr int kBY = kTY + 2;                    // 18: pressure tile rows (one halo row each side)
constexpr int kRowsPerThread = kTX * kTY / kBlock;  // 8 rows of one column per thread
constexpr int kAhead = 2;                       // planes loaded ahead of the three in use
constexpr int kStages = kAhead + 3;             // ring of plane stages in shared memory
constexpr uint32_t kSpinLimit = 1u << 24;       // bounded waits: then the block gives up

constexpr uint32_t align128(uint32_t v) { return (v + 127u) & ~127u; }

// One stage of the ring: plane k's pressure tile with halos, and its previous pressure, cell
// types and (with a speed field) scales over the tile's own cells.
template <typename T, bool SCALED>
struct Stage {
    static constexpr uint32_t b_bytes = align128(kBY * kBX * sizeof(T));
    static constexpr uint32_t a_bytes = align128(kTY * kTX * sizeof(T));
    static constexpr uint32_t t_bytes = align128(kTY * kTX);
    static constexpr uint32_t s_bytes = SCALED ? align128(kTY * kTX * 4) : 0;
    static constexpr uint32_t b_off = 0;
    static constexpr uint32_t a_off = b_off + b_bytes;
    static constexpr uint32_t t_off = a_off + a_bytes;
    static constexpr uint32_t s_off = t_off + t_bytes;
    static constexpr uint32_t bytes = s_off + s_bytes;
    // What the four copies of a stage write (the boxes, zero-filled where they leave the grid).
    static constexpr uint32_t tx_bytes =
        kBY * kBX * sizeof(T) + kTY * kTX * sizeof(T) + kTY * kTX + (SCALED ? kTY * kTX * 4 : 0);
    static constexpr uint32_t smem = kStages * bytes + 8 * kStages;  // + the stages' mbarriers
};

struct BulkArgs {
    void *a;  // the previous pressure, overwritten with the next (T)
    uint32_t pitch, ny;
    uint32_t xa, y0, z0, x1, y1, z1;  // tiles start at xa (16-aligned), y0, z0; the box ends x1, y1, z1
    uint32_t tiles_x, tiles_y, chunk;
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

// ---- interior air ------------------------------------------------------------------------------

// Thread 0 of a bulk block: the copies of plane k (the block's index-th stage) into its slot of
// the ring, all completing on the slot's barrier.
template <typename T, bool SCALED>
__device__ __forceinline__ void issue_stage(uint32_t base, uint32_t bars, int index, int k, int xt, int yt,
                                            const CUtensorMap *map_b, const CUtensorMap *map_a,
                                            const CUtensorMap *map_t, const CUtensorMap *map_s) {
    using S = Stage<T, SCALED>;
    const int slot = index % kStages;
    const uint32_t stage = base + slot * S::bytes, bar = bars + 8 * slot;
    mbar_expect_tx(bar, S::tx_bytes);
    tma_load_3d(stage + S::b_off, map_b, xt - kHX, yt - 1, k, bar);
    tma_load_3d(stage + S::a_off, map_a, xt, yt, k, bar);
    tma_load_3d(stage + S::t_off, map_t, xt, yt, k, bar);
    if (SCALED) tma_load_3d(stage + S::s_off, map_s, xt, yt, k, bar);
}

// Interior air (fdtd.hpp:242-288). A block owns a tile of kTX x kTY cells of the interior cells'
// bounding box and marches it along z through a chunk of planes. One thread issues, with TMA, each
// plane's stage kAhead planes ahead into a ring of kStages stages in shared memory, each completed
// on its own mbarrier; the block updates plane z from the stages of planes z-1, z and z+1, each
// thread 8 rows of one column. Neighbours come from shared memory, so that every value is read
// from HBM once per block; the new pressure of interior cells is stored to global memory.
// The reference's sums in its order: x-1, x+1, y-1, y+1, z-1, z+1, then the twelve edges.
template <typename T, bool WIDE, bool SCALED>
__global__ void __launch_bounds__(kBlock) bulk_kernel(const __grid_constant__ CUtensorMap map_b,
                                                      const __grid_constant__ CUtensorMap map_a,
                                                      const __grid_constant__ CUtensorMap map_t,
                                                      const __grid_constant__ CUtensorMap map_s,
                                                      const BulkArgs p) {
    using S = Stage<T, SCALED>;
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t base = smem_address(smem);
    const uint32_t bars = base + kStages * S::bytes;

    uint32_t tile = blockIdx.x;
    const uint32_t bx = tile % p.tiles_x;
    tile /= p.tiles_x;
    const uint32_t by = tile % p.tiles_y;
    const uint32_t bz = tile / p.tiles_y;
    const int xt = (int)(p.xa + bx * kTX), yt = (int)(p.y0 + by * kTY);
    const int z0 = (int)(p.z0 + bz * p.chunk);
    const int z_end = min(z0 + (int)p.chunk, (int)p.z1);
    if (z0 >= z_end) return;  // the whole block alike
    // Stages first .. last: planes z0-1 .. z_end, all inside the grid (z0 >= 1, z_end <= nz-1).
    const int first = z0 - 1, last = z_end;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(bars + 8 * s, 1);
        fence_barrier_init();
    }
    __syncthreads();

    int issued = min(last, first + kAhead + 1);  // the last stage issued (thread 0's count)
    if (threadIdx.x == 0) {
        fence_proxy_async();
        for (int k = first; k <= issued; ++k)
            issue_stage<T, SCALED>(base, bars, k - first, k, xt, yt, &map_b, &map_a, &map_t, &map_s);
    }

    const T axial = (T)p.axial, centre = (T)p.centre, diagonal = (T)p.diagonal, total = (T)p.total;
    const int xl = threadIdx.x % kTX;
    const int r0 = (threadIdx.x / kTX) * kRowsPerThread;
    const int x = xt + xl;
    T *__restrict__ a = static_cast<T *>(p.a);
    const uint64_t plane = (uint64_t)p.pitch * p.ny;
    bool ok = true, failed = false;
    int waited = first - 1;  // the last stage waited for

    for (int z = z0; z < z_end; ++z) {
        // Refill the slot of plane z-2 (its last use, plane z-1's update, is over) with plane
        // z+1+kAhead.
        if (threadIdx.x == 0 && z + 1 + kAhead <= last) {
            fence_proxy_async();
            issued = z + 1 + kAhead;
            issue_stage<T, SCALED>(base, bars, issued - first, issued, xt, yt, &map_b, &map_a, &map_t, &map_s);
        }
        // Stages z-1, z and z+1 complete (each waited for once).
        for (int k = waited + 1; k <= z + 1 && ok; ++k) {
            const int index = k - first;
            ok = mbar_wait(bars + 8 * (index % kStages), (index / kStages) & 1);
            waited = k;
        }
        if (ok) {
            const int index = z - first;
            const unsigned char *s0 = smem + (index % kStages) * S::bytes;
            const T *bm = reinterpret_cast<const T *>(smem + ((index - 1) % kStages) * S::bytes + S::b_off);
            const T *b0 = reinterpret_cast<const T *>(s0 + S::b_off);
            const T *bp = reinterpret_cast<const T *>(smem + ((index + 1) % kStages) * S::bytes + S::b_off);
            const T *pa = reinterpret_cast<const T *>(s0 + S::a_off);
            const uint8_t *pt = reinterpret_cast<const uint8_t *>(s0 + S::t_off);
            const float *ps = reinterpret_cast<const float *>(s0 + S::s_off);
#pragma unroll
            for (int r = 0; r < kRowsPerThread; ++r) {
                const int yl = r0 + r;
                const int c = yl * kTX + xl;
                // Outside the interior cells' box, and outside the grid (zero fill), no cell is
                // interior.
                if (pt[c] != kInterior) continue;
                const int q = (yl + 1) * kBX + (xl + kHX);
                const T here = b0[q];
                const T sum = b0[q - 1] + b0[q + 1] + b0[q - kBX] + b0[q + kBX] + bm[q] + bp[q];
                T next;
                if (WIDE) {
                    const T edges = b0[q - 1 - kBX] + b0[q + 1 - kBX] + b0[q - 1 + kBX] + b0[q + 1 + kBX] +
                                    bm[q - 1] + bm[q + 1] + bp[q - 1] + bp[q + 1] +
                                    bm[q - kBX] + bm[q + kBX] + bp[q - kBX] + bp[q + kBX];
                    if (SCALED) {
                        const T s = (T)ps[c];
                        next = ((T)2 - total * s) * here + (s * axial) * sum + (s * diagonal) * edges - pa[c];
                    } else {
                        next = centre * here + axial * sum + diagonal * edges - pa[c];
                    }
                } else {
                    if (SCALED) {
                        const T s = (T)ps[c];
                        next = ((T)2 - total * s) * here + (s * axial) * sum - pa[c];
                    } else {
                        next = centre * here + axial * sum - pa[c];
                    }
                }
                a[(uint64_t)x + (uint64_t)(yt + yl) * p.pitch + (uint64_t)z * plane] = next;
            }
        }
        // Every thread is done with plane z-1's stage; stop the block alike if a wait gave up.
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
    }
    if (failed) {  // the same in every thread of the block
        // Give up: report it, and let the copies in flight land before the block's shared
        // memory is released (each wait bounded again).
        if (threadIdx.x == 0) {
            atomicOr(p.error, 1u);
            for (int k = waited + 1; k <= issued; ++k) {
                const int index = k - first;
                mbar_wait(bars + 8 * (index % kStages), (index / kStages) & 1);
            }
        }
        __syncthreads();
    }
}

// ---- special rows, matched layer, probes -------------------------------------------------------

struct Tables {
    uint32_t pitch, ny, nz, sz;
    // Special rows (fdtd.hpp:860-881), as structure of arrays.
    uint32_t specials;
    const uint32_t *special, *link_start, *state_start;
    const uint8_t *link_direction;
    const float *link_weight, *coef_a, *coef_b, *coef_inv, *source;
    const float *state_weight, *state_now, *state_before, *state_gain;
    int32_t offset[18];
    // Matched layer (fdtd.hpp:2242-2264): cells, and per axis and grid coordinate x (0..n_axis)
    // {keep of the centre, push of the centre, keep of the face below, push of the face below}
    // (layer_coefficients, fdtd.hpp:2219-2238); with a speed field each cell's scale.
    uint32_t layers;
    const uint32_t *layer_cells;
    const float *layer_scale;
    const float4 *layer_coef[3];
    // Probes (fdtd.hpp:3525-3533).
    uint32_t probes;
    const uint32_t *probe_start, *probe_cells;
    const double *probe_weights;
};

template <typename T>
struct Fields {
    T *a;              // the pressure a step before, overwritten with the next
    const T *b;        // the current pressure
    T *wa;             // branch velocities a step before, overwritten with the next
    const T *wb;       // current branch velocities
    T *layer_state;    // 9 arrays of `layers`: p_x, p_y, p_z, u-_x, u+_x, u-_y, u+_y, u-_z, u+_z
    const float *signal;  // the step's drive at signal[0]
    double *out;       // probe p's record at out[p * out_stride]
    uint64_t out_stride;
};

// Special rows (fdtd.hpp:860-881), one a thread: its links, its branch states' flow, the update,
// then the branch velocities. A state's term now * wb - before * wa is worked out again for the
// velocities' update rather than kept: wa has not changed in between, so it is the same value.
template <typename T>
__global__ void __launch_bounds__(kBlock) special_kernel(const Tables g, const Fields<T> f) {
    const uint32_t k = blockIdx.x * kBlock + threadIdx.x;
    if (k >= g.specials) return;
    const uint32_t i = g.special[k];
    const T *__restrict__ b = f.b;
    T sum = 0;
    for (uint32_t l = g.link_start[k], e = g.link_start[k + 1]; l < e; ++l) {
        const uint32_t j = (uint32_t)((int64_t)i + g.offset[g.link_direction[l]]);
        sum += (T)g.link_weight[l] * b[j];
    }
    const uint32_t s0 = g.state_start[k], s1 = g.state_start[k + 1];
    T flow = 0;
    for (uint32_t j = s0; j < s1; ++j) {
        const T own = (T)g.state_now[j] * f.wb[j] - (T)g.state_before[j] * f.wa[j];
        flow += (T)g.state_weight[j] * own;
    }
    const T previous = f.a[i];
    const T next = ((T)g.coef_a[k] * b[i] + sum - (T)g.coef_b[k] * previous - flow +
                    (T)g.source[k] * (T)f.signal[0]) * (T)g.coef_inv[k];
    f.a[i] = next;
    for (uint32_t j = s0; j < s1; ++j) {
        const T own = (T)g.state_now[j] * f.wb[j] - (T)g.state_before[j] * f.wa[j];
        f.wa[j] = f.wa[j] + ((next - previous) * (T)g.state_gain[j] + own);
    }
}

// Matched-layer cells (fdtd.hpp:2242-2264), one a thread: per axis the cell's two face
// velocities, then its pressure part; the cell's pressure is the parts' sum. The state (nine
// arrays over the layer's cells, coalesced) is loaded before anything that depends on the cell's
// place.
template <typename T, bool SCALED>
__global__ void __launch_bounds__(kBlock) layer_kernel(const Tables g, const Fields<T> f) {
    const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
    const uint32_t L = g.layers;
    if (c >= L) return;
    T *st = f.layer_state;
    T part[3], below[3], above[3];
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        part[axis] = st[axis * L + c];
        below[axis] = st[(3 + 2 * axis) * L + c];
        above[axis] = st[(4 + 2 * axis) * L + c];
    }
    const uint32_t i = g.layer_cells[c];
    const uint32_t at[3] = {i % g.pitch, (i / g.pitch) % g.ny, i / g.sz};
    const uint32_t strides[3] = {1u, g.pitch, g.sz};
    const T *__restrict__ b = f.b;
    const T here = b[i];
    const T scale = SCALED ? (T)g.layer_scale[c] : (T)1;
    T total = 0;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const uint32_t stride = strides[axis], x = at[axis];
        const float4 c0 = g.layer_coef[axis][x], c1 = g.layer_coef[axis][x + 1];
        below[axis] = (T)c0.z * below[axis] - (T)c0.w * (here - b[i - stride]);
        above[axis] = (T)c1.z * above[axis] - (T)c1.w * (b[i + stride] - here);
        if (SCALED) {
            part[axis] = (T)c0.x * part[axis] - ((T)c0.y * scale) * (above[axis] - below[axis]);
        } else {
            part[axis] = (T)c0.x * part[axis] - (T)c0.y * (above[axis] - below[axis]);
        }
        total += part[axis];
    }
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        st[axis * L + c] = part[axis];
        st[(3 + 2 * axis) * L + c] = below[axis];
        st[(4 + 2 * axis) * L + c] = above[axis];
    }
    f.a[i] = total;
}

// Probe p's pressure before the step (fdtd.hpp:3525-3533): its cells' weighted sum in double, in
// the layout's order.
template <typename T>
__global__ void __launch_bounds__(kBlock) probe_kernel(const Tables g, const Fields<T> f) {
    const uint32_t p = blockIdx.x * kBlock + threadIdx.x;
    if (p >= g.probes) return;
    double value = 0.0;
    for (uint32_t k = g.probe_start[p], e = g.probe_start[p + 1]; k < e; ++k) {
        value += g.probe_weights[k] * (double)f.b[g.probe_cells[k]];
    }
    f.out[(uint64_t)p * f.out_stride] = value;
}

}  // namespace fdtd

// B200 (sm_100a) stepper for acoustic-spaces' low-frequency wave solver: the C ABI of
// include/fdtd_b200.h over hand-written CUDA kernels.
//
// One time step of WaveSolver::run (cpp/include/acoustic_spaces/fdtd.hpp:786-904 of
// naelolaiz/acoustic-spaces) reads the current pressure b and the branch velocities wb, and writes
// the next pressure over the previous one in a, the branch velocities over wa, and the matched
// layer's state in place. Every cell's new value depends only on b, wb, its own a, wa and layer
// state, so the four kinds of work of a step (probe records, interior air, special rows, matched
// layer cells) write disjoint memory and run as one launch: its blocks are split by kind.
// Consecutive steps are ordered by the launches on the handle's stream.
//
// Arithmetic: the library is built with --fmad=false and -ftz=true. Every expression keeps the
// reference's operands in the reference's order, so with T = float each operation rounds as the
// reference's -ffp-contract=off build does, subnormal results flushed to zero as its MXCSR flush
// does (fdtd.hpp:316-336): the probes' series equal the reference's bit for bit. T = double steps
// the same layout with every stored coefficient promoted.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "fdtd_b200.h"

namespace {

// ---------------------------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------------------------

thread_local std::string g_error;

int set_global(int status, const std::string &message) {
    g_error = message;
    return status;
}

// The directions of a cell's links (fdtd.hpp:924-927): six axial, then twelve edge directions.
constexpr int kSteps[18][3] = {
    {-1, 0, 0},  {1, 0, 0},  {0, -1, 0}, {0, 1, 0},   {0, 0, -1}, {0, 0, 1},
    {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 1, 0},   {-1, 0, -1}, {1, 0, -1},
    {-1, 0, 1},  {1, 0, 1},  {0, -1, -1}, {0, 1, -1}, {0, -1, 1},  {0, 1, 1}};

constexpr int kBlock = 256;   // threads per block of every kind
constexpr int kTileX = 32;    // bulk tile: 32 cells along x (one warp) ...
constexpr int kTileY = 8;     // ... by 8 rows along y, marching along z
constexpr int kSolid = 0, kInterior = 1, kSpecial = 2, kLayer = 3;

// ---------------------------------------------------------------------------------------------
// Device-side description of a grid (passed by value to every launch)
// ---------------------------------------------------------------------------------------------

struct Grid {
    uint32_t nx, ny, nz, sy, sz;
    // The bulk sweep's box: the bounding box of the interior cells, half open, and its tiling.
    uint32_t x0, y0, z0, x1, y1, z1;
    uint32_t tiles_x, tiles_y, z_chunk;
    uint32_t bulk_blocks, special_blocks, layer_blocks, probe_blocks;
    float axial, diagonal, centre, total;
    const uint8_t *types;
    const float *scale;
    // Special rows (fdtd.hpp:860-881), as structure of arrays.
    uint32_t specials;
    const uint32_t *special, *link_start, *state_start;
    const uint8_t *link_direction;
    const float *link_weight, *coef_a, *coef_b, *coef_inv, *source;
    const float *state_weight, *state_now, *state_before, *state_gain;
    int32_t offset[18];
    // Matched layer (fdtd.hpp:2242-2264): cells, per-axis coefficient tables (centre keep, face
    // keep, centre push, face push per axis), and with a speed field each cell's scale.
    uint32_t layers;
    const uint32_t *layer_cells;
    const float *layer_scale;
    const float *keep_centre[3], *keep_face[3], *push_centre[3], *push_face[3];
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

// ---------------------------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------------------------

// Interior air (fdtd.hpp:242-288): one warp-wide row of 32 cells per thread row, eight rows a
// block, marching along z through a chunk of planes with the z neighbours kept in registers.
// The reference's sums in its order: x-1, x+1, y-1, y+1, z-1, z+1, then the twelve edges.
template <typename T, bool WIDE, bool SCALED>
__device__ __forceinline__ void bulk_tile(const Grid &g, const Fields<T> &f, uint32_t tile) {
    const uint32_t bx = tile % g.tiles_x;
    const uint32_t rest = tile / g.tiles_x;
    const uint32_t by = rest % g.tiles_y;
    const uint32_t bz = rest / g.tiles_y;
    const uint32_t x = g.x0 + bx * kTileX + (threadIdx.x % kTileX);
    const uint32_t y = g.y0 + by * kTileY + (threadIdx.x / kTileX);
    uint32_t z = g.z0 + bz * g.z_chunk;
    if (x >= g.x1 || y >= g.y1 || z >= g.z1) return;
    const uint32_t z_end = min(z + g.z_chunk, g.z1);
    const uint32_t sy = g.sy, sz = g.sz;
    const T *__restrict__ b = f.b;
    T *__restrict__ a = f.a;
    uint32_t i = x + y * sy + z * sz;
    T below = b[i - sz], here = b[i];
    const T axial = (T)g.axial, centre = (T)g.centre, diagonal = (T)g.diagonal, total = (T)g.total;
    for (; z < z_end; ++z, i += sz) {
        const T above = b[i + sz];
        if (g.types[i] == kInterior) {
            const T sum = b[i - 1] + b[i + 1] + b[i - sy] + b[i + sy] + below + above;
            T next;
            if (WIDE) {
                const T edges = b[i - 1 - sy] + b[i + 1 - sy] + b[i - 1 + sy] + b[i + 1 + sy] +
                                b[i - 1 - sz] + b[i + 1 - sz] + b[i - 1 + sz] + b[i + 1 + sz] +
                                b[i - sy - sz] + b[i + sy - sz] + b[i - sy + sz] + b[i + sy + sz];
                if (SCALED) {
                    const T s = (T)g.scale[i];
                    next = ((T)2 - total * s) * here + (s * axial) * sum + (s * diagonal) * edges - a[i];
                } else {
                    next = centre * here + axial * sum + diagonal * edges - a[i];
                }
            } else {
                if (SCALED) {
                    const T s = (T)g.scale[i];
                    next = ((T)2 - total * s) * here + (s * axial) * sum - a[i];
                } else {
                    next = centre * here + axial * sum - a[i];
                }
            }
            a[i] = next;
        }
        below = here;
        here = above;
    }
}

// Special row k (fdtd.hpp:860-881): its links, its branch states' flow, the update, then the
// branch velocities. A state's term now * wb - before * wa is worked out again for the
// velocities' update rather than kept: wa has not changed in between, so it is the same value.
template <typename T>
__device__ __forceinline__ void special_row(const Grid &g, const Fields<T> &f, uint32_t k) {
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

// Matched-layer cell c (fdtd.hpp:2242-2264): per axis its two face velocities, then its pressure
// part; the cell's pressure is the parts' sum.
template <typename T, bool SCALED>
__device__ __forceinline__ void layer_cell(const Grid &g, const Fields<T> &f, uint32_t c) {
    if (c >= g.layers) return;
    const uint32_t L = g.layers;
    const uint32_t i = g.layer_cells[c];
    const uint32_t at[3] = {i % g.nx, (i / g.nx) % g.ny, i / g.sz};
    const uint32_t strides[3] = {1u, g.sy, g.sz};
    const T *__restrict__ b = f.b;
    T *st = f.layer_state;
    const T here = b[i];
    T total = 0;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const uint32_t stride = strides[axis], x = at[axis];
        T below = st[(3 + 2 * axis) * L + c], above = st[(4 + 2 * axis) * L + c];
        below = (T)g.keep_face[axis][x] * below - (T)g.push_face[axis][x] * (here - b[i - stride]);
        above = (T)g.keep_face[axis][x + 1] * above - (T)g.push_face[axis][x + 1] * (b[i + stride] - here);
        st[(3 + 2 * axis) * L + c] = below;
        st[(4 + 2 * axis) * L + c] = above;
        T part = st[axis * L + c];
        if (SCALED) {
            part = (T)g.keep_centre[axis][x] * part -
                   ((T)g.push_centre[axis][x] * (T)g.layer_scale[c]) * (above - below);
        } else {
            part = (T)g.keep_centre[axis][x] * part - (T)g.push_centre[axis][x] * (above - below);
        }
        st[axis * L + c] = part;
        total += part;
    }
    f.a[i] = total;
}

// Probe p's pressure before the step (fdtd.hpp:3525-3533): its cells' weighted sum in double, in
// the layout's order.
template <typename T>
__device__ __forceinline__ void probe_record(const Grid &g, const Fields<T> &f, uint32_t p) {
    if (p >= g.probes) return;
    double value = 0.0;
    for (uint32_t k = g.probe_start[p], e = g.probe_start[p + 1]; k < e; ++k) {
        value += g.probe_weights[k] * (double)f.b[g.probe_cells[k]];
    }
    f.out[(uint64_t)p * f.out_stride] = value;
}

template <typename T, bool WIDE, bool SCALED>
__global__ void __launch_bounds__(kBlock) step_kernel(const Grid g, const Fields<T> f) {
    uint32_t block = blockIdx.x;
    if (block < g.bulk_blocks) {
        bulk_tile<T, WIDE, SCALED>(g, f, block);
        return;
    }
    block -= g.bulk_blocks;
    if (block < g.special_blocks) {
        special_row<T>(g, f, block * kBlock + threadIdx.x);
        return;
    }
    block -= g.special_blocks;
    if (block < g.layer_blocks) {
        layer_cell<T, SCALED>(g, f, block * kBlock + threadIdx.x);
        return;
    }
    block -= g.layer_blocks;
    probe_record<T>(g, f, block * kBlock + threadIdx.x);
}

// ---------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------

struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct fdtd_solver {
    int device = 0;
    int precision = FDTD_FP32;
    bool wide = false, scaled = false;
    cudaStream_t stream = nullptr;
    std::string error;
    Grid grid{};
    uint64_t nx = 0, ny = 0, nz = 0, n = 0;
    uint64_t air = 0, interior = 0, links = 0, states = 0, layers = 0, probes = 0, specials = 0;
    uint64_t steps_done = 0;
    std::vector<void *> allocations;  // every device allocation the handle owns
    uint64_t device_bytes = 0;
    // The state: u[1] is the current pressure between runs, u[0] the one a step before; the same
    // for the branch velocities w.
    void *u[2] = {nullptr, nullptr};
    void *w[2] = {nullptr, nullptr};
    void *layer_state = nullptr;
    // Staging for fdtd_run's host buffers, grown on demand.
    float *stage_signal = nullptr;
    double *stage_out = nullptr;
    uint64_t stage_steps = 0;
};

namespace {

int fail(fdtd_solver *s, int status, const std::string &message) {
    if (s) s->error = message;
    return status;
}

int cuda_fail(fdtd_solver *s, cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (s) s->error = m;
    g_error = m;
    return e == cudaErrorMemoryAllocation ? FDTD_ENOMEM : FDTD_ECUDA;
}

#define CUDA_TRY(s, call)                                  \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(s, e_, #call); \
    } while (0)

template <typename V>
int upload(fdtd_solver *s, const V *host, size_t count, const V **out) {
    *out = nullptr;
    if (count == 0) return FDTD_OK;
    void *p = nullptr;
    CUDA_TRY(s, cudaMalloc(&p, count * sizeof(V)));
    s->allocations.push_back(p);
    s->device_bytes += count * sizeof(V);
    CUDA_TRY(s, cudaMemcpy(p, host, count * sizeof(V), cudaMemcpyHostToDevice));
    *out = static_cast<const V *>(p);
    return FDTD_OK;
}

int zeros(fdtd_solver *s, size_t bytes, void **out) {
    *out = nullptr;
    void *p = nullptr;
    CUDA_TRY(s, cudaMalloc(&p, bytes ? bytes : 16));
    s->allocations.push_back(p);
    s->device_bytes += bytes;
    CUDA_TRY(s, cudaMemset(p, 0, bytes ? bytes : 16));
    *out = p;
    return FDTD_OK;
}

// Host-side checks of every index the kernels will follow, so that no launch reads or writes
// outside its buffers whatever layout it is given. Messages follow the reference's wording where
// it refuses the same thing.
int validate(const fdtd_layout *L, std::string &why) {
    auto refuse = [&](const std::string &m) {
        why = m;
        return FDTD_EINVAL;
    };
    if (!L) return refuse("no layout");
    if (L->stencil != 7 && L->stencil != 19) return refuse("the stencil has 7 or 19 points");
    if (L->flow_count) return refuse("the GPU steps still air only: moving air stays on the CPU");
    if (L->nx < 3 || L->ny < 3 || L->nz < 3) return refuse("the grid is too small");
    const uint64_t n = L->nx * L->ny * L->nz;
    if (L->nx > (1ull << 31) || L->ny > (1ull << 31) || L->nz > (1ull << 31) || n >= (1ull << 32) ||
        n / L->nx / L->ny != L->nz)
        return refuse("the wave grid is too large for the GPU's 32-bit indices");
    if (L->weight_count < (L->stencil == 19 ? 18u : 6u) || !L->weights)
        return refuse("the layout's weights do not match its stencil");
    if (!L->types) return refuse("the layout has no cell types");
    if (L->scaled && !L->scale) return refuse("a scaled layout needs each cell's scale");
    const uint64_t nx = L->nx, ny = L->ny, nz = L->nz, sz = nx * ny;
    auto inner = [&](uint64_t i) {
        const uint64_t x = i % nx, y = (i / nx) % ny, z = i / sz;
        return x >= 1 && y >= 1 && z >= 1 && x + 1 < nx && y + 1 < ny && z + 1 < nz;
    };
    for (uint64_t i = 0; i < n; ++i) {
        const uint8_t t = L->types[i];
        if (t > kLayer) return refuse("a cell's type is not solid, interior, special or layer");
        if (t == kInterior && !inner(i)) return refuse("an interior cell lies on the grid's edge");
    }
    if (L->special_count >= (1ull << 32) || L->link_count >= (1ull << 32) || L->state_count >= (1ull << 32) ||
        L->layer_count >= (1ull << 32) || L->probe_count >= (1ull << 32))
        return refuse("the layout's tables are too large for the GPU's 32-bit indices");
    if (L->special_count && (!L->special || !L->coef_a || !L->coef_b || !L->coef_inv || !L->source))
        return refuse("the layout's special cells miss their coefficients");
    if (!L->link_start || !L->state_start) return refuse("the layout has no link_start or state_start");
    if (L->link_start[0] != 0 || L->link_start[L->special_count] != L->link_count)
        return refuse("link_start does not span the links");
    if (L->state_start[0] != 0 || L->state_start[L->special_count] != L->state_count)
        return refuse("state_start does not span the branch states");
    if (L->link_count && (!L->link_direction || !L->link_weight)) return refuse("the links miss their arrays");
    for (uint64_t k = 0; k < L->special_count; ++k) {
        if (L->link_start[k + 1] < L->link_start[k] || L->state_start[k + 1] < L->state_start[k])
            return refuse("link_start and state_start must not decrease");
        const int64_t i = L->special[k];
        if (i < 0 || (uint64_t)i >= n) return refuse("a special cell lies outside the grid");
        if (L->types[i] != kSpecial) return refuse("a special cell's type is not special");
        const int64_t x = i % (int64_t)nx, y = (i / (int64_t)nx) % (int64_t)ny, z = i / (int64_t)sz;
        for (uint64_t l = L->link_start[k]; l < L->link_start[k + 1]; ++l) {
            const uint8_t d = L->link_direction[l];
            if (d >= 18) return refuse("a link's direction is not one of the 18");
            const int64_t xx = x + kSteps[d][0], yy = y + kSteps[d][1], zz = z + kSteps[d][2];
            if (xx < 0 || yy < 0 || zz < 0 || xx >= (int64_t)nx || yy >= (int64_t)ny || zz >= (int64_t)nz)
                return refuse("a special cell links outside the grid");
        }
    }
    if (L->state_count && (!L->state_branch || !L->state_weight)) return refuse("the branch states miss their arrays");
    if (L->branch_count && (!L->branch_now || !L->branch_before || !L->branch_gain))
        return refuse("the branches miss their coefficients");
    for (uint64_t j = 0; j < L->state_count; ++j) {
        if (L->state_branch[j] < 0 || (uint64_t)L->state_branch[j] >= L->branch_count)
            return refuse("a branch state has no branch");
    }
    if (L->layer_count) {
        if (!L->layer_cells) return refuse("the matched layer has no cells");
        for (int k = 0; k < 6; ++k)
            if (!L->keep[k] || !L->push[k]) return refuse("the matched layer misses its coefficients");
        if (L->scaled && !L->layer_scale) return refuse("a scaled layout needs each layer cell's scale");
        for (uint64_t c = 0; c < L->layer_count; ++c) {
            const int64_t i = L->layer_cells[c];
            if (i < 0 || (uint64_t)i >= n || !inner((uint64_t)i))
                return refuse("a matched-layer cell lies outside the grid or on its edge");
            if (L->types[i] != kLayer) return refuse("a matched-layer cell's type is not layer");
        }
    }
    {
        // Each special and matched-layer cell is listed once: every cell's update is one
        // thread's, so that no two write the same cell.
        std::vector<uint8_t> seen(n, 0);
        for (uint64_t k = 0; k < L->special_count; ++k) {
            if (seen[L->special[k]]++) return refuse("a special cell is listed twice");
        }
        for (uint64_t c = 0; c < L->layer_count; ++c) {
            if (seen[L->layer_cells[c]]++) return refuse("a matched-layer cell is listed twice");
        }
    }
    if (!L->probe_start || L->probe_start[0] != 0) return refuse("probe_start does not start at 0");
    const uint64_t pc = L->probe_start[L->probe_count];
    if (pc && (!L->probe_cells || !L->probe_weights)) return refuse("the probes miss their cells");
    for (uint64_t p = 0; p < L->probe_count; ++p)
        if (L->probe_start[p + 1] < L->probe_start[p]) return refuse("probe_start must not decrease");
    if (pc >= (1ull << 32)) return refuse("the probes' tables are too large");
    for (uint64_t k = 0; k < pc; ++k)
        if (L->probe_cells[k] >= n) return refuse("a probe reads a cell outside the grid");
    return FDTD_OK;
}

template <typename T>
Fields<T> fields_for(const fdtd_solver *s, bool flip) {
    // flip = false: b is u[1] (current), a is u[0]; flip = true after an odd number of steps.
    Fields<T> f{};
    const int cur = flip ? 0 : 1, prev = flip ? 1 : 0;
    f.b = static_cast<const T *>(s->u[cur]);
    f.a = static_cast<T *>(s->u[prev]);
    f.wb = static_cast<const T *>(s->w[cur]);
    f.wa = static_cast<T *>(s->w[prev]);
    f.layer_state = static_cast<T *>(s->layer_state);
    return f;
}

template <typename T, bool WIDE, bool SCALED>
int launch_steps(fdtd_solver *s, const float *d_signal, uint64_t steps, double *d_out, uint64_t stride) {
    const Grid &g = s->grid;
    const uint32_t blocks = g.bulk_blocks + g.special_blocks + g.layer_blocks + g.probe_blocks;
    if (blocks == 0) return FDTD_OK;
    for (uint64_t k = 0; k < steps; ++k) {
        Fields<T> f = fields_for<T>(s, (k & 1) != 0);
        f.signal = d_signal + k;
        f.out = d_out + k;
        f.out_stride = stride;
        step_kernel<T, WIDE, SCALED><<<blocks, kBlock, 0, s->stream>>>(g, f);
    }
    CUDA_TRY(s, cudaGetLastError());
    return FDTD_OK;
}

int dispatch(fdtd_solver *s, const float *d_signal, uint64_t steps, double *d_out, uint64_t stride) {
    const bool fp64 = s->precision == FDTD_FP64;
#define CASE(T, W, S)                                                    \
    if (s->wide == W && s->scaled == S) return launch_steps<T, W, S>(s, d_signal, steps, d_out, stride);
    if (fp64) {
        CASE(double, false, false) CASE(double, false, true) CASE(double, true, false) CASE(double, true, true)
    } else {
        CASE(float, false, false) CASE(float, false, true) CASE(float, true, false) CASE(float, true, true)
    }
#undef CASE
    return fail(s, FDTD_EINVAL, "no kernel for this layout");
}

// After `steps` steps the parity swap of fdtd.hpp:900-903: u[1] stays the current level.
void settle(fdtd_solver *s, uint64_t steps) {
    if (steps % 2 == 1) {
        std::swap(s->u[0], s->u[1]);
        std::swap(s->w[0], s->w[1]);
    }
    s->steps_done += steps;
}

int build(fdtd_solver *s, const fdtd_layout *L) {
    const uint64_t nx = L->nx, ny = L->ny, nz = L->nz, n = nx * ny * nz;
    s->nx = nx, s->ny = ny, s->nz = nz, s->n = n;
    s->wide = L->stencil == 19;
    s->scaled = L->scaled != 0;
    Grid &g = s->grid;
    g.nx = (uint32_t)nx, g.ny = (uint32_t)ny, g.nz = (uint32_t)nz;
    g.sy = (uint32_t)nx, g.sz = (uint32_t)(nx * ny);
    g.axial = L->weights[0];
    g.diagonal = s->wide ? L->weights[6] : 0.0f;
    g.centre = L->centre;
    g.total = L->total;
    for (int k = 0; k < 18; ++k)
        g.offset[k] = (int32_t)(kSteps[k][0] + kSteps[k][1] * (int64_t)nx + kSteps[k][2] * (int64_t)(nx * ny));

    // The interior cells' bounding box and the air count.
    uint64_t x0 = nx, y0 = ny, z0 = nz, x1 = 0, y1 = 0, z1 = 0, interior = 0, air = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const uint8_t t = L->types[i];
        if (t != kSolid) ++air;
        if (t != kInterior) continue;
        ++interior;
        const uint64_t x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
        x0 = std::min(x0, x), x1 = std::max(x1, x + 1);
        y0 = std::min(y0, y), y1 = std::max(y1, y + 1);
        z0 = std::min(z0, z), z1 = std::max(z1, z + 1);
    }
    s->interior = interior, s->air = air;
    if (interior == 0) x0 = y0 = z0 = x1 = y1 = z1 = 1;
    g.x0 = (uint32_t)x0, g.y0 = (uint32_t)y0, g.z0 = (uint32_t)z0;
    g.x1 = (uint32_t)x1, g.y1 = (uint32_t)y1, g.z1 = (uint32_t)z1;
    g.tiles_x = (uint32_t)((x1 - x0 + kTileX - 1) / kTileX);
    g.tiles_y = (uint32_t)((y1 - y0 + kTileY - 1) / kTileY);
    // Planes per block: enough blocks for every SM several times over, long enough marches.
    const uint64_t columns = (uint64_t)g.tiles_x * g.tiles_y;
    const uint64_t depth = z1 - z0;
    uint64_t chunk = depth;
    while (chunk > 8 && columns * ((depth + chunk - 1) / chunk) < 148ull * 16) chunk = (chunk + 1) / 2;
    g.z_chunk = (uint32_t)std::max<uint64_t>(chunk, 1);
    const uint64_t tiles_z = interior ? (depth + g.z_chunk - 1) / g.z_chunk : 0;
    const uint64_t bulk = interior ? columns * tiles_z : 0;
    if (bulk >= (1ull << 31)) return fail(s, FDTD_EINVAL, "the wave grid is too large for one launch");
    g.bulk_blocks = (uint32_t)bulk;

    int rc;
    const uint8_t *types;
    if ((rc = upload(s, L->types, n, &types))) return rc;
    g.types = types;
    if (s->scaled) {
        const float *scale;
        if ((rc = upload(s, L->scale, n, &scale))) return rc;
        g.scale = scale;
    }

    // Special rows with 32-bit indices.
    const uint64_t K = L->special_count;
    s->specials = K, s->links = L->link_count, s->states = L->state_count;
    g.specials = (uint32_t)K;
    g.special_blocks = (uint32_t)((K + kBlock - 1) / kBlock);
    {
        std::vector<uint32_t> special(K), link_start(K + 1), state_start(K + 1);
        for (uint64_t k = 0; k < K; ++k) special[k] = (uint32_t)L->special[k];
        for (uint64_t k = 0; k <= K; ++k) {
            link_start[k] = (uint32_t)L->link_start[k];
            state_start[k] = (uint32_t)L->state_start[k];
        }
        const uint32_t *p;
        if ((rc = upload(s, special.data(), K, &p))) return rc;
        g.special = p;
        if ((rc = upload(s, link_start.data(), K + 1, &p))) return rc;
        g.link_start = p;
        if ((rc = upload(s, state_start.data(), K + 1, &p))) return rc;
        g.state_start = p;
    }
    const float *fp;
    const uint8_t *u8;
    if ((rc = upload(s, L->link_direction, L->link_count, &u8))) return rc;
    g.link_direction = u8;
    if ((rc = upload(s, L->link_weight, L->link_count, &fp))) return rc;
    g.link_weight = fp;
    if ((rc = upload(s, L->coef_a, K, &fp))) return rc;
    g.coef_a = fp;
    if ((rc = upload(s, L->coef_b, K, &fp))) return rc;
    g.coef_b = fp;
    if ((rc = upload(s, L->coef_inv, K, &fp))) return rc;
    g.coef_inv = fp;
    if ((rc = upload(s, L->source, K, &fp))) return rc;
    g.source = fp;
    {
        // Each state's branch coefficients gathered per state, as run() gathers them
        // (fdtd.hpp:797-805).
        const uint64_t S = L->state_count;
        std::vector<float> now(S), before(S), gain(S);
        for (uint64_t j = 0; j < S; ++j) {
            const int32_t br = L->state_branch[j];
            now[j] = L->branch_now[br], before[j] = L->branch_before[br], gain[j] = L->branch_gain[br];
        }
        if ((rc = upload(s, L->state_weight, S, &fp))) return rc;
        g.state_weight = fp;
        if ((rc = upload(s, now.data(), S, &fp))) return rc;
        g.state_now = fp;
        if ((rc = upload(s, before.data(), S, &fp))) return rc;
        g.state_before = fp;
        if ((rc = upload(s, gain.data(), S, &fp))) return rc;
        g.state_gain = fp;
    }

    // Matched layer.
    const uint64_t Lc = L->layer_count;
    s->layers = Lc;
    g.layers = (uint32_t)Lc;
    g.layer_blocks = (uint32_t)((Lc + kBlock - 1) / kBlock);
    if (Lc) {
        std::vector<uint32_t> cells(Lc);
        for (uint64_t c = 0; c < Lc; ++c) cells[c] = (uint32_t)L->layer_cells[c];
        const uint32_t *p;
        if ((rc = upload(s, cells.data(), Lc, &p))) return rc;
        g.layer_cells = p;
        const uint64_t len[3] = {nx + 1, ny + 1, nz + 1};
        for (int axis = 0; axis < 3; ++axis) {
            if ((rc = upload(s, L->keep[2 * axis], len[axis], &fp))) return rc;
            g.keep_centre[axis] = fp;
            if ((rc = upload(s, L->keep[2 * axis + 1], len[axis], &fp))) return rc;
            g.keep_face[axis] = fp;
            if ((rc = upload(s, L->push[2 * axis], len[axis], &fp))) return rc;
            g.push_centre[axis] = fp;
            if ((rc = upload(s, L->push[2 * axis + 1], len[axis], &fp))) return rc;
            g.push_face[axis] = fp;
        }
        if (s->scaled) {
            if ((rc = upload(s, L->layer_scale, Lc, &fp))) return rc;
            g.layer_scale = fp;
        }
    }

    // Probes.
    const uint64_t P = L->probe_count, pc = L->probe_start[P];
    s->probes = P;
    g.probes = (uint32_t)P;
    g.probe_blocks = (uint32_t)((P + kBlock - 1) / kBlock);
    {
        std::vector<uint32_t> start(P + 1), cells(pc);
        for (uint64_t p = 0; p <= P; ++p) start[p] = (uint32_t)L->probe_start[p];
        for (uint64_t k = 0; k < pc; ++k) cells[k] = (uint32_t)L->probe_cells[k];
        const uint32_t *p32;
        if ((rc = upload(s, start.data(), P + 1, &p32))) return rc;
        g.probe_start = p32;
        if ((rc = upload(s, cells.data(), pc, &p32))) return rc;
        g.probe_cells = p32;
        const double *pd;
        if ((rc = upload(s, L->probe_weights, pc, &pd))) return rc;
        g.probe_weights = pd;
    }

    // The state, at rest.
    const size_t e = s->precision == FDTD_FP64 ? 8 : 4;
    for (int k = 0; k < 2; ++k) {
        if ((rc = zeros(s, e * n, &s->u[k]))) return rc;
        if ((rc = zeros(s, e * L->state_count, &s->w[k]))) return rc;
    }
    if ((rc = zeros(s, e * 9 * Lc, &s->layer_state))) return rc;
    return FDTD_OK;
}

void release(fdtd_solver *s) {
    if (!s) return;
    int current = 0;
    cudaGetDevice(&current);
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (void *p : s->allocations) cudaFree(p);
    if (s->stage_signal) cudaFreeHost(s->stage_signal);
    if (s->stage_out) cudaFreeHost(s->stage_out);
    if (s->stream) cudaStreamDestroy(s->stream);
    cudaSetDevice(current);
}

struct DeviceGuard {
    int previous = -1;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&previous) != cudaSuccess) previous = -1;
        cudaSetDevice(device);
    }
    ~DeviceGuard() {
        if (previous >= 0) cudaSetDevice(previous);
    }
};

}  // namespace

// ---------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------

extern "C" {

int fdtd_abi_version(void) { return FDTD_B200_ABI_VERSION; }

const char *fdtd_global_error(void) { return g_error.c_str(); }

const char *fdtd_last_error(const fdtd_solver *s) { return s ? s->error.c_str() : g_error.c_str(); }

int fdtd_device_count(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int usable = 0;
    for (int d = 0; d < count; ++d) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, d) == cudaSuccess && prop.major == 10) ++usable;
    }
    return usable;
}

int fdtd_device_name(int device, char *buf, size_t size) {
    if (!buf || size == 0) return set_global(FDTD_EINVAL, "no buffer for the name");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return set_global(FDTD_ENODEV, "no such CUDA device");
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return set_global(FDTD_ENODEV, "no such CUDA device");
    std::snprintf(buf, size, "%s (CUDA sm_%d%d, %.0f GiB)", prop.name, prop.major, prop.minor,
                  (double)prop.totalGlobalMem / (1024.0 * 1024.0 * 1024.0));
    return FDTD_OK;
}

int fdtd_create(const fdtd_layout *layout, int precision, int device, fdtd_solver **out) {
    if (!out) return set_global(FDTD_EINVAL, "no place for the handle");
    *out = nullptr;
    if (precision != FDTD_FP32 && precision != FDTD_FP64)
        return set_global(FDTD_EINVAL, "precision is FDTD_FP32 or FDTD_FP64");
    std::string why;
    if (validate(layout, why) != FDTD_OK) return set_global(FDTD_EINVAL, why);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0 || device < 0 || device >= count) {
        cudaGetLastError();
        return set_global(FDTD_ENODEV, "no CUDA device to step the wave grid on");
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10)
        return set_global(FDTD_ENODEV, "the wave stepper is built for sm_100a (B200) only");
    DeviceGuard guard(device);
    fdtd_solver *s = new (std::nothrow) fdtd_solver();
    if (!s) return set_global(FDTD_ENOMEM, "out of host memory");
    s->device = device;
    s->precision = precision;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        const int rc = cuda_fail(nullptr, e, "cudaStreamCreate");
        delete s;
        return rc;
    }
    const int rc = build(s, layout);
    if (rc != FDTD_OK) {
        g_error = s->error;
        release(s);
        delete s;
        return rc;
    }
    *out = s;
    return FDTD_OK;
}

int fdtd_run_device(fdtd_solver *s, const float *d_signal, uint64_t steps, double *d_out, uint64_t out_stride) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (steps == 0) return FDTD_OK;
    if (!d_signal || (s->probes && !d_out)) return fail(s, FDTD_EINVAL, "no signal or output buffer");
    if (out_stride < steps && s->probes) return fail(s, FDTD_EINVAL, "the output's stride is shorter than the run");
    DeviceGuard guard(s->device);
    const int rc = dispatch(s, d_signal, steps, d_out, out_stride);
    if (rc != FDTD_OK) return rc;
    settle(s, steps);
    return FDTD_OK;
}

int fdtd_synchronize(fdtd_solver *s) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    DeviceGuard guard(s->device);
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return FDTD_OK;
}

int fdtd_run(fdtd_solver *s, const float *signal, uint64_t steps, double *out) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (steps == 0) return FDTD_OK;
    if (!signal || (s->probes && !out)) return fail(s, FDTD_EINVAL, "no signal or output buffer");
    DeviceGuard guard(s->device);
    // Device staging in pieces of bounded size (the probes' records of a piece).
    const uint64_t piece = std::min<uint64_t>(steps, std::max<uint64_t>(1024, (64ull << 20) / (8 * std::max<uint64_t>(1, s->probes))));
    if (s->stage_steps < piece) {
        if (s->stage_signal) cudaFreeHost(s->stage_signal);
        if (s->stage_out) cudaFreeHost(s->stage_out);
        s->stage_signal = nullptr, s->stage_out = nullptr, s->stage_steps = 0;
        CUDA_TRY(s, cudaMallocHost((void **)&s->stage_signal, piece * sizeof(float)));
        CUDA_TRY(s, cudaMallocHost((void **)&s->stage_out, piece * std::max<uint64_t>(1, s->probes) * sizeof(double)));
        s->stage_steps = piece;
    }
    // Device copies: the signal and the records of one piece.
    float *d_signal = nullptr;
    double *d_out = nullptr;
    CUDA_TRY(s, cudaMallocAsync((void **)&d_signal, piece * sizeof(float), s->stream));
    cudaError_t e = cudaMallocAsync((void **)&d_out, piece * std::max<uint64_t>(1, s->probes) * sizeof(double), s->stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(d_signal, s->stream);
        return cuda_fail(s, e, "cudaMallocAsync");
    }
    int rc = FDTD_OK;
    for (uint64_t begin = 0; begin < steps && rc == FDTD_OK; begin += piece) {
        const uint64_t count = std::min(piece, steps - begin);
        std::memcpy(s->stage_signal, signal + begin, count * sizeof(float));
        e = cudaMemcpyAsync(d_signal, s->stage_signal, count * sizeof(float), cudaMemcpyHostToDevice, s->stream);
        if (e != cudaSuccess) { rc = cuda_fail(s, e, "cudaMemcpyAsync"); break; }
        rc = dispatch(s, d_signal, count, d_out, count);
        if (rc != FDTD_OK) break;
        settle(s, count);
        if (s->probes) {
            e = cudaMemcpyAsync(s->stage_out, d_out, count * s->probes * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
            if (e != cudaSuccess) { rc = cuda_fail(s, e, "cudaMemcpyAsync"); break; }
        }
        e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) { rc = cuda_fail(s, e, "cudaStreamSynchronize"); break; }
        for (uint64_t p = 0; p < s->probes; ++p)
            std::memcpy(out + p * steps + begin, s->stage_out + p * count, count * sizeof(double));
    }
    cudaFreeAsync(d_signal, s->stream);
    cudaFreeAsync(d_out, s->stream);
    if (rc != FDTD_OK) return rc;
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    for (uint64_t k = 0; k < s->probes * steps; ++k) {
        if (!std::isfinite(out[k])) return fail(s, FDTD_ENONFINITE, "the wave solver's run did not stay finite");
    }
    return FDTD_OK;
}

int fdtd_reset(fdtd_solver *s) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    DeviceGuard guard(s->device);
    const size_t e = s->precision == FDTD_FP64 ? 8 : 4;
    for (int k = 0; k < 2; ++k) {
        CUDA_TRY(s, cudaMemsetAsync(s->u[k], 0, e * s->n, s->stream));
        if (s->states) CUDA_TRY(s, cudaMemsetAsync(s->w[k], 0, e * s->states, s->stream));
    }
    if (s->layers) CUDA_TRY(s, cudaMemsetAsync(s->layer_state, 0, e * 9 * s->layers, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    s->steps_done = 0;
    return FDTD_OK;
}

int fdtd_destroy(fdtd_solver *s) {
    if (!s) return FDTD_OK;
    release(s);
    delete s;
    return FDTD_OK;
}

int fdtd_get_info(const fdtd_solver *s, fdtd_info *info) {
    if (!s || !info) return set_global(FDTD_EINVAL, "no solver or info");
    info->cells = s->n;
    info->air_cells = s->air;
    info->interior_cells = s->interior;
    info->special_cells = s->specials;
    info->links = s->links;
    info->branch_states = s->states;
    info->layer_cells = s->layers;
    info->probes = s->probes;
    info->steps_done = s->steps_done;
    info->device_bytes = s->device_bytes;
    info->precision = s->precision;
    info->device = s->device;
    return FDTD_OK;
}

int fdtd_read_state(const fdtd_solver *cs, void *current, void *previous, void *branch_current,
                    void *branch_previous, void *layer_state) {
    fdtd_solver *s = const_cast<fdtd_solver *>(cs);
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    DeviceGuard guard(s->device);
    const size_t e = s->precision == FDTD_FP64 ? 8 : 4;
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (current) CUDA_TRY(s, cudaMemcpy(current, s->u[1], e * s->n, cudaMemcpyDeviceToHost));
    if (previous) CUDA_TRY(s, cudaMemcpy(previous, s->u[0], e * s->n, cudaMemcpyDeviceToHost));
    if (branch_current && s->states) CUDA_TRY(s, cudaMemcpy(branch_current, s->w[1], e * s->states, cudaMemcpyDeviceToHost));
    if (branch_previous && s->states) CUDA_TRY(s, cudaMemcpy(branch_previous, s->w[0], e * s->states, cudaMemcpyDeviceToHost));
    if (layer_state && s->layers) {
        // The device keeps the layer's state as 9 arrays; the reference keeps 9 values per cell.
        std::vector<char> soa(e * 9 * s->layers);
        CUDA_TRY(s, cudaMemcpy(soa.data(), s->layer_state, soa.size(), cudaMemcpyDeviceToHost));
        char *dst = static_cast<char *>(layer_state);
        for (uint64_t c = 0; c < s->layers; ++c)
            for (int k = 0; k < 9; ++k)
                std::memcpy(dst + e * (9 * c + k), soa.data() + e * (k * s->layers + c), e);
    }
    return FDTD_OK;
}

}  // extern "C"

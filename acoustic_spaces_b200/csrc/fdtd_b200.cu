// B200 (sm_100a) stepper for acoustic-spaces' low-frequency wave solver: the C ABI of
// include/fdtd_b200.h over the kernels of fdtd_kernels.cuh.
//
// fdtd_create validates a layout (WaveSolver::layout(), cpp/include/acoustic_spaces/
// fdtd.hpp:727-782 of naelolaiz/acoustic-spaces) on the host, copies it to the device in a pitched
// layout, and builds the TMA tensor maps of the bulk sweep. A time step (fdtd.hpp:838-886) is four
// launches: the interior air (TMA-pipelined, bulk_kernel) on the handle's stream, beside it the
// matched layer on a stream of its own and the special rows and probe records on a side stream; the
// levels swap between steps by the launches' pointers.

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "fdtd_compensated.h"
#include <unordered_map>
#include <vector>

#include "fdtd_adjoint.cuh"
#include "fdtd_b200.h"
#include "fdtd_flow.cuh"
#include "fdtd_kernels.cuh"

using namespace fdtd;

namespace {

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

constexpr uint64_t kPitchCells = 16;  // rows padded to a multiple of 16 cells
constexpr uint64_t kFineX = 32, kFineY = 16;  // the blocks tile_list counts interior cells in
constexpr uint64_t kGraphSteps = 64;  // steps of fdtd_run's captured chunk (even: the roles return)
// Grids of at least this many (pitched) cells step by direct launches in fdtd_run: their steps are
// long enough (a quarter of a millisecond and more) that launching costs nothing, and replaying a
// captured graph measured 8 % slower than the launches on the 47M-cell room (the streams
// overlapped less). Smaller grids replay the graph: below some 10M cells a step's launches and
// event waits cost as much host time as the step takes on the device.
constexpr uint64_t kGraphCells = 1ull << 25;

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The adjoint's device state (fdtd_adjoint.cuh): its tables, the two adjoint levels of the field
// and of the branch velocities, each row's L~, and the tensor maps of the sweep over the levels.
struct AdjointState {
    AdjointTables t{};
    CUtensorMap map_t;  // the cell types of the adjoint sweep: the cells special rows read left out
    CUtensorMap map_s;  // with a speed field, the scales in the adjoint sweep's boxes
    void *lam[2] = {nullptr, nullptr};
    void *om[2] = {nullptr, nullptr};
    void *tilde[2] = {nullptr, nullptr};  // L~ of the level at hand, and of the next (alternating)
    CUtensorMap lam_b[2], lam_a[2];
    void *carried = nullptr;  // the matched layer's carried values (9 per cell)
    void *hat[2] = {nullptr, nullptr};  // the matched layer's terms' factors (kHats a pitched cell), a step's and the next's
    void *pending = nullptr;  // the layer's Q^, L^, H^ of a step whose factors come with the next segment
    // The layer cells sorted by their coordinate along each axis in turn (x, then y, then z; each
    // a permutation of the cells) and each coordinate's first entry: the tables' sums by coordinate.
    const uint32_t *by_coord = nullptr, *coord_start = nullptr;
};

}  // namespace

struct fdtd_solver {
    int device = 0;
    int sms = 148;  // multiprocessors of the device
    int precision = FDTD_FP32;
    bool wide = false, scaled = false;
    cudaStream_t stream = nullptr;  // the handle's stream: the interior sweep
    cudaStream_t side = nullptr;    // special rows and probes, beside the sweep within each step
    cudaStream_t layer_stream = nullptr;  // the matched layer, beside the sweep within each step
    int layer_priority = 0;               // the device's highest stream priority
    // A step's start on the handle's stream, and the side and layer streams' ends of a step.
    cudaEvent_t joined[3] = {nullptr, nullptr, nullptr};
    std::string error;
    Tables tables{};
    BulkArgs bulk{};
    uint32_t bulk_blocks = 0;  // the persistent grid: resident blocks, at most one per tile
    // Blocks an SM of the matched-layer and special-row kernels (0: one thread a cell), chosen by
    // fdtd_autotune.
    int layer_per_sm = kLayerPerSm, special_per_sm = kSpecialPerSm;
    // Blocks an SM of the reverse step's launches of the rows far from the layer and of those near
    // it with the layer's cells (0: a block for every 128 items; fdtd_set_adjoint_launch). Measured
    // on the 4 cm room's gradient: 0 and 8 took 99 ms for 200 reverse steps, 0 and 0 102.5 ms, and
    // any cap on the far rows more (106-257 ms).
    int adjoint_far_per_sm = 0, adjoint_near_per_sm = 8;
    // How a step's kernels share the streams (fdtd_set_streams): 1, each kind on its own; 2, the
    // layer and then the special rows beside the sweep; 3, the special rows after the sweep, the
    // layer beside them; 0, all in turn (fdtd_autotune times them: where the special rows are many,
    // running them beside the sweep can cost the sweep more than it saves).
    int concurrent = 1;
    uint32_t bulk_tiles = 0;
    int bulk_per_sm = 0;      // resident bulk blocks per multiprocessor (shape 0)
    int shape_per_sm[kShapes] = {};  // the same, each shape
    // The sweep's tile shape (an index of kShapeInfo) and planes a tile, chosen by fdtd_autotune
    // or fdtd_set_tiles; the pitched cell types kept on the host to lay the tiles out again; the
    // forward list's device copy (replaced with the shape), and the adjoint's list (shape 0, no
    // full tiles).
    int bulk_shape = 0;
    uint64_t bulk_chunk = 32;
    std::vector<uint8_t> host_types;
    // The interior cells of each kFineX x kFineY block of each plane (tile_list's counts), and
    // the blocks along x and y.
    std::vector<uint32_t> fine_count;
    uint64_t fine_x = 0, fine_y = 0;
    void *tiles_device = nullptr;
    const int4 *plain_tiles = nullptr;
    uint32_t plain_count = 0;
    uint64_t nx = 0, ny = 0, nz = 0, n = 0, pitch = 0, n_device = 0;
    uint64_t air = 0, interior = 0, links = 0, states = 0, layers = 0, probes = 0, specials = 0;
    uint64_t steps_done = 0;
    std::vector<void *> allocations;  // every device allocation the handle owns
    uint64_t device_bytes = 0;
    // The state: u[1] is the current pressure between runs, u[0] the one a step before; the same
    // for the branch velocities w.
    void *u[2] = {nullptr, nullptr};
    void *w[2] = {nullptr, nullptr};
    void *increment = nullptr;              // FDTD_FP32_COMPENSATED: p_n - p_(n-1) per cell (pitched)
    std::vector<uint32_t> layer_cells;      // pitched, in the layout's order (for fdtd_read_state)
    const uint8_t *types_device = nullptr;  // the pitched cell types
    const float *scale_device = nullptr;    // with a speed field: each pitched cell's scale
    // The matched layer's state (kLayerSlots values a pitched cell: its parts and the velocities on
    // its + faces; only the layer's cells and their - faces used), in two buffers: layer_state[1]
    // holds the latest values between runs, as u[1] does.
    void *layer_state[2] = {nullptr, nullptr};
    uint32_t link_slots = 0;  // the most links of a special row (6 or 18 kernels)
    // Moving air (fdtd_flow.cuh): whether the grid's air moves, which form carries it, the carry's
    // cell lists, fields and stage buffers, and its launches' blocks.
    bool flowing = false, flow_round = false;
    Flow flow{};
    uint32_t flow_blocks = 0;
    unsigned int *d_error = nullptr;  // set by a kernel whose wait gave up
    // Tensor maps of the bulk sweep: each level as the pressure tile (with halos) and as the
    // previous-pressure tile, the cell types and the scales.
    CUtensorMap map_b[2], map_a[2], map_t, map_s;
    CUtensorMap map_d;  // FDTD_FP32_COMPENSATED: the increments, in the previous pressure's place
    // fdtd_run's chunks: the drive and the records of kGraphSteps steps on the device, and the
    // graph of a chunk's launches for each of the levels' two roles (captured on first use).
    float *d_sig = nullptr;
    double *d_rec = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool flipped = false;  // the levels' roles swapped from the handle's first (an odd count of steps)
    // Per-kernel timing (fdtd_set_timing): per timed step, a start and an end event per kind.
    bool timing = false;
    std::vector<cudaEvent_t> timing_events;  // 8 per step: (start, end) of bulk, layer, special, probe
    uint64_t timed_steps = 0;
    // The adjoint (fdtd_gradient), set up on first use and kept.
    bool adjoint_ready = false;
    AdjointState adjoint;
    std::vector<int32_t> adjoint_reader_row;  // of the kept adjoint (fdtd_set_coefficients)
    std::vector<uint32_t> adjoint_corrected_row;
    std::vector<double> adjoint_reader_base, adjoint_corrected_base;
    std::vector<uint32_t> adjoint_layer_row;  // rows linking to layer cells, and their bases
    std::vector<double> adjoint_layer_base;
    std::vector<int32_t> state_branch;  // each branch state's branch
    // The last gradient's part in the matched layer's tables (fdtd_layer_gradient), empty without.
    std::vector<double> layer_gradient;
    bool gradient_tables = true;  // whether gradients also give the layer tables' (fdtd_set_gradient_tables)
    // A tangent of the layer's tables (fdtd_set_layer_tangent): gradients then give dL/dθ along it in
    // place of the tables' gradient. Its factors a step (three per layer cell and axis it touches),
    // the device tables it uses (freed when replaced), the last gradient's value, and a taped run's
    // factors of every step beside the rows' trajectory (tape_t, with room for tape_t_steps steps;
    // stage_t: a captured chunk's, copied onto the tape after it).
    bool tangent = false;
    uint64_t tangent_factors = 0;
    std::vector<void *> tangent_device;
    bool tangent_valid = false;
    double tangent_gradient = 0.0;
    void *record_tangent = nullptr;  // while recording: the factors of a dispatch's first step
    void *tape_t = nullptr, *stage_t = nullptr;
    uint64_t tape_t_steps = 0;
    bool tape_tangent = false;  // the valid tape holds the tangent's factors of every step
    uint64_t branches = 0;
    // fdtd_gradient's device workspace, kept and handed out again in the same order while the
    // sizes asked for stay the same (a fit's iterations then allocate nothing).
    struct Block {
        void *p;
        size_t bytes;
    };
    std::vector<Block> work;
    // Graphs of a full segment's recomputation and reverse steps over the kept workspace
    // ([recompute/reverse][the levels' or adjoint levels' roles at the segment's start]), captured
    // once and replayed while the workspace and the segment stay.
    cudaGraphExec_t grad_graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    uint64_t graph_segment = 0;
    // While recording (the gradient's recomputation of a segment, or a taped run that keeps the
    // trajectory): the special rows' values and branch velocities after each step k of a dispatch,
    // written as level k + record_offset of record_u and record_w; the gradient's recomputation
    // needs no probe records (record_probes false).
    void *record_u = nullptr, *record_w = nullptr;
    void *record_layer = nullptr;  // the layer's factors of each step (kLayerFactors x layers a step)
    uint64_t record_offset = 2;
    bool record_probes = true;
    // The tape (fdtd_set_tape): a run of fdtd_run from rest keeps, for the gradient that follows,
    // its drive and either the whole trajectory of the special rows and branch velocities (levels
    // 0 .. steps+1 of tape_u, tape_w: what the gradient otherwise recomputes), when that fits in
    // tape_budget bytes, or else the state at every multiple of tape_segment steps before its end.
    uint64_t tape_segment = 0;
    uint64_t tape_budget = UINT64_MAX;  // UINT64_MAX: half the device memory free at the run
    bool tape_valid = false;
    bool tape_traj = false;  // the valid tape holds the trajectory (no checkpoints)
    std::vector<float> tape_signal;
    std::vector<void *> tape_checkpoints;
    void *tape_u = nullptr, *tape_w = nullptr;
    uint64_t tape_levels = 0;  // levels tape_u and tape_w have room for
    // A taped run's chunks record into staging (kGraphSteps levels), copied onto the tape after
    // each chunk, through graphs of their own ([the levels' roles]).
    void *stage_u = nullptr, *stage_w = nullptr;
    cudaGraphExec_t tape_graph[2] = {nullptr, nullptr};
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

#define CUDA_TRY(s, call)                                      \
    do {                                                       \
        cudaError_t e_ = (call);                               \
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
    // On the handle's stream, which every later use of the buffer follows (the streams are
    // non-blocking: they do not wait for the legacy default stream).
    CUDA_TRY(s, cudaMemsetAsync(p, 0, bytes ? bytes : 16, s->stream));
    *out = p;
    return FDTD_OK;
}

// Whether cell i's air moves: the plain form's shifts, or the round form's mask (fdtd.hpp:2049-2097
// skips the others, whose levels stand still through the carry).
bool moves(const fdtd_layout *L, uint64_t i) {
    if (L->types[i] == kSolid) return false;
    return L->wind[0] ? L->flow_mask[i] != 0 : (L->flow_x[i] != 0.0f || L->flow_y[i] != 0.0f);
}

// The cells the carry of moving cell (x, y, z) reads, as (axis, step) pairs: the plain form's x
// and y neighbours as its mask's bits allow them (fdtd.hpp:1946-1967), the round form's two
// neighbours either side along every axis (fdtd.hpp:1978-2020).
template <class Visit>
void flow_reads(const fdtd_layout *L, uint64_t i, Visit visit) {
    if (L->wind[0]) {
        for (int a = 0; a < 3; ++a)
            for (int step : {-2, -1, 1, 2}) visit(a, step);
        return;
    }
    for (int a = 0; a < 2; ++a) {
        const unsigned m = a == 0 ? (L->flow_mask[i] & 15u) : (L->flow_mask[i] >> 4);
        if (m == 15u) {
            for (int step : {-2, -1, 1, 2}) visit(a, step);
            continue;
        }
        if (m & 1u) visit(a, -1);
        if (m & 2u) visit(a, 1);
        if (m & 4u) visit(a, -2);
        if (m & 8u) visit(a, 2);
    }
}

// The moving air's arrays present, and every cell a moving cell's carry reads inside the grid
// (the reference leaves two cells of still air or wall round it).
std::string flow_check(const fdtd_layout *L) {
    const uint64_t n = L->nx * L->ny * L->nz;
    if (L->flow_count != n) return "moving air needs one mask per cell";
    if (!L->flow_mask) return "moving air needs its mask";
    const bool round = L->wind[0] != nullptr;
    for (int d = 0; d < 3; ++d)
        if (round && (!L->wind[d] || !L->loop[d])) return "the round form needs each axis's winds and loops";
    if (!round && (!L->flow_x || !L->flow_y)) return "the plain form needs the shifts along x and y";
    const uint64_t len[3] = {L->nx, L->ny, L->nz};
    for (uint64_t i = 0; i < n; ++i) {
        if (!moves(L, i)) continue;
        const uint64_t at[3] = {i % L->nx, (i / L->nx) % L->ny, i / (L->nx * L->ny)};
        bool inside = true;
        flow_reads(L, i, [&](int a, int step) {
            const int64_t c = (int64_t)at[a] + step;
            if (c < 0 || c >= (int64_t)len[a]) inside = false;
        });
        if (!inside) return "a moving cell's carry reads outside the grid";
    }
    return "";
}

int validate(const fdtd_layout *L, std::string &why) {
    auto refuse = [&](const std::string &m) {
        why = m;
        return FDTD_EINVAL;
    };
    if (!L) return refuse("no layout");
    if (L->stencil != 7 && L->stencil != 19) return refuse("the stencil has 7 or 19 points");
    if (L->nx < 3 || L->ny < 3 || L->nz < 3) return refuse("the grid is too small");
    if (L->flow_count) {
        const std::string bad = flow_check(L);
        if (!bad.empty()) return refuse(bad);
    }
    const uint64_t n = L->nx * L->ny * L->nz;
    if (L->nx > (1ull << 31) || L->ny > (1ull << 31) || L->nz > (1ull << 31) || n >= (1ull << 32) ||
        n / L->nx / L->ny != L->nz)
        return refuse("the wave grid is too large for the GPU's 32-bit indices");
    if (L->weight_count < (L->stencil == 19 ? 18u : 6u) || !L->weights)
        return refuse("the layout's weights do not match its stencil");
    if (!L->types) return refuse("the layout has no cell types");
    if (L->scaled && !L->scale) return refuse("a scaled layout needs each cell's scale");
    if (L->scaled) {
        // A cell's scale is its speed ratio squared; the reference refuses a ratio outside (0, 1]
        // (fdtd.hpp:415-425), so no scale lies outside it either.
        const uint64_t n = L->nx * L->ny * L->nz;
        for (uint64_t i = 0; i < n; ++i)
            if (!(L->scale[i] > 0.0f && L->scale[i] <= 1.0f))
                return refuse("each cell's speed of sound over the grid's lies in (0, 1]");
        for (uint64_t c = 0; c < L->layer_count; ++c)
            if (L->layer_scale && !(L->layer_scale[c] > 0.0f && L->layer_scale[c] <= 1.0f))
                return refuse("each cell's speed of sound over the grid's lies in (0, 1]");
    }
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
        if (L->stencil != 7) return refuse("the matched layer needs the 7-point stencil");
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

// A layout index (x fastest, rows of nx) as the device's pitched index.
inline uint32_t pitched(const fdtd_solver *s, uint64_t i) {
    const uint64_t x = i % s->nx, y = (i / s->nx) % s->ny, z = i / (s->nx * s->ny);
    return (uint32_t)(x + s->pitch * (y + s->ny * z));
}

EncodeTiled encoder() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

// A tensor map of the pitched 3-D array at `base` (pitch x ny x nz of `type`) read in boxes of
// box_x x box_y x 1; zero fill outside it.
int tensor_map(fdtd_solver *s, CUtensorMap *map, void *base, CUtensorMapDataType type, uint32_t bytes,
               uint32_t box_x, uint32_t box_y) {
    EncodeTiled encode = encoder();
    if (!encode) return fail(s, FDTD_ECUDA, "the CUDA driver has no cuTensorMapEncodeTiled");
    const cuuint64_t dims[3] = {s->pitch, s->ny, s->nz};
    const cuuint64_t strides[2] = {s->pitch * bytes, s->pitch * s->ny * bytes};
    const cuuint32_t box[3] = {box_x, box_y, 1};
    const cuuint32_t unit[3] = {1, 1, 1};
    const CUresult r = encode(map, type, 3, base, dims, strides, box, unit, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(s, FDTD_ECUDA, "cuTensorMapEncodeTiled refused a tensor map");
    return FDTD_OK;
}

// Planes a tile by default: at most 64, halved while there would be fewer than 8 tiles a
// multiprocessor (at least 8 planes).
uint64_t default_chunk(const fdtd_solver *s) {
    const BulkArgs &bk = s->bulk;
    const uint64_t cols = ((bk.x1 - bk.xa + 63) / 64) * ((bk.y1 - bk.y0 + 15) / 16);
    const uint64_t planes = cols * (bk.z1 - bk.z0);
    uint64_t chunk = 64;
    while (chunk > 8 && planes / chunk < (uint64_t)s->sms * 8) chunk /= 2;
    return chunk;
}

// The sweep's tile list for shape `shape`: the columns of TX x TY cells over the interior cells'
// box (x from its 16-aligned start), and in each the runs of planes that hold interior cells, cut
// into chunks of at most `chunk` planes. Grids of many rooms (stacked along z) skip the planes
// between the rooms. With `flags`, a tile whose cells are all interior in all of its planes is
// marked kFullTile.
int tile_list(fdtd_solver *s, int shape, uint64_t chunk, bool flags, std::vector<int4> &list) {
    const BulkArgs &bk = s->bulk;
    const uint64_t TX = (uint64_t)kShapeInfo[shape].tx, TY = (uint64_t)kShapeInfo[shape].ty;
    const uint64_t nz = s->nz, nx = s->nx, ny = s->ny, pitch = s->pitch;
    const uint64_t tiles_x = (bk.x1 - bk.xa + TX - 1) / TX, tiles_y = (bk.y1 - bk.y0 + TY - 1) / TY;
    const uint64_t columns = tiles_x * tiles_y;
    // The interior cells of each block of kFineX x kFineY cells of each plane, counted once for the
    // handle (its cell types never change): every shape's tile is a whole number of such blocks.
    if (s->fine_count.empty()) {
        s->fine_x = (bk.x1 - bk.xa + kFineX - 1) / kFineX, s->fine_y = (bk.y1 - bk.y0 + kFineY - 1) / kFineY;
        s->fine_count.assign(s->fine_x * s->fine_y * nz, 0);
        for (uint64_t z = bk.z0; z < bk.z1; ++z)
            for (uint64_t y = bk.y0; y < bk.y1; ++y) {
                const uint8_t *row = &s->host_types[pitch * (y + ny * z)];
                uint32_t *fine = &s->fine_count[((y - bk.y0) / kFineY * s->fine_x) * nz + z];
                for (uint64_t x0 = bk.xa; x0 < bk.x1; x0 += kFineX) {
                    uint32_t n = 0;
                    for (uint64_t x = x0, x1 = std::min<uint64_t>(x0 + kFineX, bk.x1); x < x1; ++x) n += row[x] == kInterior;
                    fine[(x0 - bk.xa) / kFineX * nz] += n;
                }
            }
    }
    static_assert(kFineX == 32 && kFineY == 16, "the shapes' tiles are whole blocks of 32 x 16 cells");
    const uint64_t per_x = TX / kFineX, per_y = TY / kFineY;
    // Per column and plane: interior cells it holds.
    std::vector<uint32_t> count(columns * nz, 0);
    for (uint64_t c = 0; c < columns; ++c) {
        const uint64_t tx = c % tiles_x, ty = c / tiles_x;
        for (uint64_t b = 0; b < per_y; ++b)
            for (uint64_t a = 0; a < per_x; ++a) {
                const uint64_t fx = tx * per_x + a, fy = ty * per_y + b;
                if (fx >= s->fine_x || fy >= s->fine_y) continue;
                const uint32_t *fine = &s->fine_count[(fy * s->fine_x + fx) * nz];
                for (uint64_t z = bk.z0; z < bk.z1; ++z) count[c * nz + z] += fine[z];
            }
    }
    list.clear();
    for (uint64_t c = 0; c < columns; ++c) {
        const uint64_t xt = bk.xa + (c % tiles_x) * TX, yt = bk.y0 + (c / tiles_x) * TY;
        // A plane of the column is full when all its TX x TY cells lie in the grid and are interior.
        const bool inside = xt + TX <= nx && yt + TY <= ny;
        for (uint64_t z = 0; z < nz;) {
            if (!count[c * nz + z]) {
                ++z;
                continue;
            }
            uint64_t end = z;
            bool full = flags && inside;
            while (end < nz && count[c * nz + end] && end - z < chunk) {
                full = full && count[c * nz + end] == TX * TY;
                ++end;
            }
            list.push_back(make_int4((int)xt, (int)yt, (int)z, (int)end | (full ? kFullTile : 0)));
            z = end;
        }
    }
    if (list.size() >= (1ull << 31)) return fail(s, FDTD_EINVAL, "the wave grid is too large for one launch");
    return FDTD_OK;
}

// Lays the sweep's tiles out for shape `shape` and `chunk` planes a tile: its list on the device
// (the previous one freed) and the tensor maps with the shape's boxes.
int use_shape(fdtd_solver *s, int shape, uint64_t chunk) {
    if (shape < 0 || shape >= kShapes) return fail(s, FDTD_EINVAL, "no such tile shape");
    if (chunk < 1 || chunk > 1024) return fail(s, FDTD_EINVAL, "planes a tile out of 1 to 1024");
    std::vector<int4> list;
    int rc;
    if ((rc = tile_list(s, shape, chunk, true, list))) return rc;
    // The previous list is no longer read once the handle's work has ended.
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (s->tiles_device) {
        auto it = std::find(s->allocations.begin(), s->allocations.end(), s->tiles_device);
        if (it != s->allocations.end()) s->allocations.erase(it);
        s->device_bytes -= sizeof(int4) * s->bulk_tiles;
        cudaFree(s->tiles_device);
        s->tiles_device = nullptr;
    }
    const int4 *d_list;
    if ((rc = upload(s, list.data(), list.size(), &d_list))) return rc;
    s->tiles_device = const_cast<int4 *>(d_list);
    s->bulk_tiles = (uint32_t)list.size();
    s->bulk.tiles = s->bulk_tiles;
    s->bulk.tile_list = d_list;
    s->bulk_blocks = s->bulk_tiles;  // one tile a block
    s->bulk_shape = shape;
    s->bulk_chunk = chunk;
    const uint32_t TX = (uint32_t)kShapeInfo[shape].tx, TY = (uint32_t)kShapeInfo[shape].ty;
    const uint32_t BX = TX + 2 * kHX, BY = TY + 2;
    const size_t e = s->precision == FDTD_FP64 ? 8 : 4;
    const CUtensorMapDataType ft = e == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    // The levels' roles at this moment (u[1] current): map_b/map_a[k] follow u[k].
    for (int k = 0; k < 2; ++k) {
        if ((rc = tensor_map(s, &s->map_b[k], s->u[k], ft, (uint32_t)e, BX, BY))) return rc;
        if ((rc = tensor_map(s, &s->map_a[k], s->u[k], ft, (uint32_t)e, TX, TY))) return rc;
    }
    if (s->increment && (rc = tensor_map(s, &s->map_d, s->increment, ft, (uint32_t)e, TX, TY))) return rc;
    if ((rc = tensor_map(s, &s->map_t, const_cast<uint8_t *>(s->types_device), CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, TX, TY)))
        return rc;
    if ((rc = tensor_map(s, &s->map_s, s->scaled ? const_cast<float *>(s->scale_device) : s->u[0],
                         CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, TX, TY)))
        return rc;
    // Captured chunks hold the old list and maps.
    for (cudaGraphExec_t &g : s->graph)
        if (g) cudaGraphExecDestroy(g), g = nullptr;
    for (cudaGraphExec_t &g : s->tape_graph)
        if (g) cudaGraphExecDestroy(g), g = nullptr;
    for (auto &row : s->grad_graph)
        for (cudaGraphExec_t &g : row)
            if (g) cudaGraphExecDestroy(g), g = nullptr;
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
    f.d = static_cast<T *>(s->increment);
    f.cell_old = static_cast<const T *>(s->layer_state[cur]);
    f.cell_new = static_cast<T *>(s->layer_state[prev]);
    return f;
}

template <typename T, bool WIDE, bool SCALED, bool COMP, class SH>
int set_up_shape(fdtd_solver *s, int *per_sm) {
    CUDA_TRY(s, cudaFuncSetAttribute(bulk_kernel<T, WIDE, SCALED, COMP, SH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)Stage<T, SCALED, SH>::smem));
    CUDA_TRY(s, cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, bulk_kernel<T, WIDE, SCALED, COMP, SH>, SH::THREADS,
                                                              Stage<T, SCALED, SH>::smem));
    return FDTD_OK;
}

// Every shape's shared memory set up; the resident blocks an SM of each kept.
template <typename T, bool WIDE, bool SCALED, bool COMP>
int set_up_kernels(fdtd_solver *s) {
    int rc;
    if ((rc = set_up_shape<T, WIDE, SCALED, COMP, Shape0>(s, &s->shape_per_sm[0]))) return rc;
    if ((rc = set_up_shape<T, WIDE, SCALED, COMP, Shape1>(s, &s->shape_per_sm[1]))) return rc;
    if ((rc = set_up_shape<T, WIDE, SCALED, COMP, Shape2>(s, &s->shape_per_sm[2]))) return rc;
    if ((rc = set_up_shape<T, WIDE, SCALED, COMP, Shape3>(s, &s->shape_per_sm[3]))) return rc;
    if ((rc = set_up_shape<T, WIDE, SCALED, COMP, Shape4>(s, &s->shape_per_sm[4]))) return rc;
    if ((rc = set_up_shape<T, WIDE, SCALED, COMP, Shape5>(s, &s->shape_per_sm[5]))) return rc;
    if ((rc = set_up_shape<T, WIDE, SCALED, COMP, Shape6>(s, &s->shape_per_sm[6]))) return rc;
    if ((rc = set_up_shape<T, WIDE, SCALED, COMP, Shape7>(s, &s->shape_per_sm[7]))) return rc;
    if ((rc = set_up_shape<T, WIDE, SCALED, COMP, Shape8>(s, &s->shape_per_sm[8]))) return rc;
    if ((rc = set_up_shape<T, WIDE, SCALED, COMP, Shape9>(s, &s->shape_per_sm[9]))) return rc;
    s->bulk_per_sm = s->shape_per_sm[0];
    return FDTD_OK;
}

// One launch of the sweep in the handle's shape.
template <typename T, bool WIDE, bool SCALED, bool COMP>
void launch_bulk(const fdtd_solver *s, const CUtensorMap &mb, const CUtensorMap &ma, const BulkArgs &args) {
#define FDTD_BULK(SH)                                                                          \
    bulk_kernel<T, WIDE, SCALED, COMP, SH><<<s->bulk_blocks, SH::THREADS, Stage<T, SCALED, SH>::smem, s->stream>>>( \
        mb, ma, s->map_t, s->map_s, args)
    switch (s->bulk_shape) {
        case 1: FDTD_BULK(Shape1); break;
        case 2: FDTD_BULK(Shape2); break;
        case 3: FDTD_BULK(Shape3); break;
        case 4: FDTD_BULK(Shape4); break;
        case 5: FDTD_BULK(Shape5); break;
        case 6: FDTD_BULK(Shape6); break;
        case 7: FDTD_BULK(Shape7); break;
        case 8: FDTD_BULK(Shape8); break;
        case 9: FDTD_BULK(Shape9); break;
        default: FDTD_BULK(Shape0); break;
    }
#undef FDTD_BULK
}

// The carry of both levels (b, the current, and a), before a step's updates.
template <typename T>
int launch_carry(fdtd_solver *s, const Fields<T> &f, cudaStream_t stream) {
    T *b = const_cast<T *>(f.b), *a = f.a;
    const dim3 grid(s->flow_blocks, 2);
    if (s->flow_round) {
        carry_kernel<T, true, 1><<<grid, kBlock, 0, stream>>>(s->flow, b, a);
        carry_kernel<T, true, 2><<<grid, kBlock, 0, stream>>>(s->flow, b, a);
        carry_kernel<T, true, 3><<<grid, kBlock, 0, stream>>>(s->flow, b, a);
    } else {
        carry_kernel<T, false, 1><<<grid, kBlock, 0, stream>>>(s->flow, b, a);
        carry_kernel<T, false, 2><<<grid, kBlock, 0, stream>>>(s->flow, b, a);
        carry_kernel<T, false, 3><<<grid, kBlock, 0, stream>>>(s->flow, b, a);
    }
    return FDTD_OK;
}

template <typename T, bool WIDE, bool SCALED, bool COMP = false>
int launch_steps(fdtd_solver *s, const float *d_signal, uint64_t steps, double *d_out, uint64_t stride) {
    const Tables &g = s->tables;
    // The layer and special kernels loop over their cells: a few blocks an SM each (the handle's
    // layer_per_sm, special_per_sm; 0: a thread a cell), leaving the sweep's blocks their places.
    const uint64_t special_cap = s->special_per_sm ? (uint64_t)s->sms * s->special_per_sm : UINT64_MAX;
    const uint64_t layer_cap = s->layer_per_sm ? (uint64_t)s->sms * s->layer_per_sm : UINT64_MAX;
    const uint32_t special_blocks = (uint32_t)std::min<uint64_t>((s->specials + kBlock - 1) / kBlock, special_cap);
    const uint32_t probe_blocks = (uint32_t)((s->probes + kProbeWarps - 1) / kProbeWarps);
    const uint32_t layer_blocks = (uint32_t)std::min<uint64_t>((s->layers + kBlock - 1) / kBlock, layer_cap);
    // Each step: the interior sweep on the handle's stream; beside it the matched layer on the
    // layer stream, of the highest priority (its blocks take the thread slots that the sweep's
    // shared memory leaves free on every multiprocessor), and the special rows and probes on the
    // side stream. The three write disjoint memory; each step starts when all three have ended the
    // step before. While timing, all run one after another on the handle's stream, so that each
    // kernel's events bracket that kernel alone.
    // The streams (fdtd_set_streams): 1, the three kinds each on its own; 2, the layer and then the
    // special rows and probes on the side stream beside the sweep; 3, the special rows and probes
    // after the sweep on its stream, the layer beside them; 0, all in turn; 4 and 5, as 1 and 2
    // with the special rows launched at the highest priority as well. A kernel's blocks wait until
    // those of the kernels before it at the same priority have all been dispatched, so beside a
    // sweep of many waves the special rows would otherwise start only in its last wave.
    const int mode = s->timing ? 0 : s->concurrent;
    const bool fork = mode != 0;
    const int streams = mode >= 4 ? mode - 3 : mode;
    const bool special_first = mode >= 4;
    cudaStream_t side = streams == 1 || streams == 2 ? s->side : s->stream;
    cudaStream_t layer = streams == 1 || streams == 3 ? s->layer_stream : (streams == 2 ? s->side : s->stream);
    auto launch_special = [&](auto kernel, const Fields<T> &f) -> cudaError_t {
        if (!special_first) {
            kernel<<<special_blocks, kBlock, 0, side>>>(g, f);
            return cudaGetLastError();
        }
        cudaLaunchConfig_t config{};
        config.gridDim = dim3(special_blocks);
        config.blockDim = dim3(kBlock);
        config.stream = side;
        cudaLaunchAttribute priority{};
        priority.id = cudaLaunchAttributePriority;
        priority.val.priority = s->layer_priority;
        config.attrs = &priority;
        config.numAttrs = 1;
        return cudaLaunchKernelEx(&config, kernel, g, f);
    };
    for (uint64_t k = 0; k < steps; ++k) {
        const bool flip = (k & 1) != 0;
        Fields<T> f = fields_for<T>(s, flip);
        f.signal = d_signal + k;
        f.out = d_out + k;
        f.out_stride = stride;
        if (s->record_u) {
            // The special rows' new values, level k + record_offset of the trajectory.
            f.traj_u = static_cast<T *>(s->record_u) + (k + s->record_offset) * s->specials;
            f.traj_w = static_cast<T *>(s->record_w) + (k + s->record_offset) * s->states;
        }
        // The matched layer's factors of step k (the gradient's recomputation).
        if (s->record_layer) f.traj_layer = static_cast<T *>(s->record_layer) + k * kLayerFactors * s->layers;
        // The factors of step k along the tables' tangent (a gradient's recomputation, or a taped run).
        if (s->record_tangent) f.traj_tangent = static_cast<T *>(s->record_tangent) + k * s->tangent_factors;
        if (fork) {
            if (k > 0) {
                CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->joined[1], 0));
                if (layer_blocks) CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->joined[2], 0));
            }
        }
        // Moving air: the probes read the levels before the carry moves them (fdtd.hpp:833-840
        // after the record of fdtd.hpp:3525-3533); the step's updates follow the carry.
        if (s->flowing) {
            if (probe_blocks && s->record_probes) probe_kernel<T><<<probe_blocks, kBlock, 0, s->stream>>>(g, f);
            launch_carry<T>(s, f, s->stream);
        }
        if (fork) {
            CUDA_TRY(s, cudaEventRecord(s->joined[0], s->stream));
            CUDA_TRY(s, cudaStreamWaitEvent(side, s->joined[0], 0));
            if (layer_blocks) CUDA_TRY(s, cudaStreamWaitEvent(layer, s->joined[0], 0));
        }
        cudaEvent_t *ev = nullptr;
        if (s->timing) {
            // (Created on demand; recorded only outside graph captures.)
            const size_t base = s->timing_events.size();
            for (int e = 0; e < 8; ++e) {
                cudaEvent_t event;
                CUDA_TRY(s, cudaEventCreate(&event));
                s->timing_events.push_back(event);
            }
            ev = &s->timing_events[base];
            ++s->timed_steps;
        }
        if (ev) CUDA_TRY(s, cudaEventRecord(ev[0], s->stream));
        if (s->bulk_blocks) {
            BulkArgs args = s->bulk;
            args.a = f.a;
            args.d = f.d;
            const int cur = flip ? 0 : 1, prev = flip ? 1 : 0;
            // (Compensated: the increments stand in the previous pressure's place.)
            launch_bulk<T, WIDE, SCALED, COMP>(s, s->map_b[cur], COMP ? s->map_d : s->map_a[prev], args);
        }
        if (ev) CUDA_TRY(s, cudaEventRecord(ev[1], s->stream));
        if (ev) CUDA_TRY(s, cudaEventRecord(ev[2], layer));
        if (layer_blocks) {
            // With the priority as a launch attribute too, so that a captured graph keeps it.
            cudaLaunchConfig_t config{};
            config.gridDim = dim3(layer_blocks);
            config.blockDim = dim3(kBlock);
            config.stream = layer;
            cudaLaunchAttribute priority{};
            priority.id = cudaLaunchAttributePriority;
            priority.val.priority = s->layer_priority;
            config.attrs = &priority;
            config.numAttrs = 1;
            CUDA_TRY(s, cudaLaunchKernelEx(&config, layer_kernel<T, SCALED, COMP>, g, f));
        }
        if (ev) CUDA_TRY(s, cudaEventRecord(ev[3], layer));
        if (ev) CUDA_TRY(s, cudaEventRecord(ev[4], side));
        if (special_blocks) {
            if (g.link_mask)
                CUDA_TRY(s, launch_special(special_kernel<T, 0, COMP>, f));
            else if (s->link_slots <= 6)
                CUDA_TRY(s, launch_special(special_kernel<T, 6, COMP>, f));
            else
                CUDA_TRY(s, launch_special(special_kernel<T, 18, COMP>, f));
        }
        if (ev) CUDA_TRY(s, cudaEventRecord(ev[5], side));
        if (ev) CUDA_TRY(s, cudaEventRecord(ev[6], side));
        // (A recomputation for the gradient records the special rows instead of the probes.)
        if (probe_blocks && s->record_probes && !s->flowing) probe_kernel<T><<<probe_blocks, kBlock, 0, side>>>(g, f);
        if (ev) CUDA_TRY(s, cudaEventRecord(ev[7], side));
        if (fork) {
            CUDA_TRY(s, cudaEventRecord(s->joined[1], side));
            if (layer_blocks) CUDA_TRY(s, cudaEventRecord(s->joined[2], layer));
        }
    }
    // The handle's stream ends after all three.
    if (fork && steps) {
        CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->joined[1], 0));
        if (layer_blocks) CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->joined[2], 0));
    }
    CUDA_TRY(s, cudaGetLastError());
    return FDTD_OK;
}

template <typename T, bool W, bool S, bool C>
int dispatch_run(fdtd_solver *s, const float *d_signal, uint64_t steps, double *d_out, uint64_t stride) {
    return launch_steps<T, W, S, C>(s, d_signal, steps, d_out, stride);
}

// The instantiation for the grid: precision (and compensated single), stencil, speed field.
#define FDTD_BY_KIND(CALL)                                                                                   \
    do {                                                                                                     \
        if (s->precision == FDTD_FP64) {                                                                     \
            if (!s->wide) return s->scaled ? CALL(double, false, true, false) : CALL(double, false, false, false); \
            return s->scaled ? CALL(double, true, true, false) : CALL(double, true, false, false);           \
        }                                                                                                    \
        if (s->precision == FDTD_FP32_COMPENSATED) {                                                         \
            if (!s->wide) return s->scaled ? CALL(float, false, true, true) : CALL(float, false, false, true); \
            return s->scaled ? CALL(float, true, true, true) : CALL(float, true, false, true);               \
        }                                                                                                    \
        if (!s->wide) return s->scaled ? CALL(float, false, true, false) : CALL(float, false, false, false); \
        return s->scaled ? CALL(float, true, true, false) : CALL(float, true, false, false);                 \
    } while (0)

int dispatch(fdtd_solver *s, const float *d_signal, uint64_t steps, double *d_out, uint64_t stride) {
#define RUN_CALL(T, W, S, C) dispatch_run<T, W, S, C>(s, d_signal, steps, d_out, stride)
    FDTD_BY_KIND(RUN_CALL);
#undef RUN_CALL
}

int set_up(fdtd_solver *s) {
#define SET_CALL(T, W, S, C) set_up_kernels<T, W, S, C>(s)
    FDTD_BY_KIND(SET_CALL);
#undef SET_CALL
}

// After `steps` steps the parity swap of fdtd.hpp:900-903: u[1] stays the current level.
void settle(fdtd_solver *s, uint64_t steps) {
    if (steps % 2 == 1) {
        s->flipped = !s->flipped;
        std::swap(s->u[0], s->u[1]);
        std::swap(s->w[0], s->w[1]);
        std::swap(s->layer_state[0], s->layer_state[1]);
        std::swap(s->map_b[0], s->map_b[1]);
        std::swap(s->map_a[0], s->map_a[1]);
    }
    s->steps_done += steps;
}

// Whether a kernel's wait gave up since the last check (then clears the flag).
int check_device_error(fdtd_solver *s) {
    unsigned int flag = 0;
    CUDA_TRY(s, cudaMemcpyAsync(&flag, s->d_error, sizeof flag, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (flag) {
        CUDA_TRY(s, cudaMemsetAsync(s->d_error, 0, sizeof flag, s->stream));
        CUDA_TRY(s, cudaStreamSynchronize(s->stream));
        if (flag & kWaitTestBit)
            return fail(s, FDTD_ECUDA, "a bounded wait gave up (fdtd_test_wait: the flag it waited on was never set)");
        return fail(s, FDTD_ECUDA, "a pipeline wait of the interior sweep gave up; the step's results are not valid");
    }
    return FDTD_OK;
}

// Captures the launches of kGraphSteps steps on the handle's chunk buffers, for the levels'
// present roles, as one executable graph (its side-stream branch forked and joined by events).
int capture(fdtd_solver *s, cudaGraphExec_t *out) {
    const bool timing = s->timing;
    s->timing = false;  // no timing events inside a graph
    CUDA_TRY(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = dispatch(s, s->d_sig, kGraphSteps, s->d_rec, kGraphSteps);
    s->timing = timing;
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    if (rc != FDTD_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(s, e, "cudaStreamEndCapture");
    // The nodes' own priorities (the matched layer's), not the launching stream's.
    const cudaError_t i = cudaGraphInstantiateWithFlags(out, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (i != cudaSuccess) return cuda_fail(s, i, "cudaGraphInstantiate");
    return FDTD_OK;
}

// Moving air on the device: the moving cells and the still air cells their carry reads (pitched),
// the form's fields pitched, and two stage buffers for each level (zero, as the cells never
// written stay: walls and padding read as still, silent air).
int set_up_flow(fdtd_solver *s, const fdtd_layout *L) {
    s->flowing = true;
    s->flow_round = L->wind[0] != nullptr;
    const uint64_t n = s->n, nx = s->nx, ny = s->ny;
    std::vector<uint32_t> cells, halo;
    std::vector<uint8_t> seen(n, 0);
    for (uint64_t i = 0; i < n; ++i)
        if (moves(L, i)) cells.push_back(pitched(s, i)), seen[i] = 1;
    const int64_t stride[3] = {1, (int64_t)nx, (int64_t)(nx * ny)};
    for (uint64_t i = 0; i < n; ++i) {
        if (!moves(L, i)) continue;
        flow_reads(L, i, [&](int a, int step) {
            const uint64_t j = (uint64_t)((int64_t)i + step * stride[a]);
            if (L->types[j] != kSolid && !seen[j]) seen[j] = 1, halo.push_back(pitched(s, j));
        });
    }
    std::sort(halo.begin(), halo.end());
    Flow &f = s->flow;
    f.moving = (uint32_t)cells.size();
    cells.insert(cells.end(), halo.begin(), halo.end());
    f.count = (uint32_t)cells.size();
    f.sy = (uint32_t)s->pitch;
    f.sz = (uint32_t)(s->pitch * ny);
    int rc;
    if ((rc = upload(s, cells.data(), cells.size(), &f.cells))) return rc;
    auto pitch_up = [&](const auto *host, auto **out) {
        using V = std::remove_const_t<std::remove_pointer_t<decltype(host)>>;
        std::vector<V> a(s->n_device, V(0));
        for (uint64_t z = 0; z < s->nz; ++z)
            for (uint64_t y = 0; y < ny; ++y)
                std::memcpy(&a[s->pitch * (y + ny * z)], &host[nx * (y + ny * z)], nx * sizeof(V));
        return upload(s, a.data(), a.size(), out);
    };
    if ((rc = pitch_up(L->flow_mask, &f.mask))) return rc;
    if (s->flow_round) {
        for (int d = 0; d < 3; ++d) {
            if ((rc = pitch_up(L->wind[d], &f.wind[d]))) return rc;
            if ((rc = pitch_up(L->loop[d], &f.loop[d]))) return rc;
        }
    } else {
        if ((rc = pitch_up(L->flow_x, &f.shift_x))) return rc;
        if ((rc = pitch_up(L->flow_y, &f.shift_y))) return rc;
    }
    const size_t e = s->precision == FDTD_FP64 ? 8 : 4;
    for (int k = 0; k < 2; ++k) {
        if ((rc = zeros(s, e * s->n_device, &f.t1[k]))) return rc;
        if ((rc = zeros(s, e * s->n_device, &f.t2[k]))) return rc;
    }
    s->flow_blocks = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((f.count + kBlock - 1) / kBlock, 4ull * s->sms));
    return FDTD_OK;
}

int build(fdtd_solver *s, const fdtd_layout *L) {
    const uint64_t nx = L->nx, ny = L->ny, nz = L->nz, n = nx * ny * nz;
    s->nx = nx, s->ny = ny, s->nz = nz, s->n = n;
    s->pitch = (nx + kPitchCells - 1) / kPitchCells * kPitchCells;
    s->n_device = s->pitch * ny * nz;
    if (s->n_device >= (1ull << 32)) return fail(s, FDTD_EINVAL, "the wave grid is too large for the GPU's 32-bit indices");
    s->wide = L->stencil == 19;
    s->scaled = L->scaled != 0;
    s->layers = L->layer_count;  // the sweep's instantiation depends on it
    const size_t e = s->precision == FDTD_FP64 ? 8 : 4;
    Tables &g = s->tables;
    g.pitch = (uint32_t)s->pitch;
    g.ny = (uint32_t)ny;
    g.nz = (uint32_t)nz;
    g.sz = (uint32_t)(s->pitch * ny);
    g.plane = (uint32_t)(s->pitch * ny);
    g.by_plane = FastDiv(g.plane);
    g.by_pitch = FastDiv(g.pitch);
    for (int k = 0; k < 18; ++k)
        g.offset[k] = (int32_t)(kSteps[k][0] + kSteps[k][1] * (int64_t)s->pitch + kSteps[k][2] * (int64_t)(s->pitch * ny));

    // Cell types and scales, pitched; the interior cells' bounding box and the air count.
    std::vector<uint8_t> types(s->n_device, (uint8_t)kSolid);
    std::vector<float> scale(s->scaled ? s->n_device : 0, 0.0f);
    uint64_t x0 = nx, y0 = ny, z0 = nz, x1 = 0, y1 = 0, z1 = 0, interior = 0, air = 0;
    for (uint64_t z = 0; z < nz; ++z)
        for (uint64_t y = 0; y < ny; ++y) {
            const uint64_t row = nx * (y + ny * z), drow = s->pitch * (y + ny * z);
            std::memcpy(&types[drow], &L->types[row], nx);
            if (s->scaled) std::memcpy(&scale[drow], &L->scale[row], nx * sizeof(float));
            for (uint64_t x = 0; x < nx; ++x) {
                const uint8_t t = L->types[row + x];
                if (t != kSolid) ++air;
                if (t != kInterior) continue;
                ++interior;
                x0 = std::min(x0, x), x1 = std::max(x1, x + 1);
                y0 = std::min(y0, y), y1 = std::max(y1, y + 1);
                z0 = std::min(z0, z), z1 = std::max(z1, z + 1);
            }
        }
    s->interior = interior, s->air = air;

    int rc;
    const uint8_t *d_types;
    if ((rc = upload(s, types.data(), types.size(), &d_types))) return rc;
    s->types_device = d_types;
    const float *d_scale = nullptr;
    if (s->scaled && (rc = upload(s, scale.data(), scale.size(), &d_scale))) return rc;
    s->scale_device = d_scale;

    // The state, at rest; the error flag.
    for (int k = 0; k < 2; ++k) {
        if ((rc = zeros(s, e * s->n_device, &s->u[k]))) return rc;
        if ((rc = zeros(s, e * L->state_count, &s->w[k]))) return rc;
    }
    if (s->precision == FDTD_FP32_COMPENSATED && (rc = zeros(s, e * s->n_device, &s->increment))) return rc;
    if (L->layer_count)
        for (int k = 0; k < 2; ++k)
            if ((rc = zeros(s, e * kLayerSlots * s->n_device, &s->layer_state[k]))) return rc;
    void *flag;
    if ((rc = zeros(s, sizeof(unsigned int), &flag))) return rc;
    s->d_error = static_cast<unsigned int *>(flag);
    void *chunk;
    if ((rc = zeros(s, sizeof(float) * kGraphSteps, &chunk))) return rc;
    s->d_sig = static_cast<float *>(chunk);
    if ((rc = zeros(s, sizeof(double) * kGraphSteps * std::max<uint64_t>(1, L->probe_count), &chunk))) return rc;
    s->d_rec = static_cast<double *>(chunk);
    if (L->flow_count && (rc = set_up_flow(s, L))) return rc;

    // The bulk sweep: tiles of kTX x kTY over the box, x from a 16-aligned start; chunks of planes
    // enough for every multiprocessor several times over.
    BulkArgs &bk = s->bulk;
    bk.pitch = (uint32_t)s->pitch;
    bk.ny = (uint32_t)ny;
    bk.axial = L->weights[0];
    bk.diagonal = s->wide ? L->weights[6] : 0.0f;
    bk.centre = L->centre;
    bk.total = L->total;
    bk.error = s->d_error;
    std::vector<float> row_residual(L->special_count);
    fdtd_compensated_residuals(L, &bk.residual, row_residual.data());
    if (interior) {
        bk.xa = (uint32_t)(x0 / 16 * 16);
        bk.y0 = (uint32_t)y0, bk.z0 = (uint32_t)z0;
        bk.x1 = (uint32_t)x1, bk.y1 = (uint32_t)y1, bk.z1 = (uint32_t)z1;
        s->host_types = std::move(types);
        s->bulk_chunk = default_chunk(s);
        // The adjoint's sweep: the default shape and chunk, every tile checking its cell types
        // (the adjoint's types leave out cells that a full tile of the forward sweep holds).
        std::vector<int4> plain;
        if ((rc = tile_list(s, 0, s->bulk_chunk, false, plain))) return rc;
        const int4 *d_plain;
        if ((rc = upload(s, plain.data(), plain.size(), &d_plain))) return rc;
        s->plain_tiles = d_plain;
        s->plain_count = (uint32_t)plain.size();
        if ((rc = set_up(s))) return rc;
        if ((rc = use_shape(s, 0, s->bulk_chunk))) return rc;
    }

    // Special rows with 32-bit pitched indices.
    const uint64_t K = L->special_count;
    s->specials = K, s->links = L->link_count, s->states = L->state_count;
    g.specials = (uint32_t)K;
    const float *fp;
    const uint8_t *u8;
    {
        std::vector<uint32_t> special(K), state_start(K + 1);
        uint64_t slots = 0;
        for (uint64_t k = 0; k < K; ++k) {
            special[k] = pitched(s, (uint64_t)L->special[k]);
            slots = std::max<uint64_t>(slots, L->link_start[k + 1] - L->link_start[k]);
        }
        for (uint64_t k = 0; k <= K; ++k) state_start[k] = (uint32_t)L->state_start[k];
        if (slots > 18) return fail(s, FDTD_EINVAL, "a special cell has more than 18 links");
        // The links, slot-major (ELL): slot l of row k at l * K + k.
        std::vector<uint8_t> count(K), direction(slots * K, 0);
        std::vector<float> weight(slots * K, 0.0f);
        for (uint64_t k = 0; k < K; ++k) {
            const uint64_t l0 = L->link_start[k], l1 = L->link_start[k + 1];
            count[k] = (uint8_t)(l1 - l0);
            for (uint64_t l = l0; l < l1; ++l) {
                direction[(l - l0) * K + k] = L->link_direction[l];
                weight[(l - l0) * K + k] = L->link_weight[l];
            }
        }
        g.link_slots = (uint32_t)slots;
        s->link_slots = (uint32_t)slots;
        const uint32_t *p;
        if ((rc = upload(s, special.data(), K, &p))) return rc;
        g.special = p;
        if ((rc = upload(s, state_start.data(), K + 1, &p))) return rc;
        g.state_start = p;
        if ((rc = upload(s, count.data(), K, &u8))) return rc;
        g.link_count = u8;
        if ((rc = upload(s, direction.data(), direction.size(), &u8))) return rc;
        g.link_direction = u8;
        if ((rc = upload(s, weight.data(), weight.size(), &fp))) return rc;
        g.link_weight = fp;
        // Every row's links axial, in the directions' order, of the axial weight: masks.
        bool axial_rows = K > 0 && L->weight_count >= 1;
        std::vector<uint8_t> mask(K, 0);
        for (uint64_t k = 0; k < K && axial_rows; ++k) {
            int last = -1;
            for (uint64_t l = L->link_start[k]; l < L->link_start[k + 1] && axial_rows; ++l) {
                const int d = L->link_direction[l];
                axial_rows = d < 6 && d > last && std::memcmp(&L->link_weight[l], &L->weights[0], sizeof(float)) == 0;
                last = d;
                mask[k] |= (uint8_t)(1u << (d & 7));
            }
        }
        g.link_mask = nullptr;
        g.link_axial = L->weights[0];
        if (axial_rows) {
            if ((rc = upload(s, mask.data(), K, &u8))) return rc;
            g.link_mask = u8;
        }
    }
    if ((rc = upload(s, L->coef_a, K, &fp))) return rc;
    g.coef_a = fp;
    if ((rc = upload(s, L->coef_b, K, &fp))) return rc;
    g.coef_b = fp;
    if ((rc = upload(s, L->coef_inv, K, &fp))) return rc;
    g.coef_inv = fp;
    if ((rc = upload(s, L->source, K, &fp))) return rc;
    g.source = fp;
    if (s->precision == FDTD_FP32_COMPENSATED) {
        if ((rc = upload(s, row_residual.data(), K, &fp))) return rc;
        g.row_residual = fp;
    }
    {
        // Each state's branch coefficients gathered per state, as run() gathers them
        // (fdtd.hpp:797-805).
        const uint64_t S = L->state_count;
        s->state_branch.assign(L->state_branch, L->state_branch + S);
        s->branches = L->branch_count;
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
    if (Lc) {
        std::vector<uint32_t> cells(Lc);
        for (uint64_t c = 0; c < Lc; ++c) cells[c] = pitched(s, (uint64_t)L->layer_cells[c]);
        // Which of each layer cell's lower neighbours are in the layer too (their face is theirs).
        std::vector<uint8_t> below(Lc, 0);
        const uint64_t strides[3] = {1, nx, nx * ny};
        for (uint64_t c = 0; c < Lc; ++c)
            for (int axis = 0; axis < 3; ++axis)
                if (L->types[(uint64_t)L->layer_cells[c] - strides[axis]] == kLayer) below[c] |= (uint8_t)(1u << axis);
        s->layer_cells = cells;
        const uint32_t *p;
        if ((rc = upload(s, cells.data(), Lc, &p))) return rc;
        g.layer_cells = p;
        if ((rc = upload(s, below.data(), Lc, &u8))) return rc;
        g.layer_below = u8;
        const uint64_t len[3] = {nx + 1, ny + 1, nz + 1};
        for (int axis = 0; axis < 3; ++axis) {
            std::vector<float4> packed(len[axis]);
            for (uint64_t x = 0; x < len[axis]; ++x)
                packed[x] = make_float4(L->keep[2 * axis][x], L->push[2 * axis][x], L->keep[2 * axis + 1][x],
                                        L->push[2 * axis + 1][x]);
            const float4 *p4;
            if ((rc = upload(s, packed.data(), len[axis], &p4))) return rc;
            g.layer_coef[axis] = p4;
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
    {
        std::vector<uint32_t> start(P + 1), cells(pc);
        for (uint64_t p = 0; p <= P; ++p) start[p] = (uint32_t)L->probe_start[p];
        for (uint64_t k = 0; k < pc; ++k) cells[k] = pitched(s, L->probe_cells[k]);
        const uint32_t *p32;
        if ((rc = upload(s, start.data(), P + 1, &p32))) return rc;
        g.probe_start = p32;
        if ((rc = upload(s, cells.data(), pc, &p32))) return rc;
        g.probe_cells = p32;
        const double *pd;
        if ((rc = upload(s, L->probe_weights, pc, &pd))) return rc;
        g.probe_weights = pd;
    }
    return FDTD_OK;
}

void release(fdtd_solver *s) {
    if (!s) return;
    int current = 0;
    cudaGetDevice(&current);
    cudaSetDevice(s->device);
    for (cudaStream_t stream : {s->stream, s->side, s->layer_stream})
        if (stream) cudaStreamSynchronize(stream);
    for (cudaGraphExec_t g : s->graph)
        if (g) cudaGraphExecDestroy(g);
    for (cudaGraphExec_t g : s->tape_graph)
        if (g) cudaGraphExecDestroy(g);
    for (auto &row : s->grad_graph)
        for (cudaGraphExec_t g : row)
            if (g) cudaGraphExecDestroy(g);
    for (const auto &b : s->work) cudaFree(b.p);
    for (cudaEvent_t e : s->timing_events) cudaEventDestroy(e);
    for (void *p : s->allocations) cudaFree(p);
    if (s->stage_signal) cudaFreeHost(s->stage_signal);
    if (s->stage_out) cudaFreeHost(s->stage_out);
    for (cudaEvent_t e : s->joined)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t stream : {s->layer_stream, s->side, s->stream})
        if (stream) cudaStreamDestroy(stream);
    cudaSetDevice(current);
}

// ---------------------------------------------------------------------------------------------
// The adjoint (see fdtd_adjoint.cuh)
// ---------------------------------------------------------------------------------------------

template <typename V>
int download(fdtd_solver *s, const V *device, size_t count, std::vector<V> &host) {
    host.resize(count);
    if (count) CUDA_TRY(s, cudaMemcpy(host.data(), device, count * sizeof(V), cudaMemcpyDeviceToHost));
    return FDTD_OK;
}

// The adjoint's tables on the host: the readers of each special row's cell (the transposed links)
// and the interior cells next to special rows with their corrections.
struct AdjointLists {
    std::vector<uint32_t> reader_start, reader_index, cells, starts, rows;
    std::vector<uint32_t> masks;        // each corrected cell's special neighbours (bit d: direction d)
    std::vector<uint8_t> types;         // the sweep's cell types
    std::vector<float> scales;          // with a speed field: each corrected cell's scale
    std::vector<uint32_t> special_read_start, corrected_read_start, read_probe;  // the probes' terms by cell
    std::vector<double> read_weight;
    // Each reader's and correction's coefficient as coef_inv[row] x base (row -1: the base alone),
    // so that new coefficients (fdtd_set_coefficients) give new products without a new set-up.
    std::vector<int32_t> reader_row;
    std::vector<double> reader_base, corrected_base;
    std::vector<uint8_t> reader_kind;
    std::vector<double> reader_coef, coefs;
    // The matched layer: rows linking to each layer cell (start, row, coefficient and its base),
    // the probes' terms of each layer cell, each layer cell's interior axial neighbours, and the
    // layer-term masks of the special rows, corrected cells and layer cells (AdjointTables).
    std::vector<uint32_t> layer_from_start, layer_from_row, layer_read_start;
    std::vector<double> layer_from_coef, layer_from_base;
    std::vector<uint8_t> layer_interior, special_layer_mask, corrected_layer_mask, layer_mask;
    std::vector<uint32_t> by_coord, coord_start;  // the layer cells by coordinate, per axis
    // The rows and corrected cells, those that gather no layer terms first (AdjointTables).
    std::vector<uint32_t> special_order, corrected_order;
    uint32_t special_far = 0, corrected_far = 0;
};

// The lists from the handle's own device tables.
//
// With a speed field the interior update scales each row by its own cell's factor s_i, so the
// operator is no longer symmetric: its transpose takes s_j of every reader j. The adjoint of an
// interior cell is then carried as v = s lam, whose reverse step is the forward scaled sweep
// itself: v_i = (2 - total s_i) V_i + s_i axial sum V_j - v+_i, V the level after. What reads or
// feeds an interior cell's adjoint follows from that: a special row gathers axial x v_j from an
// interior reader j (its coefficient a s_j times lam_j), and a corrected cell's terms from special
// rows and probes enter times its own s. Special rows and branch states keep their plain adjoints.
// The 19-point operator is symmetric as the 7-point one is: its readers and corrections reach the
// twelve edge neighbours too, with the diagonal weight.
int adjoint_lists(fdtd_solver *s, AdjointLists &out) {
    const Tables &g = s->tables;
    const uint64_t K = s->specials;
    std::vector<uint32_t> special;
    std::vector<uint8_t> count, direction, types;
    std::vector<float> weight, coef_a, coef_inv;
    int rc;
    if ((rc = download(s, g.special, K, special))) return rc;
    if ((rc = download(s, g.link_count, K, count))) return rc;
    if ((rc = download(s, g.link_direction, (size_t)g.link_slots * K, direction))) return rc;
    if ((rc = download(s, g.link_weight, (size_t)g.link_slots * K, weight))) return rc;
    if ((rc = download(s, g.coef_a, K, coef_a))) return rc;
    if ((rc = download(s, g.coef_inv, K, coef_inv))) return rc;
    if ((rc = download(s, s->types_device, s->n_device, types))) return rc;
    std::vector<float> scale;
    if (s->scaled && (rc = download(s, s->scale_device, s->n_device, scale))) return rc;
    const double axial = (double)s->bulk.axial, diagonal = (double)s->bulk.diagonal;
    const int directions = s->wide ? 18 : 6;
    // The pitched cell one step from cell i along direction d, if it lies in the grid.
    auto neighbour = [&](uint32_t i, int d, uint32_t *j) {
        const int64_t x = (int64_t)(i % s->pitch) + kSteps[d][0];
        const int64_t y = (int64_t)((i / s->pitch) % s->ny) + kSteps[d][1];
        const int64_t z = (int64_t)(i / (s->pitch * s->ny)) + kSteps[d][2];
        if (x < 0 || y < 0 || z < 0 || x >= (int64_t)s->nx || y >= (int64_t)s->ny || z >= (int64_t)s->nz) return false;
        *j = (uint32_t)((int64_t)i + g.offset[d]);
        return true;
    };
    std::unordered_map<uint32_t, uint32_t> row_of;
    row_of.reserve(K * 2);
    for (uint64_t k = 0; k < K; ++k) row_of[special[k]] = (uint32_t)k;
    // Readers of each special row's cell: the row itself, its interior neighbours, the special
    // rows linking to it; and the interior cells special rows link to.
    struct Reader {
        uint64_t index;  // | kind << 63
        int32_t row;     // the reading row whose coef_inv multiplies `base`, or -1
        double base;
    };
    std::vector<std::vector<Reader>> readers(K);
    std::unordered_map<uint32_t, std::vector<std::pair<uint32_t, double>>> corrected;  // (row, base)
    const uint64_t kind_bit = 1ull << 63;
    // The matched layer's cells by pitched index, and the rows linking to each.
    const uint64_t Lc = s->layers;
    std::unordered_map<uint32_t, uint32_t> layer_of;
    layer_of.reserve(Lc * 2);
    for (uint64_t c = 0; c < Lc; ++c) layer_of[s->layer_cells[c]] = (uint32_t)c;
    std::vector<std::vector<std::pair<uint32_t, double>>> layer_from(Lc);  // (row, base)
    // A cell's layer-term mask: bit d for an axial neighbour d in the layer, bit 6 for itself.
    auto layer_mask = [&](uint32_t i) {
        uint32_t mask = types[i] == kLayer ? 64u : 0u;
        for (int d = 0; d < 6; ++d) {
            uint32_t j;
            if (neighbour(i, d, &j) && types[j] == kLayer) mask |= 1u << d;
        }
        return (uint8_t)mask;
    };
    // Interior cells next to the layer read its terms: formed whole by correct_kernel.
    for (uint64_t c = 0; c < Lc; ++c)
        for (int d = 0; d < 6; ++d) {
            uint32_t j;
            if (neighbour(s->layer_cells[c], d, &j) && types[j] == kInterior) corrected[j];
        }
    for (uint64_t k = 0; k < K; ++k) {
        const uint32_t i = special[k];
        readers[k].push_back({kind_bit | k, (int32_t)k, (double)coef_a[k]});
        for (int d = 0; d < directions; ++d) {
            uint32_t j;
            if (neighbour(i, d, &j) && types[j] == kInterior) {
                readers[k].push_back({j, -1, d < 6 ? axial : diagonal});
                corrected[j];  // an interior cell next to a special row: formed by correct_kernel
            }
        }
        for (uint32_t l = 0; l < count[k]; ++l) {
            const uint64_t at = (uint64_t)l * K + k;
            const uint32_t j = (uint32_t)((int64_t)i + g.offset[direction[at]]);
            auto it = row_of.find(j);
            if (it != row_of.end()) {
                readers[it->second].push_back({kind_bit | k, (int32_t)k, (double)weight[at]});
            } else if (types[j] == kInterior) {
                corrected[j].push_back({(uint32_t)k, (double)weight[at]});
            } else if (types[j] == kLayer) {
                layer_from[layer_of.at(j)].push_back({(uint32_t)k, (double)weight[at]});
            } else {
                return fail(s, FDTD_EINVAL, "a special row links to a cell that holds no air");
            }
        }
    }
    out.reader_start.assign(K + 1, 0);
    for (uint64_t k = 0; k < K; ++k) {
        for (const Reader &r : readers[k]) {
            out.reader_index.push_back((uint32_t)(r.index & ~kind_bit));
            out.reader_kind.push_back((r.index & kind_bit) ? 1 : 0);
            out.reader_row.push_back(r.row);
            out.reader_base.push_back(r.base);
            out.reader_coef.push_back(r.row >= 0 ? (double)coef_inv[r.row] * r.base : r.base);
        }
        out.reader_start[k + 1] = (uint32_t)out.reader_index.size();
    }
    // The probes' terms grouped by cell, each cell's in the order of the probes and their cells;
    // the interior cells that probes read are formed whole by correct_kernel too.
    std::vector<uint32_t> probe_start, probe_cells;
    std::vector<double> probe_weights;
    if ((rc = download(s, g.probe_start, (size_t)g.probes + 1, probe_start))) return rc;
    if ((rc = download(s, g.probe_cells, (size_t)probe_start[g.probes], probe_cells))) return rc;
    if ((rc = download(s, g.probe_weights, (size_t)probe_start[g.probes], probe_weights))) return rc;
    std::unordered_map<uint32_t, std::vector<std::pair<uint32_t, double>>> probed;  // cell: (probe, weight)
    for (uint32_t p = 0; p < g.probes; ++p)
        for (uint32_t e = probe_start[p]; e < probe_start[p + 1]; ++e) {
            const uint32_t cell = probe_cells[e];
            if (row_of.count(cell) || types[cell] == kInterior || types[cell] == kLayer)
                probed[cell].push_back({p, probe_weights[e]});
            if (types[cell] == kInterior) corrected[cell];
        }
    auto read_terms = [&](uint32_t cell, double factor) {
        auto it = probed.find(cell);
        if (it != probed.end())
            for (const auto &[p, w] : it->second) out.read_probe.push_back(p), out.read_weight.push_back(w * factor);
        return (uint32_t)out.read_probe.size();
    };
    out.special_read_start.assign(1, 0);
    for (uint64_t k = 0; k < K; ++k) out.special_read_start.push_back(read_terms(special[k], 1.0));
    out.special_layer_mask.resize(K);
    for (uint64_t k = 0; k < K; ++k) out.special_layer_mask[k] = Lc ? layer_mask(special[k]) : 0;
    out.corrected_read_start.assign(1, out.special_read_start.back());
    out.starts.assign(1, 0);
    out.types = types;
    for (auto &[cell, list] : corrected) {
        const double factor = s->scaled ? (double)scale[cell] : 1.0;
        out.cells.push_back(cell);
        if (s->scaled) out.scales.push_back(scale[cell]);
        out.corrected_read_start.push_back(read_terms(cell, factor));
        out.types[cell] = kSpecial;  // left to correct_kernel
        // The neighbours left out of its stencil: special rows, and layer cells (whose updates read
        // it through their faces: the layer's terms). (An interior cell's neighbours all lie in
        // the grid.)
        uint32_t mask = 0;
        for (int d = 0; d < directions; ++d) {
            const uint32_t j = (uint32_t)((int64_t)cell + g.offset[d]);
            if (row_of.count(j) || types[j] == kLayer) mask |= 1u << d;
        }
        out.masks.push_back(mask);
        out.corrected_layer_mask.push_back(Lc ? layer_mask(cell) : 0);
        for (const auto &[r, base] : list) {
            out.rows.push_back(r);
            out.corrected_base.push_back(base * factor);
            out.coefs.push_back((double)coef_inv[r] * (base * factor));
        }
        out.starts.push_back((uint32_t)out.rows.size());
    }
    // The layer cells: the rows linking to each, the probes' terms, the interior neighbours whose
    // adjoints they read, and their layer-term masks.
    out.layer_from_start.assign(1, 0);
    out.layer_read_start.assign(1, out.corrected_read_start.back());
    for (uint64_t c = 0; c < Lc; ++c) {
        const uint32_t i = s->layer_cells[c];
        for (const auto &[r, base] : layer_from[c]) {
            out.layer_from_row.push_back(r);
            out.layer_from_base.push_back(base);
            out.layer_from_coef.push_back((double)coef_inv[r] * base);
        }
        out.layer_from_start.push_back((uint32_t)out.layer_from_row.size());
        out.layer_read_start.push_back(read_terms(i, 1.0));
        uint8_t inner = 0;
        for (int d = 0; d < 6; ++d) {
            uint32_t j;
            if (neighbour(i, d, &j) && types[j] == kInterior) inner |= (uint8_t)(1u << d);
        }
        out.layer_interior.push_back(inner);
        // (bit 7: rows link to the cell or probes read it — most layer cells have neither)
        const size_t n_from = out.layer_from_start.size(), n_read = out.layer_read_start.size();
        const bool listed = out.layer_from_start[n_from - 1] > out.layer_from_start[n_from - 2] ||
                            out.layer_read_start[n_read - 1] > out.layer_read_start[n_read - 2];
        out.layer_mask.push_back((uint8_t)(layer_mask(i) | (listed ? 128u : 0u)));
    }
    // The rows and the corrected cells, those whose updates gather none of the layer's terms
    // first, each part in its own order.
    for (int near = 0; near < 2; ++near) {
        for (uint64_t k = 0; k < K; ++k)
            if ((out.special_layer_mask[k] != 0) == (near != 0)) out.special_order.push_back((uint32_t)k);
        for (uint64_t c = 0; c < out.cells.size(); ++c)
            if ((out.corrected_layer_mask[c] != 0) == (near != 0)) out.corrected_order.push_back((uint32_t)c);
        if (!near) out.special_far = (uint32_t)out.special_order.size(), out.corrected_far = (uint32_t)out.corrected_order.size();
    }
    // Per axis, the layer cells sorted by their coordinate along it (counting sort, stable), and
    // where each coordinate's cells begin: coordinates 0 .. n_a - 1 of axis a follow axis a - 1's.
    if (Lc) {
        const uint64_t len[3] = {s->nx, s->ny, s->nz};
        out.coord_start.assign(1, 0);
        for (int a = 0; a < 3; ++a) {
            std::vector<uint32_t> count(len[a] + 1, 0);
            std::vector<uint32_t> coord(Lc);
            for (uint64_t c = 0; c < Lc; ++c) {
                const uint64_t i = s->layer_cells[c], z = i / (s->pitch * s->ny), r = i - z * s->pitch * s->ny;
                const uint64_t y = r / s->pitch, at[3] = {r - y * s->pitch, y, z};
                coord[c] = (uint32_t)at[a];
                ++count[at[a] + 1];
            }
            for (uint64_t x = 0; x < len[a]; ++x) count[x + 1] += count[x];
            const size_t base = out.by_coord.size();
            out.by_coord.resize(base + Lc);
            std::vector<uint32_t> next(count.begin(), count.end() - 1);
            for (uint64_t c = 0; c < Lc; ++c) out.by_coord[base + next[coord[c]]++] = (uint32_t)c;
            for (uint64_t x = 0; x < len[a]; ++x) out.coord_start.push_back((uint32_t)(base + count[x + 1]));
        }
    }
    return FDTD_OK;
}

// A host array copied into device memory from `pool` (pool.take(bytes, &p, zero) gives the
// memory), in order on the handle's stream (the host array is staged before the call returns).
template <class Pool, typename V>
int place(fdtd_solver *s, Pool &pool, const std::vector<V> &host, const V **out) {
    *out = nullptr;
    if (host.empty()) return FDTD_OK;
    void *p;
    int rc;
    if ((rc = pool.take(host.size() * sizeof(V), &p, false))) return rc;
    CUDA_TRY(s, cudaMemcpyAsync(p, host.data(), host.size() * sizeof(V), cudaMemcpyHostToDevice, s->stream));
    *out = static_cast<const V *>(p);
    return FDTD_OK;
}

// The adjoint's device state from its lists, in memory from `pool`.
template <class Pool>
int place_adjoint(fdtd_solver *s, const AdjointLists &l, Pool &pool, AdjointState &a) {
    const Tables &g = s->tables;
    const uint64_t K = s->specials, S = s->states;
    const size_t e = s->precision == FDTD_FP64 ? 8 : 4;
    AdjointTables &t = a.t;
    t.specials = (uint32_t)K, t.states = (uint32_t)S;
    t.special = g.special, t.state_start = g.state_start;
    t.state_weight = g.state_weight, t.state_now = g.state_now, t.state_before = g.state_before, t.state_gain = g.state_gain;
    t.coef_b = g.coef_b, t.coef_inv = g.coef_inv;
    t.axial = s->bulk.axial;
    t.centre = s->bulk.centre;
    t.total = s->bulk.total;
    t.diagonal = s->wide ? s->bulk.diagonal : 0.0f;
    t.wide = s->wide ? 1 : 0;
    for (int d = 0; d < 18; ++d) t.offset[d] = g.offset[d];
    t.corrected = (uint32_t)l.cells.size();
    int rc;
    if ((rc = place(s, pool, l.reader_start, &t.reader_start))) return rc;
    if ((rc = place(s, pool, l.reader_index, &t.reader_index))) return rc;
    if ((rc = place(s, pool, l.reader_kind, &t.reader_kind))) return rc;
    if ((rc = place(s, pool, l.reader_coef, &t.reader_coef))) return rc;
    if ((rc = place(s, pool, l.cells, &t.corrected_cell))) return rc;
    if ((rc = place(s, pool, l.starts, &t.corrected_start))) return rc;
    if ((rc = place(s, pool, l.rows, &t.corrected_row))) return rc;
    if ((rc = place(s, pool, l.masks, &t.corrected_mask))) return rc;
    if ((rc = place(s, pool, l.scales, &t.corrected_scale))) return rc;
    const uint8_t *sweep_types;
    if ((rc = place(s, pool, l.types, &sweep_types))) return rc;
    if ((rc = place(s, pool, l.coefs, &t.corrected_coef))) return rc;
    if ((rc = place(s, pool, l.special_read_start, &t.special_read_start))) return rc;
    if ((rc = place(s, pool, l.corrected_read_start, &t.corrected_read_start))) return rc;
    if ((rc = place(s, pool, l.read_probe, &t.read_probe))) return rc;
    if ((rc = place(s, pool, l.read_weight, &t.read_weight))) return rc;
    // The matched layer: the forward's cells and tables, the lists, the masks; its carried values
    // and the hats (six pitched levels) are the adjoint's own.
    t.layers = (uint32_t)s->layers;
    t.layer_cells = g.layer_cells;
    for (int axis = 0; axis < 3; ++axis) t.layer_coef[axis] = g.layer_coef[axis];
    t.layer_scale = g.layer_scale;
    t.pitch = g.pitch, t.plane = g.plane;
    t.by_plane = g.by_plane, t.by_pitch = g.by_pitch;
    t.cells = s->n_device;
    if ((rc = place(s, pool, l.special_layer_mask, &t.special_layer_mask))) return rc;
    if ((rc = place(s, pool, l.corrected_layer_mask, &t.corrected_layer_mask))) return rc;
    if ((rc = place(s, pool, l.layer_mask, &t.layer_mask))) return rc;
    if ((rc = place(s, pool, l.layer_from_start, &t.layer_from_start))) return rc;
    if ((rc = place(s, pool, l.layer_from_row, &t.layer_from_row))) return rc;
    if ((rc = place(s, pool, l.layer_from_coef, &t.layer_from_coef))) return rc;
    if ((rc = place(s, pool, l.layer_read_start, &t.layer_read_start))) return rc;
    if ((rc = place(s, pool, l.layer_interior, &t.layer_interior))) return rc;
    if ((rc = place(s, pool, l.special_order, &t.special_order))) return rc;
    if ((rc = place(s, pool, l.corrected_order, &t.corrected_order))) return rc;
    t.special_far = l.special_far, t.corrected_far = l.corrected_far;
    if (s->layers) {
        if ((rc = pool.take(e * kCarried * s->layers, &a.carried, true))) return rc;
        for (int k = 0; k < 2; ++k)
            if ((rc = pool.take(e * kHats * s->n_device, &a.hat[k], true))) return rc;
        if ((rc = pool.take(e * 9 * s->layers, &a.pending, true))) return rc;
        if ((rc = place(s, pool, l.by_coord, &a.by_coord))) return rc;
        if ((rc = place(s, pool, l.coord_start, &a.coord_start))) return rc;
    }
    for (int k = 0; k < 2; ++k) {
        if ((rc = pool.take(e * s->n_device, &a.lam[k], true))) return rc;
        if ((rc = pool.take(e * S, &a.om[k], true))) return rc;
    }
    for (int k = 0; k < 2; ++k)
        if ((rc = pool.take(e * K, &a.tilde[k], true))) return rc;
    if (s->bulk_blocks) {
        const CUtensorMapDataType ft = s->precision == FDTD_FP64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
        for (int k = 0; k < 2; ++k) {
            if ((rc = tensor_map(s, &a.lam_b[k], a.lam[k], ft, (uint32_t)e, kBX, kBY))) return rc;
            if ((rc = tensor_map(s, &a.lam_a[k], a.lam[k], ft, (uint32_t)e, kTX, kTY))) return rc;
        }
        if ((rc = tensor_map(s, &a.map_t, const_cast<uint8_t *>(sweep_types), CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, kTX,
                             kTY)))
            return rc;
        if ((rc = tensor_map(s, &a.map_s, s->scaled ? const_cast<float *>(s->scale_device) : a.lam[0],
                             CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, kTX, kTY)))
            return rc;
    }
    return FDTD_OK;
}

// Device memory the handle owns until fdtd_destroy.
struct Owned {
    fdtd_solver *s;
    int take(size_t bytes, void **out, bool zero) {
        if (zero) return zeros(s, bytes, out);
        *out = nullptr;
        void *p = nullptr;
        CUDA_TRY(s, cudaMalloc(&p, bytes ? bytes : 16));
        s->allocations.push_back(p);
        s->device_bytes += bytes;
        *out = p;
        return FDTD_OK;
    }
};

// The handle's adjoint, set up on first use and kept; every copy and clear has ended on return.
int set_up_adjoint(fdtd_solver *s) {
    if (s->adjoint_ready) return FDTD_OK;
    AdjointLists lists;
    int rc;
    if ((rc = adjoint_lists(s, lists))) return rc;
    Owned owned{s};
    if ((rc = place_adjoint(s, lists, owned, s->adjoint))) return rc;
    CUDA_TRY(s, cudaDeviceSynchronize());  // the clears (default stream) and copies (handle's stream)
    s->adjoint_reader_row = std::move(lists.reader_row);
    s->adjoint_reader_base = std::move(lists.reader_base);
    s->adjoint_corrected_row = std::move(lists.rows);
    s->adjoint_corrected_base = std::move(lists.corrected_base);
    s->adjoint_layer_row = std::move(lists.layer_from_row);
    s->adjoint_layer_base = std::move(lists.layer_from_base);
    s->adjoint_ready = true;
    return FDTD_OK;
}

// fdtd_gradient's workspace on the handle: the blocks of the last call handed out again in order
// while the sizes match, each cleared on the handle's stream; from the first that does not, new
// ones (the graphs over the old ones dropped).
struct Kept {
    fdtd_solver *s;
    size_t next = 0;
    void drop_graphs() {
        for (auto &row : s->grad_graph)
            for (cudaGraphExec_t &g : row)
                if (g) cudaGraphExecDestroy(g), g = nullptr;
    }
    int take(size_t bytes, void **out) {
        *out = nullptr;
        const size_t size = bytes ? bytes : 16;
        if (next < s->work.size() && s->work[next].bytes != size) {
            CUDA_TRY(s, cudaStreamSynchronize(s->stream));
            for (size_t i = next; i < s->work.size(); ++i) cudaFree(s->work[i].p);
            s->work.resize(next);
            drop_graphs();
        }
        if (next == s->work.size()) {
            void *p = nullptr;
            CUDA_TRY(s, cudaMalloc(&p, size));
            s->work.push_back({p, size});
            drop_graphs();
        }
        *out = s->work[next++].p;
        CUDA_TRY(s, cudaMemsetAsync(*out, 0, size, s->stream));
        return FDTD_OK;
    }
};

// A checkpoint of the state between runs: the current and the previous level, the current and
// the previous branch velocities, and with a matched layer its current state (layer_state[1]).
uint64_t checkpoint_bytes(const fdtd_solver *s) {
    const uint64_t e = s->precision == FDTD_FP64 ? 8 : 4;
    uint64_t bytes = 2 * e * s->n_device + 2 * e * s->states;
    if (s->layers) bytes += kLayerSlots * e * s->n_device;
    return bytes;
}

int save_checkpoint(fdtd_solver *s, char *c) {
    const uint64_t e = s->precision == FDTD_FP64 ? 8 : 4, level = e * s->n_device, states = e * s->states;
    CUDA_TRY(s, cudaMemcpyAsync(c, s->u[1], level, cudaMemcpyDeviceToDevice, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(c + level, s->u[0], level, cudaMemcpyDeviceToDevice, s->stream));
    c += 2 * level;
    if (states) {
        CUDA_TRY(s, cudaMemcpyAsync(c, s->w[1], states, cudaMemcpyDeviceToDevice, s->stream));
        CUDA_TRY(s, cudaMemcpyAsync(c + states, s->w[0], states, cudaMemcpyDeviceToDevice, s->stream));
    }
    c += 2 * states;
    if (s->layers) CUDA_TRY(s, cudaMemcpyAsync(c, s->layer_state[1], kLayerSlots * level, cudaMemcpyDeviceToDevice, s->stream));
    return FDTD_OK;
}

int restore_checkpoint(fdtd_solver *s, const char *c) {
    const uint64_t e = s->precision == FDTD_FP64 ? 8 : 4, level = e * s->n_device, states = e * s->states;
    CUDA_TRY(s, cudaMemcpyAsync(s->u[1], c, level, cudaMemcpyDeviceToDevice, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(s->u[0], c + level, level, cudaMemcpyDeviceToDevice, s->stream));
    c += 2 * level;
    if (states) {
        CUDA_TRY(s, cudaMemcpyAsync(s->w[1], c, states, cudaMemcpyDeviceToDevice, s->stream));
        CUDA_TRY(s, cudaMemcpyAsync(s->w[0], c + states, states, cudaMemcpyDeviceToDevice, s->stream));
    }
    c += 2 * states;
    if (s->layers) CUDA_TRY(s, cudaMemcpyAsync(s->layer_state[1], c, kLayerSlots * level, cudaMemcpyDeviceToDevice, s->stream));
    return FDTD_OK;
}

// One word of device memory set in stream order (a captured graph reads it when it runs).
__global__ void set_address_kernel(const void **slot, const void *value) { *slot = value; }

// Whether the handle holds the tape of a run of this drive with these segments: gradient<T> then
// takes the tape's checkpoints or trajectory and recomputes no forward pass of its own.
// (A trajectory holds no matched layer's tables' factors: a gradient in the layer's tables
// recomputes; one along a tangent of the tables needs the tangent's factors on the tape.)
bool holds_tape(const fdtd_solver *s, const float *signal, uint64_t steps, uint64_t segment) {
    if (segment == 0 || segment > steps) segment = steps;
    if (s->tape_traj && s->layers && s->gradient_tables && !s->tangent) return false;
    if (s->tape_traj && s->layers && s->tangent && !s->tape_tangent) return false;
    return s->tape_valid && s->tape_signal.size() == steps && std::min<uint64_t>(s->tape_segment, steps) == segment &&
           std::memcmp(s->tape_signal.data(), signal, sizeof(float) * steps) == 0;
}

// The gradient (fdtd_gradient) with the adjoint state `adj` and scratch from `scratch`
// (scratch.take(bytes, &p): device memory cleared to 0 in order on the handle's stream).
template <typename T, class Pool>
int gradient(fdtd_solver *s, const AdjointState &adj, Pool &scratch, const float *signal, uint64_t steps,
             const double *dloss, uint64_t segment, double *grads[5], bool graphs) {
    const uint64_t K = s->specials, S = s->states, P = s->probes;
    const size_t e = sizeof(T);
    if (segment == 0 || segment > steps) segment = steps;
    const uint64_t segments = (steps + segment - 1) / segment;
    void *p;
    int rc;
    // On the device: the drive, dL/dy, one segment's trajectory, the gradient's sums, and the
    // state at the start of every segment after the first (the checkpoints).
    if ((rc = scratch.take(sizeof(float) * steps, &p))) return rc;
    float *d_signal = static_cast<float *>(p);
    CUDA_TRY(s, cudaMemcpyAsync(d_signal, signal, sizeof(float) * steps, cudaMemcpyHostToDevice, s->stream));
    if ((rc = scratch.take(sizeof(double) * std::max<uint64_t>(1, P) * steps, &p))) return rc;
    double *d_dloss = static_cast<double *>(p);
    if (P) CUDA_TRY(s, cudaMemcpyAsync(d_dloss, dloss, sizeof(double) * P * steps, cudaMemcpyHostToDevice, s->stream));
    if ((rc = scratch.take(e * K * (segment + 2), &p))) return rc;
    T *traj_u = static_cast<T *>(p);
    if ((rc = scratch.take(e * S * (segment + 2), &p))) return rc;
    T *traj_w = static_cast<T *>(p);
    if ((rc = scratch.take(sizeof(double) * std::max<uint64_t>(1, P) * segment, &p))) return rc;
    double *d_out = static_cast<double *>(p);
    // The drive and dL/dy of the segment at hand.
    if ((rc = scratch.take(sizeof(float) * segment, &p))) return rc;
    float *seg_signal = static_cast<float *>(p);
    if ((rc = scratch.take(sizeof(double) * std::max<uint64_t>(1, P) * segment, &p))) return rc;
    double *seg_dloss = static_cast<double *>(p);
    double *g[5];
    const uint64_t g_len[5] = {K, K, S, S, S};  // coef_b, coef_inv, now, before, gain
    for (int k = 0; k < 5; ++k) {
        if ((rc = scratch.take(sizeof(double) * g_len[k], &p))) return rc;
        g[k] = static_cast<double *>(p);
    }
    const uint64_t level_bytes = e * s->n_device, state_bytes = e * S;
    // The matched layer: its factors of each step of a segment, and its gradient's sums per cell.
    const uint64_t Lc = s->layers;
    const bool tangent = Lc && s->tangent;  // along a tangent of the tables, in place of the tables
    const bool tables = Lc && s->gradient_tables && !tangent;
    T *traj_layer = nullptr;
    double *g_layer = nullptr, *table_sums = nullptr;
    const uint64_t coords = s->nx + s->ny + s->nz;
    if (tables) {
        if ((rc = scratch.take(e * kLayerFactors * Lc * segment, &p))) return rc;
        traj_layer = static_cast<T *>(p);
        if ((rc = scratch.take(sizeof(double) * kLayerFactors * Lc, &p))) return rc;
        g_layer = static_cast<double *>(p);
        if ((rc = scratch.take(sizeof(double) * 6 * coords, &p))) return rc;
        table_sums = static_cast<double *>(p);
    }
    // The forward pass from rest, keeping checkpoints[m] = the state at the start of segment m+1;
    // or, when the handle holds the tape of a run of this drive with these segments, its states.
    const bool taped = holds_tape(s, signal, steps, segment);
    const bool trajectory = taped && s->tape_traj;  // the tape holds every level: nothing to recompute
    // Along a tangent: one segment's factors (unless the tape holds every step's), each cell's sum
    // over the steps, the sums' partial and whole totals, and the device word that holds where the
    // factors of a segment start (a captured reverse step reads it).
    const uint64_t Tf = s->tangent_factors;
    T *traj_tan = nullptr;
    double *tan_acc = nullptr, *tan_parts = nullptr;
    const T **tan_base = nullptr;
    const uint32_t tan_blocks = (uint32_t)std::min<uint64_t>(256, std::max<uint64_t>(1, (Lc + kBlock - 1) / kBlock));
    if (tangent) {
        if (!trajectory) {
            if ((rc = scratch.take(e * Tf * segment, &p))) return rc;
            traj_tan = static_cast<T *>(p);
        }
        if ((rc = scratch.take(sizeof(double) * Lc, &p))) return rc;
        tan_acc = static_cast<double *>(p);
        if ((rc = scratch.take(sizeof(double) * (tan_blocks + 1), &p))) return rc;
        tan_parts = static_cast<double *>(p);
        if ((rc = scratch.take(sizeof(void *), &p))) return rc;
        tan_base = static_cast<const T **>(p);
    }
    std::vector<char *> checkpoints;
    if (taped && !trajectory)
        for (uint64_t k = 0; k + 1 < segments; ++k) checkpoints.push_back(static_cast<char *>(s->tape_checkpoints[k]));
    else if (!taped && (rc = fdtd_reset(s)) != FDTD_OK)
        return rc;
    for (uint64_t k = 0; !taped && k + 1 < segments; ++k) {
        if ((rc = dispatch(s, d_signal + k * segment, segment, d_out, segment)) != FDTD_OK) return rc;
        settle(s, segment);
        if ((rc = scratch.take(checkpoint_bytes(s), &p))) return rc;
        checkpoints.push_back(static_cast<char *>(p));
        if ((rc = save_checkpoint(s, checkpoints.back())) != FDTD_OK) return rc;
    }
    // The adjoint levels beyond the end, and their L~, are at rest; the sums start at 0.
    for (int k = 0; k < 2; ++k) {
        CUDA_TRY(s, cudaMemsetAsync(adj.lam[k], 0, level_bytes, s->stream));
        if (S) CUDA_TRY(s, cudaMemsetAsync(adj.om[k], 0, state_bytes, s->stream));
        if (K) CUDA_TRY(s, cudaMemsetAsync(adj.tilde[k], 0, sizeof(T) * K, s->stream));
    }
    // (The layer's hats of the first reverse step are those of rest: zero.)
    if (Lc) {
        CUDA_TRY(s, cudaMemsetAsync(adj.carried, 0, e * kCarried * Lc, s->stream));
        for (int k = 0; k < 2; ++k) CUDA_TRY(s, cudaMemsetAsync(adj.hat[k], 0, e * kHats * s->n_device, s->stream));
    }
    AdjointTables t = adj.t;
    t.tangent_axes = s->tables.tangent_axes, t.tangent_start = s->tables.tangent_start;
    const uint32_t row_blocks = (uint32_t)((std::max<uint64_t>(std::max<uint64_t>(K, S), 1) + kBlock - 1) / kBlock);
    const uint32_t layer_blocks = (uint32_t)((Lc + kBlock - 1) / kBlock);
    auto blocks_of = [](uint32_t count) { return (count + kBlock - 1) / kBlock; };
    // (Without a layer every row and cell is far from it.)
    const RowsPart far{0, t.special_far, blocks_of(t.special_far), 0, t.corrected_far, blocks_of(t.corrected_far), 0};
    const RowsPart near{t.special_far, (uint32_t)K, blocks_of((uint32_t)K - t.special_far),
                        t.corrected_far, t.corrected, blocks_of(t.corrected - t.corrected_far), layer_blocks};
    // Each launch's blocks, at most the handle's count an SM (fdtd_set_adjoint_launch; 0: a block
    // for every 128 items).
    auto capped = [&](uint32_t blocks, int per_sm) {
        return per_sm > 0 ? std::min<uint32_t>(blocks, (uint32_t)(s->sms * per_sm)) : blocks;
    };
    const uint32_t far_grid = capped(far.blocks(), s->adjoint_far_per_sm);
    const uint32_t near_grid = capped(near.blocks(), s->adjoint_near_per_sm);
    const uint32_t smem = s->scaled ? Stage<T, true>::smem : Stage<T, false>::smem;
    int x = 0;  // lam[x], om[x]: level n+1; lam[1-x], om[1-x]: level n+2, then level n
    // A segment's recomputation (the dispatch of its steps, recording the special rows), and its
    // reverse steps.
    auto recompute = [&](uint64_t count) -> int {
        s->record_u = traj_u, s->record_w = traj_w, s->record_offset = 2, s->record_probes = false;
        s->record_layer = tables ? traj_layer : nullptr;
        s->record_tangent = tangent ? traj_tan : nullptr;
        const int r = dispatch(s, seg_signal, count, d_out, segment);
        s->record_u = s->record_w = s->record_layer = s->record_tangent = nullptr, s->record_probes = true;
        return r;
    };
    auto reverse = [&](uint64_t count) -> int {
        int xx = x;
        for (uint64_t m = count; m-- > 0;) {
            T *lam_next = static_cast<T *>(adj.lam[xx]), *lam_out = static_cast<T *>(adj.lam[1 - xx]);
            T *om_next = static_cast<T *>(adj.om[xx]), *om_out = static_cast<T *>(adj.om[1 - xx]);
            // The sweep of the interior on the handle's stream; beside it, in one launch on the side
            // stream, the special rows (with their L~ of level n for the next step) and the cells
            // that special rows or probes read (correct_kernel's): all write disjoint cells, and
            // each step starts when both streams have ended the one before.
            const T *tilde = static_cast<const T *>(adj.tilde[xx]);
            T *tilde_out = static_cast<T *>(adj.tilde[1 - xx]);
            CUDA_TRY(s, cudaEventRecord(s->joined[0], s->stream));
            CUDA_TRY(s, cudaStreamWaitEvent(s->side, s->joined[0], 0));
            if (layer_blocks) CUDA_TRY(s, cudaStreamWaitEvent(s->layer_stream, s->joined[0], 0));
            // The layer's hats of step m (formed in the step before, or zero), and where the layer
            // cells put those of step m - 1: the other buffer, with the tables' factors of step
            // m - 1 of this segment, or (m = 0) the values that wait for the segment before.
            T *hat = static_cast<T *>(adj.hat[xx]);
            LayerNext<T> next{static_cast<T *>(adj.hat[1 - xx]), static_cast<T *>(adj.carried), nullptr, nullptr,
                              tables ? g_layer : nullptr};
            if (tables) {
                if (m > 0) next.traj = traj_layer + (m - 1) * kLayerFactors * Lc;
                else next.pending = static_cast<T *>(adj.pending);
            }
            if (tangent) {
                next.tangent_base = tan_base;
                if (m > 0) next.tangent_offset = (m - 1) * Tf;
                else next.pending = static_cast<T *>(adj.pending);
            }
            // The rows and corrected cells far from the layer on the side stream; on the layer's
            // stream (the highest priority) the rows and cells that gather the layer's hats and
            // the layer's own cells.
            if (far.blocks())
                rows_adjoint_kernel<T><<<far_grid, kBlock, 0, s->side>>>(
                    t, far, lam_next, om_next, tilde, hat, lam_out, om_out, traj_u, traj_w, (uint32_t)m, g[1], g[0],
                    g[2], g[3], g[4], tilde_out, seg_dloss, segment, m, next);
            if (layer_blocks) {
                rows_adjoint_kernel<T><<<near_grid, kBlock, 0, s->layer_stream>>>(t, near, lam_next, om_next, tilde, hat, lam_out, om_out,
                                                            traj_u, traj_w, (uint32_t)m, g[1], g[0], g[2], g[3], g[4],
                                                            tilde_out, seg_dloss, segment, m, next);
                CUDA_TRY(s, cudaEventRecord(s->joined[2], s->layer_stream));
            }
            CUDA_TRY(s, cudaEventRecord(s->joined[1], s->side));
            if (s->bulk_blocks) {
                // The forward sweep of the grid's own kind (with a speed field it steps v = s lam).
                BulkArgs args = s->bulk;
                args.a = lam_out;
                args.tile_list = s->plain_tiles;
                args.tiles = s->plain_count;
                const uint32_t blocks = s->plain_count;
                const CUtensorMap &mb = adj.lam_b[xx], &ma = adj.lam_a[1 - xx];
                if (s->wide && s->scaled)
                    bulk_kernel<T, true, true><<<blocks, kBlock, smem, s->stream>>>(mb, ma, adj.map_t, adj.map_s, args);
                else if (s->wide)
                    bulk_kernel<T, true, false><<<blocks, kBlock, smem, s->stream>>>(mb, ma, adj.map_t, adj.map_s, args);
                else if (s->scaled)
                    bulk_kernel<T, false, true, false, Shape7><<<blocks, Shape7::THREADS, smem, s->stream>>>(
                        mb, ma, adj.map_t, adj.map_s, args);
                else
                    bulk_kernel<T, false, false, false, Shape7><<<blocks, Shape7::THREADS, smem, s->stream>>>(
                        mb, ma, adj.map_t, adj.map_s, args);
            }
            CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->joined[1], 0));
            if (layer_blocks) CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->joined[2], 0));
            xx = 1 - xx;
        }
        CUDA_TRY(s, cudaGetLastError());
        return FDTD_OK;
    };
    // With `graphs` (a kept workspace, whose blocks stay put), a full segment's recomputation and
    // reverse steps are captured once as graphs and replayed: on the small grids of a fit, a step's
    // launches and event records and waits take more host time than the step takes on the device.
    if (graphs && s->graph_segment != segment) {
        Kept{s}.drop_graphs();
        s->graph_segment = segment;
    }
    auto run = [&](int which, int key, auto &&body, uint64_t count) -> int {
        if (!graphs || count != segment || segments == 1) return body(count);
        cudaGraphExec_t &exec = s->grad_graph[which][key];
        if (!exec) {
            const bool timing = s->timing;
            s->timing = false;  // no timing events inside a graph
            cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
            const int r = e == cudaSuccess ? body(count) : FDTD_OK;
            s->timing = timing;
            if (e != cudaSuccess) return cuda_fail(s, e, "cudaStreamBeginCapture");
            cudaGraph_t graph = nullptr;
            e = cudaStreamEndCapture(s->stream, &graph);
            if (r != FDTD_OK) {
                if (graph) cudaGraphDestroy(graph);
                return r;
            }
            if (e != cudaSuccess) return cuda_fail(s, e, "cudaStreamEndCapture");
            e = cudaGraphInstantiateWithFlags(&exec, graph, cudaGraphInstantiateFlagUseNodePriority);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return cuda_fail(s, e, "cudaGraphInstantiate");
        }
        CUDA_TRY(s, cudaGraphLaunch(exec, s->stream));
        return FDTD_OK;
    };
    // Along a tangent: each cell's products of a segment into its double sum.
    auto flush_tangent = [&]() {
        layer_tangent_flush_kernel<T><<<layer_blocks, kBlock, 0, s->stream>>>((uint32_t)Lc, static_cast<T *>(adj.carried),
                                                                              tan_acc);
    };
    for (uint64_t k = segments; k-- > 0;) {
        const uint64_t s0 = k * segment, s1 = std::min(steps, s0 + segment), count = s1 - s0;
        if (tangent) {
            // Where the segment's factors start; and the products of its last step, whose Q^, L^,
            // H^ the segment after left waiting.
            const T *base = trajectory ? static_cast<const T *>(s->tape_t) + s0 * Tf : traj_tan;
            set_address_kernel<<<1, 1, 0, s->stream>>>(reinterpret_cast<const void **>(tan_base), base);
            CUDA_TRY(s, cudaGetLastError());
        }
        if (trajectory) {
            if (tangent && k + 1 < segments) {
                layer_pending_tangent_kernel<T><<<layer_blocks, kBlock, 0, s->stream>>>(
                    t, static_cast<const T *>(adj.pending), static_cast<const T *>(s->tape_t) + (s0 + count - 1) * Tf,
                    tan_acc);
                CUDA_TRY(s, cudaGetLastError());
            }
            // The segment's levels s0 .. s1+1 from the tape, into the segment's trajectory buffers.
            CUDA_TRY(s, cudaMemcpyAsync(traj_u, static_cast<const T *>(s->tape_u) + s0 * K, e * K * (count + 2),
                                        cudaMemcpyDeviceToDevice, s->stream));
            if (S)
                CUDA_TRY(s, cudaMemcpyAsync(traj_w, static_cast<const T *>(s->tape_w) + s0 * S, e * S * (count + 2),
                                            cudaMemcpyDeviceToDevice, s->stream));
            if (P)
                CUDA_TRY(s, cudaMemcpy2DAsync(seg_dloss, sizeof(double) * segment, d_dloss + s0, sizeof(double) * steps,
                                              sizeof(double) * count, P, cudaMemcpyDeviceToDevice, s->stream));
            if ((rc = run(1, x, reverse, count)) != FDTD_OK) return rc;
            if (tangent) flush_tangent();
            if (count & 1) x = 1 - x;
            continue;
        }
        // Recompute the segment from its start, recording each level of the special rows.
        if (k == 0) {
            if ((rc = fdtd_reset(s)) != FDTD_OK) return rc;
        } else if ((rc = restore_checkpoint(s, checkpoints[k - 1])) != FDTD_OK) {
            return rc;
        }
        // Level 0 is the segment's previous level, level 1 its current one, level l + 1 the one
        // after the segment's step l (recorded by the dispatch).
        record_kernel<T><<<row_blocks, kBlock, 0, s->stream>>>(t, static_cast<const T *>(s->u[0]),
                                                               static_cast<const T *>(s->w[0]), traj_u, traj_w);
        record_kernel<T><<<row_blocks, kBlock, 0, s->stream>>>(t, static_cast<const T *>(s->u[1]),
                                                               static_cast<const T *>(s->w[1]), traj_u + K, traj_w + S);
        CUDA_TRY(s, cudaMemcpyAsync(seg_signal, d_signal + s0, sizeof(float) * count, cudaMemcpyDeviceToDevice, s->stream));
        if ((rc = run(0, s->flipped ? 1 : 0, recompute, count)) != FDTD_OK) return rc;
        settle(s, count);
        // The reverse steps of the segment, with its columns of dL/dy.
        if (P)
            CUDA_TRY(s, cudaMemcpy2DAsync(seg_dloss, sizeof(double) * segment, d_dloss + s0, sizeof(double) * steps,
                                          sizeof(double) * count, P, cudaMemcpyDeviceToDevice, s->stream));
        // The layer's products of this segment's last step, whose Q^, L^, H^ the segment after
        // left waiting: its factors are recorded now.
        if (tables && k + 1 < segments) {
            layer_pending_kernel<T><<<layer_blocks, kBlock, 0, s->stream>>>(
                t, static_cast<const T *>(adj.pending), traj_layer + (count - 1) * kLayerFactors * Lc, g_layer);
            CUDA_TRY(s, cudaGetLastError());
        }
        if (tangent && k + 1 < segments) {
            layer_pending_tangent_kernel<T><<<layer_blocks, kBlock, 0, s->stream>>>(
                t, static_cast<const T *>(adj.pending), traj_tan + (count - 1) * Tf, tan_acc);
            CUDA_TRY(s, cudaGetLastError());
        }
        if ((rc = run(1, x, reverse, count)) != FDTD_OK) return rc;
        if (tangent) flush_tangent();
        if (count & 1) x = 1 - x;
    }
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if ((rc = check_device_error(s)) != FDTD_OK) return rc;
    for (int k = 0; k < 5; ++k)
        if (grads[k] && g_len[k]) CUDA_TRY(s, cudaMemcpy(grads[k], g[k], sizeof(double) * g_len[k], cudaMemcpyDeviceToHost));
    s->tangent_valid = false;
    if (tangent) {
        // dL/dθ: the cells' sums in a fixed order, in two launches.
        const uint64_t span = (Lc + tan_blocks - 1) / tan_blocks;
        layer_tangent_sum_kernel<<<tan_blocks, kBlock, 0, s->stream>>>(tan_acc, Lc, span, tan_parts);
        layer_tangent_sum_kernel<<<1, kBlock, 0, s->stream>>>(tan_parts, tan_blocks, tan_blocks, tan_parts + tan_blocks);
        CUDA_TRY(s, cudaGetLastError());
        // (on the handle's stream, which does not wait for the legacy default stream's copies)
        CUDA_TRY(s, cudaMemcpyAsync(&s->tangent_gradient, tan_parts + tan_blocks, sizeof(double), cudaMemcpyDeviceToHost,
                                    s->stream));
        CUDA_TRY(s, cudaStreamSynchronize(s->stream));
        s->tangent_valid = true;
    }
    if (tables) {
        // The layer tables' gradient: the cells' sums by coordinate on the device, in a fixed
        // order, then each coordinate's six sums into its tables' entries (a product of the cells
        // at coordinate x goes to the face entries x + 1 or x).
        layer_table_sums_kernel<<<(uint32_t)coords, kBlock, 0, s->stream>>>(
            g_layer, (uint32_t)Lc, adj.by_coord, adj.coord_start, (uint32_t)s->nx, (uint32_t)(s->nx + s->ny), table_sums);
        CUDA_TRY(s, cudaGetLastError());
        std::vector<double> sums(6 * coords);
        CUDA_TRY(s, cudaMemcpyAsync(sums.data(), table_sums, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(s, cudaStreamSynchronize(s->stream));
        const uint64_t len[3] = {s->nx + 1, s->ny + 1, s->nz + 1};
        uint64_t keep_at[6], push_at[6], at = 0;  // offsets of keep/keep_face (x, y, z), then push/push_face
        for (int a = 0; a < 3; ++a) keep_at[2 * a] = at, at += len[a], keep_at[2 * a + 1] = at, at += len[a];
        for (int a = 0; a < 3; ++a) push_at[2 * a] = at, at += len[a], push_at[2 * a + 1] = at, at += len[a];
        s->layer_gradient.assign(at, 0.0);
        double *out = s->layer_gradient.data();
        uint64_t block = 0;
        for (int a = 0; a < 3; ++a)
            for (uint64_t x = 0; x + 1 < len[a]; ++x, ++block) {
                const double *f = sums.data() + 6 * block;
                out[keep_at[2 * a] + x] += f[0];
                out[push_at[2 * a] + x] += f[1];
                out[keep_at[2 * a + 1] + x + 1] += f[2];
                out[push_at[2 * a + 1] + x + 1] += f[3];
                out[keep_at[2 * a + 1] + x] += f[4];
                out[push_at[2 * a + 1] + x] += f[5];
            }
    } else {
        s->layer_gradient.clear();
    }
    return fdtd_reset(s);
}

// ---- fdtd_gradient_noalloc: the gradient's device memory from a static pool ------------------------

// The pool, in static device memory (one per device, held until the process exits); aligned for
// the tensor maps over the adjoint levels (16 bytes) and for coalesced access. Host code reaches it
// only through the address cudaGetSymbolAddress gives (pool_address).
constexpr size_t kPoolBytes = FDTD_GRADIENT_STATIC_BYTES;
constexpr size_t kPoolAlign = 256;
static __device__ __align__(256) unsigned char g_gradient_pool[kPoolBytes];

constexpr size_t pool_round(size_t bytes) { return ((bytes ? bytes : 16) + kPoolAlign - 1) / kPoolAlign * kPoolAlign; }

// The pool's address on the current device. Looked up on every call, not cached: the address
// belongs to the context that loaded the module, and a caller that destroys and recreates the
// device's primary context (cudaDeviceReset) gets the module loaded again, possibly elsewhere.
// Once the module is loaded the lookup is a table read.
int pool_address(fdtd_solver *s, void **out) {
    *out = nullptr;
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_gradient_pool);
    if (e != cudaSuccess) return cuda_fail(s, e, "cudaGetSymbolAddress of the gradient's static pool");
    *out = p;
    return FDTD_OK;
}

// Blocks of the pool handed out in order; each to be cleared is cleared on the handle's stream,
// in order with the gradient's own work.
struct StaticPool {
    fdtd_solver *s;
    char *base;
    size_t used = 0;
    int take(size_t bytes, void **out, bool zero) {
        *out = nullptr;
        const size_t size = pool_round(bytes);
        if (used + size > kPoolBytes) return fail(s, FDTD_EINVAL, "the gradient's buffers outgrow the static pool");
        *out = base + used;
        used += size;
        if (zero) CUDA_TRY(s, cudaMemsetAsync(*out, 0, size, s->stream));
        return FDTD_OK;
    }
    int take(size_t bytes, void **out) { return take(bytes, out, true); }  // gradient<T>'s scratch
};

// The pool's bytes for one gradient: the blocks place_adjoint and then gradient<T> take, in order
// (the checkpoints only where no tape supplies the segments' states).
size_t pool_bytes(const fdtd_solver *s, const AdjointLists &l, uint64_t steps, uint64_t segment, bool taped) {
    const size_t e = s->precision == FDTD_FP64 ? 8 : 4;
    const uint64_t K = s->specials, S = s->states, P = std::max<uint64_t>(1, s->probes), n = s->n_device;
    size_t total = 0;
    auto list = [&](size_t count, size_t unit) { total += count ? pool_round(count * unit) : 0; };
    list(l.reader_start.size(), 4), list(l.reader_index.size(), 4), list(l.reader_kind.size(), 1);
    list(l.reader_coef.size(), 8), list(l.cells.size(), 4), list(l.starts.size(), 4), list(l.rows.size(), 4);
    list(l.coefs.size(), 8), list(l.special_read_start.size(), 4), list(l.corrected_read_start.size(), 4);
    list(l.masks.size(), 4), list(l.scales.size(), 4), list(l.types.size(), 1);
    list(l.read_probe.size(), 4), list(l.read_weight.size(), 8);
    list(l.special_layer_mask.size(), 1), list(l.corrected_layer_mask.size(), 1), list(l.layer_mask.size(), 1);
    list(l.layer_from_start.size(), 4), list(l.layer_from_row.size(), 4), list(l.layer_from_coef.size(), 8);
    list(l.layer_read_start.size(), 4), list(l.layer_interior.size(), 1);
    list(l.special_order.size(), 4), list(l.corrected_order.size(), 4);
    const uint64_t Lc = s->layers;
    if (Lc) total += pool_round(e * kCarried * Lc) + 2 * pool_round(e * kHats * n) + pool_round(e * 9 * Lc);
    total += 2 * (pool_round(e * n) + pool_round(e * S)) + 2 * pool_round(e * K);
    if (segment == 0 || segment > steps) segment = steps;
    const uint64_t segments = (steps + segment - 1) / segment;
    total += pool_round(4 * steps) + pool_round(8 * P * steps) + pool_round(e * K * (segment + 2)) +
             pool_round(e * S * (segment + 2)) + pool_round(8 * P * segment) + pool_round(4 * segment) +
             pool_round(8 * P * segment);
    total += 2 * pool_round(8 * K) + 3 * pool_round(8 * S);
    if (Lc) total += pool_round(4 * l.by_coord.size()) + pool_round(4 * l.coord_start.size());
    if (Lc && s->gradient_tables && !s->tangent)
        total += pool_round(e * kLayerFactors * Lc * segment) + pool_round(8 * kLayerFactors * Lc) +
                 pool_round(8 * 6 * (s->nx + s->ny + s->nz));
    if (Lc && s->tangent) {
        const bool trajectory = taped && s->tape_traj;
        const uint64_t blocks = std::min<uint64_t>(256, std::max<uint64_t>(1, (Lc + kBlock - 1) / kBlock));
        if (!trajectory) total += pool_round(e * s->tangent_factors * segment);
        total += pool_round(8 * Lc) + pool_round(8 * (blocks + 1)) + pool_round(sizeof(void *));
    }
    if (!taped) total += (segments - 1) * pool_round(checkpoint_bytes(s));
    return total;
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

#ifndef FDTD_BUILD_ID
#define FDTD_BUILD_ID "unknown"
#endif
const char *fdtd_build_id(void) { return FDTD_BUILD_ID; }

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
    if (precision != FDTD_FP32 && precision != FDTD_FP64 && precision != FDTD_FP32_COMPENSATED)
        return set_global(FDTD_EINVAL, "precision is FDTD_FP32, FDTD_FP64 or FDTD_FP32_COMPENSATED");
    std::string why;
    if (validate(layout, why) != FDTD_OK) return set_global(FDTD_EINVAL, why);
    if (layout->flow_count && precision == FDTD_FP32_COMPENSATED)
        return set_global(FDTD_EINVAL, "the compensated form steps still air only");
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
    s->sms = prop.multiProcessorCount;
    s->precision = precision;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking);
    // The matched layer's stream at the highest priority: its blocks are placed as soon as a
    // multiprocessor has room, beside the sweep's, rather than after the sweep's last wave.
    int lowest = 0, highest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&lowest, &highest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s->layer_stream, cudaStreamNonBlocking, highest);
    s->layer_priority = highest;
    for (cudaEvent_t &event : s->joined)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&event, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        const int rc = cuda_fail(nullptr, e, "cudaStreamCreate");
        release(s);
        delete s;
        return rc;
    }
    int rc = build(s, layout);
    // Every upload and clearing of the set-up complete before the handle's streams use them.
    if (rc == FDTD_OK) {
        const cudaError_t synced = cudaDeviceSynchronize();
        if (synced != cudaSuccess) rc = cuda_fail(s, synced, "cudaDeviceSynchronize");
    }
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

void *fdtd_stream(const fdtd_solver *s) { return s ? static_cast<void *>(s->stream) : nullptr; }

int fdtd_synchronize(fdtd_solver *s) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    DeviceGuard guard(s->device);
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return check_device_error(s);
}

int fdtd_run(fdtd_solver *s, const float *signal, uint64_t steps, double *out) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (steps == 0) return FDTD_OK;
    if (!signal || (s->probes && !out)) return fail(s, FDTD_EINVAL, "no signal or output buffer");
    DeviceGuard guard(s->device);
    // Pinned host staging for a piece of the run (the drive and the probes' records), grown on
    // demand; the device side is the handle's chunk buffers, kGraphSteps steps at a time.
    const uint64_t P = std::max<uint64_t>(1, s->probes);
    const uint64_t piece = std::min<uint64_t>(steps, std::max<uint64_t>(kGraphSteps, (64ull << 20) / (8 * P)));
    if (s->stage_steps < piece) {
        if (s->stage_signal) cudaFreeHost(s->stage_signal);
        if (s->stage_out) cudaFreeHost(s->stage_out);
        s->stage_signal = nullptr, s->stage_out = nullptr, s->stage_steps = 0;
        CUDA_TRY(s, cudaMallocHost((void **)&s->stage_signal, piece * sizeof(float)));
        CUDA_TRY(s, cudaMallocHost((void **)&s->stage_out, piece * P * sizeof(double)));
        s->stage_steps = piece;
    }
    // A tape (fdtd_set_tape) of a run from rest: the trajectory of the special rows and branch
    // velocities when it fits the budget; else the state at every multiple of the segment before
    // the run's end, in the checkpoints' layout of the gradient (current level, previous level,
    // current and previous branch velocities).
    const bool taping = s->tape_segment && s->steps_done == 0;
    uint64_t tape_segment = taping ? std::min(s->tape_segment, steps) : 0;
    const size_t e = s->precision == FDTD_FP64 ? 8 : 4;
    const uint64_t K = s->specials, S = s->states;
    bool keep_traj = false;
    if (taping) {
        s->tape_valid = false;
        s->tape_traj = false;
        s->tape_tangent = false;
        uint64_t budget = s->tape_budget;
        if (budget == UINT64_MAX) {
            size_t free_bytes = 0, total_bytes = 0;
            CUDA_TRY(s, cudaMemGetInfo(&free_bytes, &total_bytes));
            budget = free_bytes / 2 + e * (K + S) * s->tape_levels + e * s->tangent_factors * s->tape_t_steps;
            // (what the tape holds already counts)
        }
        // (A grid with a matched layer whose gradients give its tables keeps checkpoints: the
        // gradient recomputes the layer's factors a segment at a time. Without the tables the
        // layer steps back on its carried values alone, and the rows' trajectory is all it needs;
        // along a tangent of the tables, the trajectory keeps the tangent's factors of every step.)
        const uint64_t tangent_bytes = s->layers && s->tangent ? e * s->tangent_factors * steps : 0;
        keep_traj = K + S > 0 && (!s->layers || !s->gradient_tables || s->tangent) &&
                    e * (K + S) * (steps + 2) + tangent_bytes <= budget;
    }
    const bool keep_tangent = keep_traj && s->layers && s->tangent;
    if (keep_traj) {
        int r;
        if (s->tape_levels < steps + 2) {
            // Grow the tape (freeing the old one first).
            for (void **p : {&s->tape_u, &s->tape_w}) {
                if (!*p) continue;
                cudaFree(*p);
                s->allocations.erase(std::find(s->allocations.begin(), s->allocations.end(), *p));
                *p = nullptr;
            }
            s->device_bytes -= e * (K + S) * s->tape_levels;
            s->tape_levels = 0;
            if ((r = zeros(s, e * K * (steps + 2), &s->tape_u)) != FDTD_OK) return r;
            if ((r = zeros(s, e * S * (steps + 2), &s->tape_w)) != FDTD_OK) return r;
            s->tape_levels = steps + 2;
        }
        if (!s->stage_u) {
            if ((r = zeros(s, e * K * kGraphSteps, &s->stage_u)) != FDTD_OK) return r;
            if ((r = zeros(s, e * S * kGraphSteps, &s->stage_w)) != FDTD_OK) return r;
        }
        if (keep_tangent && s->tape_t_steps < steps) {
            if (s->tape_t) {
                cudaFree(s->tape_t);
                s->allocations.erase(std::find(s->allocations.begin(), s->allocations.end(), s->tape_t));
                s->device_bytes -= e * s->tangent_factors * s->tape_t_steps;
                s->tape_t = nullptr, s->tape_t_steps = 0;
            }
            if ((r = zeros(s, e * s->tangent_factors * steps, &s->tape_t)) != FDTD_OK) return r;
            s->tape_t_steps = steps;
        }
        if (keep_tangent && !s->stage_t && (r = zeros(s, e * s->tangent_factors * kGraphSteps, &s->stage_t)) != FDTD_OK)
            return r;
        // Levels 0 and 1: the state at rest.
        CUDA_TRY(s, cudaMemsetAsync(s->tape_u, 0, e * K * 2, s->stream));
        if (S) CUDA_TRY(s, cudaMemsetAsync(s->tape_w, 0, e * S * 2, s->stream));
        tape_segment = steps;  // no checkpoints
    }
    // While keeping the trajectory, every step records into the staging (restored on return).
    struct Recording {
        fdtd_solver *s;
        ~Recording() { s->record_u = s->record_w = s->record_tangent = nullptr, s->record_offset = 2; }
    } recording{s};
    if (keep_traj) s->record_u = s->stage_u, s->record_w = s->stage_w, s->record_offset = 0, s->record_probes = true;
    if (taping && !keep_traj) {
        const uint64_t needed = (steps + tape_segment - 1) / tape_segment - 1;
        while (s->tape_checkpoints.size() < needed) {
            void *p = nullptr;
            CUDA_TRY(s, cudaMalloc(&p, checkpoint_bytes(s)));
            s->allocations.push_back(p);
            s->device_bytes += checkpoint_bytes(s);
            s->tape_checkpoints.push_back(p);
        }
    }
    int rc = FDTD_OK;
    for (uint64_t begin = 0; begin < steps && rc == FDTD_OK; begin += piece) {
        const uint64_t count = std::min(piece, steps - begin);
        std::memcpy(s->stage_signal, signal + begin, count * sizeof(float));
        for (uint64_t done = 0; done < count && rc == FDTD_OK;) {
            uint64_t chunk = std::min<uint64_t>(kGraphSteps, count - done);
            const uint64_t at = begin + done;  // steps of this run done before the chunk
            if (taping) chunk = std::min(chunk, (at / tape_segment + 1) * tape_segment - at);
            CUDA_TRY(s, cudaMemcpyAsync(s->d_sig, s->stage_signal + done, chunk * sizeof(float), cudaMemcpyHostToDevice,
                                        s->stream));
            const bool graphed = chunk == kGraphSteps && s->n_device < kGraphCells;
            // (The tangent's factors: straight onto the tape, or a captured chunk's into staging.)
            if (keep_tangent)
                s->record_tangent = graphed ? s->stage_t : static_cast<char *>(s->tape_t) + e * s->tangent_factors * at;
            if (graphed) {
                // A whole chunk: the captured graph of its steps for the levels' present roles
                // (with the trajectory's recording, a graph of its own).
                cudaGraphExec_t &graph = keep_traj ? s->tape_graph[s->flipped ? 1 : 0] : s->graph[s->flipped ? 1 : 0];
                if (!graph && (rc = capture(s, &graph)) != FDTD_OK) break;
                CUDA_TRY(s, cudaGraphLaunch(graph, s->stream));
            } else if ((rc = dispatch(s, s->d_sig, chunk, s->d_rec, kGraphSteps)) != FDTD_OK) {
                break;
            }
            settle(s, chunk);
            if (keep_traj) {
                // The chunk's levels at + 2 .. at + chunk + 1 onto the tape.
                CUDA_TRY(s, cudaMemcpyAsync(static_cast<char *>(s->tape_u) + e * K * (at + 2), s->stage_u, e * K * chunk,
                                            cudaMemcpyDeviceToDevice, s->stream));
                if (S)
                    CUDA_TRY(s, cudaMemcpyAsync(static_cast<char *>(s->tape_w) + e * S * (at + 2), s->stage_w,
                                                e * S * chunk, cudaMemcpyDeviceToDevice, s->stream));
                if (keep_tangent && graphed)
                    CUDA_TRY(s, cudaMemcpyAsync(static_cast<char *>(s->tape_t) + e * s->tangent_factors * at, s->stage_t,
                                                e * s->tangent_factors * chunk, cudaMemcpyDeviceToDevice, s->stream));
            }
            if (taping && !keep_traj && (at + chunk) % tape_segment == 0 && at + chunk < steps) {
                char *c = static_cast<char *>(s->tape_checkpoints[(at + chunk) / tape_segment - 1]);
                if ((rc = save_checkpoint(s, c)) != FDTD_OK) break;
            }
            if (s->probes) {
                CUDA_TRY(s, cudaMemcpy2DAsync(s->stage_out + done, count * sizeof(double), s->d_rec,
                                              kGraphSteps * sizeof(double), chunk * sizeof(double), s->probes,
                                              cudaMemcpyDeviceToHost, s->stream));
            }
            done += chunk;
        }
        if (rc != FDTD_OK) break;
        CUDA_TRY(s, cudaStreamSynchronize(s->stream));
        for (uint64_t p = 0; p < s->probes; ++p)
            std::memcpy(out + p * steps + begin, s->stage_out + p * count, count * sizeof(double));
    }
    if (rc != FDTD_OK) return rc;
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if ((rc = check_device_error(s)) != FDTD_OK) return rc;
    if (taping) {
        s->tape_signal.assign(signal, signal + steps);
        s->tape_valid = true;
        s->tape_traj = keep_traj;
        s->tape_tangent = keep_tangent;
    }
    for (uint64_t k = 0; k < s->probes * steps; ++k) {
        if (!std::isfinite(out[k])) return fail(s, FDTD_ENONFINITE, "the wave solver's run did not stay finite");
    }
    return FDTD_OK;
}

int fdtd_gradient_noalloc(fdtd_solver *s, const float *signal, uint64_t steps, const double *dloss_dy,
                          uint64_t segment, double *grad_coef_b, double *grad_coef_inv, double *grad_now,
                          double *grad_before, double *grad_gain) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (s->precision == FDTD_FP32_COMPENSATED)
        return fail(s, FDTD_EINVAL, "the gradient steps FDTD_FP32 or FDTD_FP64, not the compensated form");
    if (steps == 0) return fail(s, FDTD_EINVAL, "no steps to differentiate");
    if (s->flowing) return fail(s, FDTD_EINVAL, "the gradient steps still air only");
    if (!signal || (s->probes && !dloss_dy)) return fail(s, FDTD_EINVAL, "no signal or loss gradient");
    DeviceGuard guard(s->device);
    void *base;
    int rc;
    if ((rc = pool_address(s, &base)) != FDTD_OK) return rc;
    AdjointLists lists;
    if ((rc = adjoint_lists(s, lists)) != FDTD_OK) return rc;
    const size_t need = pool_bytes(s, lists, steps, segment, holds_tape(s, signal, steps, segment));
    if (need > kPoolBytes) {
        char message[200];
        std::snprintf(message, sizeof message,
                      "the gradient needs %llu bytes of device memory; the static pool holds %llu: fewer steps, a "
                      "longer segment, or fdtd_gradient",
                      (unsigned long long)need, (unsigned long long)kPoolBytes);
        return fail(s, FDTD_EINVAL, message);
    }
    // This handle's earlier calls have ended (each ends with its stream), so the pool is free here
    // unless another call overlaps this one, which the header warns of.
    StaticPool pool{s, static_cast<char *>(base)};
    AdjointState adj;
    if ((rc = place_adjoint(s, lists, pool, adj)) != FDTD_OK) return rc;
    double *grads[5] = {grad_coef_b, grad_coef_inv, grad_now, grad_before, grad_gain};
    // (No graphs: instantiating one allocates.)
    return s->precision == FDTD_FP64 ? gradient<double>(s, adj, pool, signal, steps, dloss_dy, segment, grads, false)
                                     : gradient<float>(s, adj, pool, signal, steps, dloss_dy, segment, grads, false);
}

int fdtd_set_coefficients(fdtd_solver *s, const float *coef_b, const float *coef_inv, const float *branch_now,
                          const float *branch_before, const float *branch_gain) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    // (The compensated form's row residuals are worked out from the coefficients at creation.)
    if (s->precision == FDTD_FP32_COMPENSATED)
        return fail(s, FDTD_EINVAL, "coefficients are set on FDTD_FP32 or FDTD_FP64 handles");
    DeviceGuard guard(s->device);
    const uint64_t K = s->specials, S = s->states;
    for (cudaStream_t stream : {s->stream, s->side, s->layer_stream}) CUDA_TRY(s, cudaStreamSynchronize(stream));
    Tables &g = s->tables;
    if (coef_b && K) CUDA_TRY(s, cudaMemcpy(const_cast<float *>(g.coef_b), coef_b, 4 * K, cudaMemcpyHostToDevice));
    if (coef_inv && K) CUDA_TRY(s, cudaMemcpy(const_cast<float *>(g.coef_inv), coef_inv, 4 * K, cudaMemcpyHostToDevice));
    const float *branch[3] = {branch_now, branch_before, branch_gain};
    const float *state[3] = {g.state_now, g.state_before, g.state_gain};
    std::vector<float> gathered(S);
    for (int c = 0; c < 3; ++c) {
        if (!branch[c] || !S) continue;
        for (uint64_t j = 0; j < S; ++j) gathered[j] = branch[c][s->state_branch[j]];
        CUDA_TRY(s, cudaMemcpy(const_cast<float *>(state[c]), gathered.data(), 4 * S, cudaMemcpyHostToDevice));
    }
    if (coef_inv && s->adjoint_ready) {
        // The adjoint's products with coef_inv, as its set-up forms them.
        AdjointTables &t = s->adjoint.t;
        std::vector<double> coef(s->adjoint_reader_row.size());
        for (size_t e = 0; e < coef.size(); ++e) {
            const int32_t r = s->adjoint_reader_row[e];
            coef[e] = r >= 0 ? (double)coef_inv[r] * s->adjoint_reader_base[e] : s->adjoint_reader_base[e];
        }
        if (!coef.empty())
            CUDA_TRY(s, cudaMemcpy(const_cast<double *>(t.reader_coef), coef.data(), 8 * coef.size(), cudaMemcpyHostToDevice));
        coef.resize(s->adjoint_corrected_row.size());
        for (size_t e = 0; e < coef.size(); ++e)
            coef[e] = (double)coef_inv[s->adjoint_corrected_row[e]] * s->adjoint_corrected_base[e];
        if (!coef.empty())
            CUDA_TRY(s, cudaMemcpy(const_cast<double *>(t.corrected_coef), coef.data(), 8 * coef.size(),
                                   cudaMemcpyHostToDevice));
        coef.resize(s->adjoint_layer_row.size());
        for (size_t e = 0; e < coef.size(); ++e)
            coef[e] = (double)coef_inv[s->adjoint_layer_row[e]] * s->adjoint_layer_base[e];
        if (!coef.empty())
            CUDA_TRY(s, cudaMemcpy(const_cast<double *>(t.layer_from_coef), coef.data(), 8 * coef.size(),
                                   cudaMemcpyHostToDevice));
    }
    // (Copies from pageable memory may return before they land; the handle's streams do not wait
    // for the default stream.)
    CUDA_TRY(s, cudaDeviceSynchronize());
    s->tape_valid = false;
    return FDTD_OK;
}

int fdtd_test_wait(fdtd_solver *s, uint32_t spins) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (spins == 0 || spins > (1u << 24)) return fail(s, FDTD_EINVAL, "spins are 1 to 2^24");
    DeviceGuard guard(s->device);
    void *p = nullptr;
    CUDA_TRY(s, cudaMalloc(&p, sizeof(unsigned int)));
    cudaError_t e = cudaMemsetAsync(p, 0, sizeof(unsigned int), s->stream);
    if (e == cudaSuccess) {
        wait_test_kernel<<<1, 32, 0, s->stream>>>(static_cast<const unsigned int *>(p), spins, s->d_error);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(p);
    if (e != cudaSuccess) return cuda_fail(s, e, "fdtd_test_wait");
    return check_device_error(s);
}

int fdtd_level_plane(fdtd_solver *s, uint64_t z, int which, void **ptr, uint64_t *bytes) {
    if (!s || !ptr || !bytes) return set_global(FDTD_EINVAL, "no solver or no place for the plane");
    if (z >= s->nz || (which != 0 && which != 1)) return fail(s, FDTD_EINVAL, "no such plane or level");
    const size_t e = s->precision == FDTD_FP64 ? 8 : 4;
    *bytes = e * s->pitch * s->ny;
    *ptr = static_cast<char *>(s->u[which ? 0 : 1]) + *bytes * z;
    return FDTD_OK;
}

int fdtd_run_linked(fdtd_solver *const *solvers, uint32_t count, const fdtd_plane_link *links, uint32_t link_count,
                    const float *const *d_signals, uint64_t steps, double *const *d_outs, uint64_t out_stride) {
    if (!solvers || count == 0) return set_global(FDTD_EINVAL, "no solvers to run");
    if (link_count && !links) return set_global(FDTD_EINVAL, "no links");
    if (!d_signals) return set_global(FDTD_EINVAL, "no signals");
    for (uint32_t h = 0; h < count; ++h) {
        fdtd_solver *s = solvers[h];
        if (!s) return set_global(FDTD_EINVAL, "a null solver in the group");
        if (!d_signals[h]) return fail(s, FDTD_EINVAL, "no signal for a solver of the group");
        if (s->probes && (!d_outs || !d_outs[h])) return fail(s, FDTD_EINVAL, "no output buffer for a solver of the group");
        if (s->probes && out_stride < steps) return fail(s, FDTD_EINVAL, "the output's stride is shorter than the run");
        if (s->precision != solvers[0]->precision)
            return set_global(FDTD_EINVAL, "the group's solvers step in one precision");
        if (s->flowing) return fail(s, FDTD_EINVAL, "linked slabs step still air only");
        for (uint32_t g = 0; g < h; ++g)
            if (solvers[g] == s) return set_global(FDTD_EINVAL, "a solver appears twice in the group");
    }
    const size_t e = solvers[0]->precision == FDTD_FP64 ? 8 : 4;
    for (uint32_t l = 0; l < link_count; ++l) {
        const fdtd_plane_link &k = links[l];
        if (k.from >= count || k.to >= count || k.from == k.to) return set_global(FDTD_EINVAL, "a link joins no two solvers of the group");
        const fdtd_solver *a = solvers[k.from], *b = solvers[k.to];
        if (k.from_plane >= a->nz || k.to_plane >= b->nz) return set_global(FDTD_EINVAL, "a link's plane lies outside its grid");
        if (a->pitch != b->pitch || a->ny != b->ny) return set_global(FDTD_EINVAL, "linked grids have planes of different sizes");
        // Only a plane of solid cells (nothing of its own steps it) may be filled from another grid.
        for (uint64_t y = 0; y < b->ny; ++y)
            for (uint64_t x = 0; x < b->nx; ++x)
                if (b->host_types.size() && b->host_types[x + b->pitch * (y + b->ny * k.to_plane)] != kSolid)
                    return set_global(FDTD_EINVAL, "a link fills a plane that holds air of its own grid");
    }
    if (steps == 0) return FDTD_OK;
    // Peer access between the devices the links join (a no-op where it is already on).
    for (uint32_t l = 0; l < link_count; ++l) {
        const int da = solvers[links[l].from]->device, db = solvers[links[l].to]->device;
        if (da == db) continue;
        int can = 0;
        cudaDeviceCanAccessPeer(&can, da, db);
        if (can) {
            DeviceGuard guard(da);
            const cudaError_t pe = cudaDeviceEnablePeerAccess(db, 0);
            if (pe != cudaSuccess && pe != cudaErrorPeerAccessAlreadyEnabled) return cuda_fail(solvers[0], pe, "cudaDeviceEnablePeerAccess");
            cudaGetLastError();
        }
    }
    // Per solver, the event after its step and the copies out of it (its neighbours' next step
    // waits for it).
    std::vector<cudaEvent_t> copied(count, nullptr);
    auto release_events = [&]() {
        for (cudaEvent_t ev : copied)
            if (ev) cudaEventDestroy(ev);
    };
    for (uint32_t h = 0; h < count; ++h) {
        DeviceGuard guard(solvers[h]->device);
        const cudaError_t ce = cudaEventCreateWithFlags(&copied[h], cudaEventDisableTiming);
        if (ce != cudaSuccess) {
            release_events();
            return cuda_fail(solvers[h], ce, "cudaEventCreate");
        }
    }
    int rc = FDTD_OK;
    for (uint64_t k = 0; k < steps && rc == FDTD_OK; ++k) {
        // Each solver's step k, after the planes its neighbours sent it at step k - 1.
        for (uint32_t h = 0; h < count && rc == FDTD_OK; ++h) {
            fdtd_solver *s = solvers[h];
            DeviceGuard guard(s->device);
            if (k > 0)
                for (uint32_t l = 0; l < link_count; ++l)
                    if (links[l].to == h) {
                        const cudaError_t we = cudaStreamWaitEvent(s->stream, copied[links[l].from], 0);
                        if (we != cudaSuccess) rc = cuda_fail(s, we, "cudaStreamWaitEvent");
                    }
            if (rc == FDTD_OK) rc = dispatch(s, d_signals[h] + k, 1, d_outs ? d_outs[h] + k : nullptr, out_stride);
            if (rc == FDTD_OK) settle(s, 1);
        }
        // Then the planes of the new levels, each on its source's stream after its step.
        for (uint32_t l = 0; l < link_count && rc == FDTD_OK; ++l) {
            fdtd_solver *a = solvers[links[l].from], *b = solvers[links[l].to];
            DeviceGuard guard(a->device);
            const uint64_t plane = e * a->pitch * a->ny;
            const char *src = static_cast<const char *>(a->u[1]) + plane * links[l].from_plane;
            char *dst = static_cast<char *>(b->u[1]) + plane * links[l].to_plane;
            const cudaError_t me = a->device == b->device
                                       ? cudaMemcpyAsync(dst, src, plane, cudaMemcpyDeviceToDevice, a->stream)
                                       : cudaMemcpyPeerAsync(dst, b->device, src, a->device, plane, a->stream);
            if (me != cudaSuccess) rc = cuda_fail(a, me, "the plane's copy");
        }
        for (uint32_t h = 0; h < count && rc == FDTD_OK; ++h) {
            DeviceGuard guard(solvers[h]->device);
            const cudaError_t re = cudaEventRecord(copied[h], solvers[h]->stream);
            if (re != cudaSuccess) rc = cuda_fail(solvers[h], re, "cudaEventRecord");
        }
    }
    // Every solver's stream ends after the copies into its grid (its level is then complete).
    for (uint32_t l = 0; l < link_count && rc == FDTD_OK; ++l) {
        fdtd_solver *b = solvers[links[l].to];
        DeviceGuard guard(b->device);
        const cudaError_t we = cudaStreamWaitEvent(b->stream, copied[links[l].from], 0);
        if (we != cudaSuccess) rc = cuda_fail(b, we, "cudaStreamWaitEvent");
    }
    // (Destroying an event whose work is pending is allowed: it is released when it completes.)
    release_events();
    return rc;
}

int fdtd_set_launch(fdtd_solver *s, int layer_per_sm, int special_per_sm) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (layer_per_sm < 0 || special_per_sm < 0 || layer_per_sm > 64 || special_per_sm > 64)
        return fail(s, FDTD_EINVAL, "blocks per multiprocessor are 0 (a thread a cell) to 64");
    DeviceGuard guard(s->device);
    for (cudaStream_t stream : {s->stream, s->side, s->layer_stream}) CUDA_TRY(s, cudaStreamSynchronize(stream));
    s->layer_per_sm = layer_per_sm, s->special_per_sm = special_per_sm;
    // The captured chunks and the gradient's graphs hold the old launch shapes.
    Kept{s}.drop_graphs();
    for (cudaGraphExec_t &g : s->graph)
        if (g) cudaGraphExecDestroy(g), g = nullptr;
    for (cudaGraphExec_t &g : s->tape_graph)
        if (g) cudaGraphExecDestroy(g), g = nullptr;
    return FDTD_OK;
}

int fdtd_set_tiles(fdtd_solver *s, int shape, uint64_t planes) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (shape < 0 || shape >= kShapes)
        return fail(s, FDTD_EINVAL, "the tile shape is an index 0 to " + std::to_string(kShapes - 1));
    if (planes < 1 || planes > 1024) return fail(s, FDTD_EINVAL, "planes a tile are 1 to 1024");
    if (!s->bulk_tiles) return FDTD_OK;  // no interior cells: no sweep
    if (s->shape_per_sm[shape] < 1) return fail(s, FDTD_EINVAL, "the tile shape does not fit a multiprocessor here");
    DeviceGuard guard(s->device);
    for (cudaStream_t stream : {s->stream, s->side, s->layer_stream}) CUDA_TRY(s, cudaStreamSynchronize(stream));
    Kept{s}.drop_graphs();
    return use_shape(s, shape, planes);
}

int fdtd_get_tiles(const fdtd_solver *s, fdtd_tiles *out) {
    if (!s || !out) return set_global(FDTD_EINVAL, "no solver or no output");
    out->shape = s->bulk_shape;
    out->tile_x = kShapeInfo[s->bulk_shape].tx;
    out->tile_y = kShapeInfo[s->bulk_shape].ty;
    out->stages = kShapeInfo[s->bulk_shape].stages;
    out->planes = s->bulk_chunk;
    out->tiles = s->bulk_tiles;
    out->blocks_per_sm = s->shape_per_sm[s->bulk_shape];
    out->concurrent = s->concurrent;
    out->threads = kShapeInfo[s->bulk_shape].threads;
    out->cols = kShapeInfo[s->bulk_shape].cols;
    return FDTD_OK;
}

int fdtd_set_adjoint_launch(fdtd_solver *s, int far_per_sm, int near_per_sm) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (far_per_sm < 0 || near_per_sm < 0 || far_per_sm > 32 || near_per_sm > 32)
        return fail(s, FDTD_EINVAL, "blocks an SM are 0 to 32");
    DeviceGuard guard(s->device);
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    s->adjoint_far_per_sm = far_per_sm, s->adjoint_near_per_sm = near_per_sm;
    Kept{s}.drop_graphs();  // the gradient's graphs hold the old launches
    return FDTD_OK;
}

int fdtd_set_streams(fdtd_solver *s, int concurrent) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    DeviceGuard guard(s->device);
    for (cudaStream_t stream : {s->stream, s->side, s->layer_stream}) CUDA_TRY(s, cudaStreamSynchronize(stream));
    if (concurrent < 0 || concurrent > 5) return fail(s, FDTD_EINVAL, "the streams' arrangement is 0 to 5");
    s->concurrent = concurrent;
    // The captured chunks and the gradient's graphs hold the old streams' order.
    Kept{s}.drop_graphs();
    for (cudaGraphExec_t &g : s->graph)
        if (g) cudaGraphExecDestroy(g), g = nullptr;
    for (cudaGraphExec_t &g : s->tape_graph)
        if (g) cudaGraphExecDestroy(g), g = nullptr;
    return FDTD_OK;
}

int fdtd_autotune(fdtd_solver *s, uint64_t trial_steps, int *layer_per_sm, int *special_per_sm) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (s->steps_done != 0) return fail(s, FDTD_EINVAL, "fdtd_autotune runs from rest (after fdtd_create or fdtd_reset)");
    if (trial_steps == 0) trial_steps = 8;
    DeviceGuard guard(s->device);
    int rc = FDTD_OK;
    // The drive (zeros) and the records of the trials, on the device; the fields' values do not
    // change the kernels' memory traffic.
    void *sig = nullptr, *rec = nullptr;
    CUDA_TRY(s, cudaMalloc(&sig, sizeof(float) * trial_steps));
    struct Free {
        void *&a, *&b;
        ~Free() { cudaFree(a), cudaFree(b); }
    } release_trials{sig, rec};
    CUDA_TRY(s, cudaMemsetAsync(sig, 0, sizeof(float) * trial_steps, s->stream));
    CUDA_TRY(s, cudaMalloc(&rec, sizeof(double) * trial_steps * std::max<uint64_t>(1, s->probes)));
    cudaEvent_t start, end;
    CUDA_TRY(s, cudaEventCreate(&start));
    CUDA_TRY(s, cudaEventCreate(&end));
    const bool timing = s->timing;
    s->timing = false;
    // Times trial_steps steps of the handle's present choice: one untimed dispatch, then the
    // faster of two timed ones (a single short pass was too noisy to rank close choices); ms < 0
    // when it could not run.
    struct Trial {
        int shape;
        uint64_t chunk;
        int layer, special, mode;
        float ms;
    };
    std::vector<Trial> trials;  // every choice timed, for the finalists
    bool recording = true;
    auto trial = [&](float &ms) -> int {
        ms = -1.0f;
        for (int pass = 0; pass < 3; ++pass) {
            if (pass > 0) CUDA_TRY(s, cudaEventRecord(start, s->stream));
            const int r = dispatch(s, static_cast<const float *>(sig), trial_steps, static_cast<double *>(rec), trial_steps);
            if (r != FDTD_OK) return r;
            settle(s, trial_steps);
            if (pass == 0) continue;
            CUDA_TRY(s, cudaEventRecord(end, s->stream));
            CUDA_TRY(s, cudaEventSynchronize(end));
            float t = 0.0f;
            CUDA_TRY(s, cudaEventElapsedTime(&t, start, end));
            if (ms < 0.0f || t < ms) ms = t;
        }
        if (recording)
            trials.push_back(Trial{s->bulk_shape, s->bulk_chunk, s->layer_per_sm, s->special_per_sm, s->concurrent, ms});
        return FDTD_OK;
    };
    // The sweep's tile shape and planes a tile (the default chunk, a quarter, half and twice it,
    // within 8 to 64) with the layer and special launches as they are; then those launches (the
    // streams beside one another or in turn, the layer's and the special rows' blocks an SM) given
    // the tiles; then the tiles once more given the launches, as the kernels share the SMs.
    auto tune_tiles = [&]() -> int {
        if (!s->bulk_tiles) return FDTD_OK;
        const uint64_t base = default_chunk(s);
        float best_tiles = -1.0f;
        int best_shape = s->bulk_shape, r = FDTD_OK;
        uint64_t best_chunk = s->bulk_chunk;
        for (int shape = 0; shape < kShapes && r == FDTD_OK; ++shape) {
            if (s->shape_per_sm[shape] < 1) continue;  // does not fit an SM in this precision
            for (uint64_t chunk : {base / 4, base / 2, base, base * 2}) {
                if (chunk < 8 || chunk > 64) continue;
                if ((r = use_shape(s, shape, chunk)) != FDTD_OK) break;
                float ms;
                if ((r = trial(ms)) != FDTD_OK) break;
                if (best_tiles < 0.0f || ms < best_tiles) best_tiles = ms, best_shape = shape, best_chunk = chunk;
            }
        }
        return r == FDTD_OK ? use_shape(s, best_shape, best_chunk) : r;
    };
    const int layers[] = {4, 8, 12, 16, 0}, specials[] = {2, 4, 8, 0};
    int best_layer = s->layer_per_sm, best_special = s->special_per_sm, best_concurrent = s->concurrent;
    auto tune_launch = [&]() -> int {
        float best = -1.0f;
        int r = FDTD_OK;
        for (int c : {1, 4, 2, 5, 3, 0}) {
            s->concurrent = c;
            for (int l : layers) {
                if (r != FDTD_OK) break;
                if (!s->layers && l != layers[0]) continue;
                for (int k : specials) {
                    if (!s->specials && k != specials[0]) continue;
                    s->layer_per_sm = l, s->special_per_sm = k;
                    float ms;
                    if ((r = trial(ms)) != FDTD_OK) break;
                    if (best < 0.0f || ms < best) best = ms, best_layer = l, best_special = k, best_concurrent = c;
                }
            }
        }
        s->concurrent = best_concurrent, s->layer_per_sm = best_layer, s->special_per_sm = best_special;
        return r;
    };
    if (rc == FDTD_OK) rc = tune_tiles();
    if (rc == FDTD_OK) rc = tune_launch();
    if (rc == FDTD_OK) rc = tune_tiles();
    // The finalists: the best few whole choices seen, each timed three times more (the kernels
    // share the SMs, and a short trial can favour a choice that a longer run does not keep).
    if (rc == FDTD_OK && trials.size() > 1) {
        std::sort(trials.begin(), trials.end(), [](const Trial &a, const Trial &b) { return a.ms < b.ms; });
        std::vector<Trial> finalists;
        for (const Trial &t : trials) {
            bool seen = false;
            for (const Trial &f : finalists) seen = seen || (f.shape == t.shape && f.chunk == t.chunk && f.layer == t.layer &&
                                                              f.special == t.special && f.mode == t.mode);
            if (!seen) finalists.push_back(t);
            if (finalists.size() == 4) break;
        }
        Trial best{};
        best.ms = -1.0f;
        recording = false;
        for (Trial f : finalists) {
            if (s->bulk_tiles && (f.shape != s->bulk_shape || f.chunk != s->bulk_chunk) &&
                (rc = use_shape(s, f.shape, f.chunk)) != FDTD_OK)
                break;
            s->layer_per_sm = f.layer, s->special_per_sm = f.special, s->concurrent = f.mode;
            float least = -1.0f;
            for (int repeat = 0; repeat < 3 && rc == FDTD_OK; ++repeat) {
                float ms;
                if ((rc = trial(ms)) == FDTD_OK && (least < 0.0f || ms < least)) least = ms;
            }
            if (rc != FDTD_OK) break;
            if (best.ms < 0.0f || least < best.ms) best = f, best.ms = least;
        }
        if (rc == FDTD_OK && best.ms >= 0.0f) {
            if (s->bulk_tiles && (best.shape != s->bulk_shape || best.chunk != s->bulk_chunk))
                rc = use_shape(s, best.shape, best.chunk);
            best_layer = best.layer, best_special = best.special, best_concurrent = best.mode;
            s->concurrent = best.mode;
        }
    }
    s->timing = timing;
    cudaEventDestroy(start);
    cudaEventDestroy(end);
    if (rc != FDTD_OK) return rc;
    s->layer_per_sm = best_layer, s->special_per_sm = best_special;
    // The captured chunks and the gradient's graphs hold the old launch shapes.
    Kept{s}.drop_graphs();
    for (cudaGraphExec_t &g : s->graph)
        if (g) cudaGraphExecDestroy(g), g = nullptr;
    for (cudaGraphExec_t &g : s->tape_graph)
        if (g) cudaGraphExecDestroy(g), g = nullptr;
    if ((rc = check_device_error(s)) != FDTD_OK) return rc;
    if (layer_per_sm) *layer_per_sm = best_layer;
    if (special_per_sm) *special_per_sm = best_special;
    return fdtd_reset(s);
}

int fdtd_set_tape_budget(fdtd_solver *s, uint64_t bytes) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    s->tape_budget = bytes;
    s->tape_valid = false;
    return FDTD_OK;
}

int fdtd_set_tape(fdtd_solver *s, uint64_t segment) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (segment && s->precision == FDTD_FP32_COMPENSATED) return fail(s, FDTD_EINVAL, "the gradient steps FDTD_FP32 or FDTD_FP64, not the compensated form");
    if (segment && s->flowing) return fail(s, FDTD_EINVAL, "the gradient steps still air only");
    s->tape_segment = segment;
    s->tape_valid = false;
    return FDTD_OK;
}

int fdtd_set_timing(fdtd_solver *s, int enable) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    s->timing = enable != 0;
    return FDTD_OK;
}

int fdtd_get_timing(fdtd_solver *s, double ms[4], uint64_t *steps) {
    if (!s || !ms) return set_global(FDTD_EINVAL, "no solver or buffer");
    DeviceGuard guard(s->device);
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->side));
    for (int k = 0; k < 4; ++k) ms[k] = 0.0;
    for (size_t base = 0; base + 8 <= s->timing_events.size(); base += 8) {
        for (int k = 0; k < 4; ++k) {
            float t = 0.0f;
            CUDA_TRY(s, cudaEventElapsedTime(&t, s->timing_events[base + 2 * k], s->timing_events[base + 2 * k + 1]));
            ms[k] += t;
        }
    }
    if (steps) *steps = s->timed_steps;
    for (cudaEvent_t e : s->timing_events) cudaEventDestroy(e);
    s->timing_events.clear();
    s->timed_steps = 0;
    return FDTD_OK;
}

int fdtd_gradient(fdtd_solver *s, const float *signal, uint64_t steps, const double *dloss_dy, uint64_t segment,
                  double *grad_coef_b, double *grad_coef_inv, double *grad_now, double *grad_before, double *grad_gain) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (s->precision == FDTD_FP32_COMPENSATED)
        return fail(s, FDTD_EINVAL, "the gradient steps FDTD_FP32 or FDTD_FP64, not the compensated form");
    if (steps == 0) return fail(s, FDTD_EINVAL, "no steps to differentiate");
    if (s->flowing) return fail(s, FDTD_EINVAL, "the gradient steps still air only");
    if (!signal || (s->probes && !dloss_dy)) return fail(s, FDTD_EINVAL, "no signal or loss gradient");
    DeviceGuard guard(s->device);
    int rc = set_up_adjoint(s);
    if (rc != FDTD_OK) return rc;
    double *grads[5] = {grad_coef_b, grad_coef_inv, grad_now, grad_before, grad_gain};
    Kept kept{s};
    return s->precision == FDTD_FP64
               ? gradient<double>(s, s->adjoint, kept, signal, steps, dloss_dy, segment, grads, true)
               : gradient<float>(s, s->adjoint, kept, signal, steps, dloss_dy, segment, grads, true);
}

int fdtd_set_gradient_tables(fdtd_solver *s, int enable) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    s->gradient_tables = enable != 0;
    // (A tape taken without the tables may hold the rows' trajectory alone: it serves no
    // gradient in the tables, which then runs the forward pass again.)
    s->layer_gradient.clear();
    return FDTD_OK;
}

int fdtd_set_layer_tangent(fdtd_solver *s, const double *tangent, uint64_t count) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    DeviceGuard guard(s->device);
    for (cudaStream_t stream : {s->stream, s->side, s->layer_stream}) CUDA_TRY(s, cudaStreamSynchronize(stream));
    if (tangent && !s->layers) return fail(s, FDTD_EINVAL, "the grid has no matched layer");
    const uint64_t len[3] = {s->nx + 1, s->ny + 1, s->nz + 1};
    const uint64_t old_factors = s->tangent_factors;
    if (tangent && count != 4 * (len[0] + len[1] + len[2]))
        return fail(s, FDTD_EINVAL, "a tangent of the layer's tables has 4 (nx + ny + nz + 3) values, as fdtd_layer_gradient's");
    for (uint64_t k = 0; tangent && k < count; ++k)
        if (!std::isfinite(tangent[k])) return fail(s, FDTD_EINVAL, "the tangent of the layer's tables is not finite");
    // The old tangent's device tables; the captured graphs and the tape that used them.
    for (void *p : s->tangent_device) {
        auto it = std::find(s->allocations.begin(), s->allocations.end(), p);
        if (it != s->allocations.end()) s->allocations.erase(it);
        cudaFree(p);
    }
    s->tangent_device.clear();
    Tables &g = s->tables;
    for (int a = 0; a < 3; ++a) g.tangent_centre[a] = g.tangent_face[a] = nullptr;
    g.tangent_axes = nullptr, g.tangent_start = nullptr;
    s->tangent = false, s->tangent_factors = 0, s->tangent_valid = false;
    s->tape_valid = false;
    Kept{s}.drop_graphs();
    for (cudaGraphExec_t &graph : s->tape_graph)
        if (graph) cudaGraphExecDestroy(graph), graph = nullptr;
    // (A tape and staging sized for another tangent's factors, or for none, are laid out again.)
    auto drop_tape = [&]() {
        for (void **p : {&s->tape_t, &s->stage_t}) {
            if (!*p) continue;
            auto it = std::find(s->allocations.begin(), s->allocations.end(), *p);
            if (it != s->allocations.end()) s->allocations.erase(it);
            cudaFree(*p);
            *p = nullptr;
        }
        s->device_bytes -= s->precision == FDTD_FP64 ? 8 * old_factors * s->tape_t_steps : 4 * old_factors * s->tape_t_steps;
        s->tape_t_steps = 0;
    };
    if (!tangent) {
        drop_tape();
        return FDTD_OK;
    }
    // Per axis, {keep, push} of the centres and of the faces by coordinate (the entries' order of
    // fdtd_layer_gradient: the six keep tables, then the six push tables).
    std::vector<double2> centre[3], face[3];
    uint64_t at = 0;
    for (int a = 0; a < 3; ++a) {
        centre[a].resize(len[a]), face[a].resize(len[a]);
        for (uint64_t x = 0; x < len[a]; ++x) centre[a][x].x = tangent[at + x], face[a][x].x = tangent[at + len[a] + x];
        at += 2 * len[a];
    }
    for (int a = 0; a < 3; ++a) {
        for (uint64_t x = 0; x < len[a]; ++x) centre[a][x].y = tangent[at + x], face[a][x].y = tangent[at + len[a] + x];
        at += 2 * len[a];
    }
    auto touches = [](const double2 &v) { return v.x != 0.0 || v.y != 0.0; };
    // Each layer cell's axes whose entries at its coordinate (centre, face) or the next (face) the
    // tangent moves, and its first factor in a step's.
    const uint64_t Lc = s->layers, plane = s->pitch * s->ny;
    std::vector<uint8_t> axes(Lc);
    std::vector<uint32_t> start(Lc);
    uint64_t factors = 0;
    for (uint64_t c = 0; c < Lc; ++c) {
        const uint64_t i = s->layer_cells[c], r = i % plane;
        const uint64_t coord[3] = {r % s->pitch, r / s->pitch, i / plane};
        uint8_t bits = 0;
        for (int a = 0; a < 3; ++a)
            if (touches(centre[a][coord[a]]) || touches(face[a][coord[a]]) || touches(face[a][coord[a] + 1]))
                bits |= (uint8_t)(1u << a);
        axes[c] = bits;
        start[c] = (uint32_t)factors;
        factors += 3 * (uint64_t)__builtin_popcount(bits);
        if (factors >= (1ull << 32)) return fail(s, FDTD_EINVAL, "the tangent's factors are too many for 32-bit indices");
    }
    int rc;
    for (int a = 0; a < 3; ++a) {
        const double2 *p;
        if ((rc = upload(s, centre[a].data(), len[a], &p))) return rc;
        g.tangent_centre[a] = p;
        s->tangent_device.push_back(const_cast<double2 *>(p));
        if ((rc = upload(s, face[a].data(), len[a], &p))) return rc;
        g.tangent_face[a] = p;
        s->tangent_device.push_back(const_cast<double2 *>(p));
    }
    const uint8_t *pa;
    const uint32_t *ps;
    if ((rc = upload(s, axes.data(), Lc, &pa))) return rc;
    s->tangent_device.push_back(const_cast<uint8_t *>(pa));
    if ((rc = upload(s, start.data(), Lc, &ps))) return rc;
    s->tangent_device.push_back(const_cast<uint32_t *>(ps));
    g.tangent_axes = pa, g.tangent_start = ps;
    if (old_factors != factors) drop_tape();
    s->tangent_factors = factors;
    s->tangent = true;
    return FDTD_OK;
}

int fdtd_layer_tangent_gradient(const fdtd_solver *s, double *out) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (!out) return set_global(FDTD_EINVAL, "no output");
    if (!s->tangent_valid)
        return set_global(FDTD_EINVAL, "no gradient along a tangent of the layer's tables since the tangent was set");
    *out = s->tangent_gradient;
    return FDTD_OK;
}

int fdtd_layer_gradient(const fdtd_solver *s, double *tables) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    if (!tables) return set_global(FDTD_EINVAL, "no output");
    if (s->layer_gradient.empty())
        return set_global(FDTD_EINVAL, "no gradient of the matched layer's tables: the grid has no layer, or no "
                                       "gradient was taken since the handle was made");
    std::memcpy(tables, s->layer_gradient.data(), sizeof(double) * s->layer_gradient.size());
    return FDTD_OK;
}

int fdtd_reset(fdtd_solver *s) {
    if (!s) return set_global(FDTD_EINVAL, "no solver");
    DeviceGuard guard(s->device);
    const size_t e = s->precision == FDTD_FP64 ? 8 : 4;
    for (int k = 0; k < 2; ++k) {
        CUDA_TRY(s, cudaMemsetAsync(s->u[k], 0, e * s->n_device, s->stream));
        if (s->states) CUDA_TRY(s, cudaMemsetAsync(s->w[k], 0, e * s->states, s->stream));
    }
    if (s->increment) CUDA_TRY(s, cudaMemsetAsync(s->increment, 0, e * s->n_device, s->stream));
    if (s->layers)
        for (int k = 0; k < 2; ++k) CUDA_TRY(s, cudaMemsetAsync(s->layer_state[k], 0, e * kLayerSlots * s->n_device, s->stream));
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
    // The levels are pitched on the device: their rows of nx cells are copied out one plane of
    // rows at a time.
    void *levels[2] = {current, previous};
    const void *sources[2] = {s->u[1], s->increment ? s->increment : s->u[0]};
    std::vector<float> here;
    if (s->increment && previous && !current) {
        here.resize(s->n);
        levels[0] = here.data();
    }
    for (int k = 0; k < 2; ++k) {
        if (!levels[k]) continue;
        CUDA_TRY(s, cudaMemcpy2D(levels[k], e * s->nx, sources[k], e * s->pitch, e * s->nx, s->ny * s->nz,
                                 cudaMemcpyDeviceToHost));
    }
    if (s->increment && previous) {
        // Compensated: the level before is the pressure less its increment.
        const float *p = static_cast<const float *>(levels[0]);
        float *q = static_cast<float *>(previous);
        for (uint64_t i = 0; i < s->n; ++i) q[i] = p[i] - q[i];
    }
    if (branch_current && s->states) CUDA_TRY(s, cudaMemcpy(branch_current, s->w[1], e * s->states, cudaMemcpyDeviceToHost));
    if (branch_previous && s->states) CUDA_TRY(s, cudaMemcpy(branch_previous, s->w[0], e * s->states, cudaMemcpyDeviceToHost));
    if (layer_state && s->layers) {
        // The reference's nine values per cell (fdtd.hpp:2245): the parts, then per axis the
        // velocity of the - face (the + face of the cell below) and of the + face.
        const std::vector<uint32_t> &cells = s->layer_cells;
        std::vector<char> state(e * kLayerSlots * s->n_device);
        CUDA_TRY(s, cudaMemcpy(state.data(), s->layer_state[1], state.size(), cudaMemcpyDeviceToHost));
        char *dst = static_cast<char *>(layer_state);
        const uint64_t strides[3] = {1, s->pitch, s->pitch * s->ny};
        for (uint64_t c = 0; c < s->layers; ++c) {
            const uint64_t i = cells[c];
            for (int k = 0; k < 3; ++k) std::memcpy(dst + e * (9 * c + k), state.data() + e * (kLayerSlots * i + k), e);
            for (int axis = 0; axis < 3; ++axis) {
                const uint64_t below = kLayerSlots * (i - strides[axis]) + 3 + axis, own = kLayerSlots * i + 3 + axis;
                std::memcpy(dst + e * (9 * c + 3 + 2 * axis), state.data() + e * below, e);
                std::memcpy(dst + e * (9 * c + 4 + 2 * axis), state.data() + e * own, e);
            }
        }
    }
    return FDTD_OK;
}

}  // extern "C"

/*
 * fdtd_b200.h — C ABI of the B200 (sm_100a) stepper for acoustic-spaces' low-frequency wave
 * solver.
 *
 * The library steps a grid that the reference's C++ solver laid out: the arrays of
 * WaveSolver::layout() (cpp/include/acoustic_spaces/fdtd.hpp:727-782 of naelolaiz/acoustic-spaces),
 * borrowed for the duration of fdtd_create() and copied to the GPU. Each step does what
 * WaveSolver::run() does (fdtd.hpp:786-904): it records every probe's pressure before the step
 * (summed in double, fdtd.hpp:3525-3533), updates the interior air (fdtd.hpp:242-288), the special
 * (boundary and source) cells with their branch velocities (fdtd.hpp:860-881) and the matched
 * layer (fdtd.hpp:2242-2264), then swaps the two pressure levels and the two branch-velocity sets.
 * In FDTD_FP32 the arithmetic is the reference's, operation for operation, in single precision
 * with no fused multiply-adds and with subnormal results flushed to zero, as the reference's
 * -ffp-contract=off build with its MXCSR flush does: the probes' time series equal the
 * reference's bit for bit. FDTD_FP64 steps the same layout in double (each stored coefficient
 * promoted), the GPU counterpart of the FP64 oracle.
 *
 * Every entry point returns FDTD_OK (0) or a negative status and never aborts; the message of the
 * last failure is fdtd_last_error(handle), or fdtd_global_error() where no handle exists (a failed
 * fdtd_create). Argument errors carry the reference's own wording where the reference refuses
 * the same thing (fdtd.hpp:371-411, engine/gpu.py:495-504).
 *
 * Calls on one handle must not overlap; different handles are independent. Each handle owns one
 * CUDA stream on the device it was created on.
 */
#ifndef FDTD_B200_H
#define FDTD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDTD_B200_ABI_VERSION 3

/* Status codes. */
#define FDTD_OK 0
#define FDTD_EINVAL (-1)  /* a refused argument: the reference's std::invalid_argument / ValueError */
#define FDTD_ECUDA (-2)   /* a CUDA runtime error (message from the runtime) */
#define FDTD_ENOMEM (-3)  /* device or host memory exhausted */
#define FDTD_ENODEV (-4)  /* no CUDA device of compute capability 10.0 */
#define FDTD_ENONFINITE (-5) /* fdtd_run: the pressure stopped being finite (wave.py:1220-1224) */

/* Arithmetic of the fields. */
#define FDTD_FP32 0
#define FDTD_FP64 1
/*
 * Compensated single precision (no counterpart in the reference): the same scheme in float,
 * stepped on each cell's pressure and its increment p_n - p_(n-1) (kept in place of the previous
 * level), every neighbour entering as a difference from the cell's own pressure, and the matched
 * layer's pressure carried on from its own rather than summed from its split parts. Rounding is
 * then relative to the increments, not to the pressures, so that long runs of rooms with a net
 * mass or an open face into the layer stay close to FDTD_FP64, at 16 bytes of traffic per
 * interior cell and step against FDTD_FP32's 12 and FDTD_FP64's 24. Not bit-equal to the
 * reference; fdtd_gradient, fdtd_set_tape and fdtd_set_coefficients refuse it. fdtd_read_state's
 * previous level is the pressure less its increment.
 */
#define FDTD_FP32_COMPENSATED 2

/*
 * The grid's layout, named after WaveSolver::layout()'s arrays (fdtd.hpp:727-782). Counts are
 * given explicitly; the arrays are borrowed only during fdtd_create(). Moving air
 * (fdtd.hpp:1672-2119), which the reference steps on its CPU only (engine/wave.py:1158-1160):
 * with flow_count = nx*ny*nz, each step first carries both pressure levels along with the air
 * (three-stage strong-stability-preserving Runge-Kutta), either the plain way (flow_x, flow_y and
 * the neighbour bits of flow_mask) or, where wind[0] is not NULL, round the solids (wind and
 * loop per axis, flow_mask 1 for a moving cell and 2 at the border of the moving air).
 */
typedef struct fdtd_layout {
    uint64_t nx, ny, nz;          /* "shape": x fastest, sy = nx, sz = nx * ny */
    uint32_t stencil;             /* "stencil": 7 or 19 */
    uint32_t weight_count;        /* length of "weights": 6 or 18 */
    const float *weights;         /* "weights": the update's link weights per direction */
    float centre;                 /* "centre" */
    float total;                  /* "total": the update's weights summed */
    uint32_t scaled;              /* "scaled": 1 with a speed of sound per cell */
    const float *scale;           /* "scale": nx*ny*nz when scaled, else NULL */
    const float *layer_scale;     /* "layer_scale": layer_count when scaled, else NULL */
    const uint8_t *types;         /* "types": nx*ny*nz of 0 solid, 1 interior, 2 special, 3 layer */
    uint64_t special_count;
    const int64_t *special;       /* "special": each special cell's index */
    const uint64_t *link_start;   /* "link_start": special_count + 1 */
    uint64_t link_count;
    const uint8_t *link_direction; /* "link_direction": 0..17, fdtd.hpp:924-927's order */
    const float *link_weight;     /* "link_weight" */
    const float *coef_a;          /* "coef_a", "coef_b", "coef_inv", "source": special_count each */
    const float *coef_b;
    const float *coef_inv;
    const float *source;
    const uint64_t *state_start;  /* "state_start": special_count + 1 */
    uint64_t state_count;
    const int32_t *state_branch;  /* "state_branch": each branch state's branch */
    const float *state_weight;    /* "state_weight" */
    uint64_t branch_count;
    const float *branch_now;      /* "branch_now", "branch_before", "branch_gain": branch_count */
    const float *branch_before;
    const float *branch_gain;
    uint64_t layer_count;
    const int64_t *layer_cells;   /* "layer_cells" */
    /* "keep_x", "keep_face_x", "keep_y", "keep_face_y", "keep_z", "keep_face_z" and the same of
       "push_*": each nx+1, ny+1 or nz+1 long when layer_count > 0, else NULL. */
    const float *keep[6];
    const float *push[6];
    uint64_t probe_count;
    const uint64_t *probe_start;  /* "probe_start": probe_count + 1 */
    const uint64_t *probe_cells;  /* "probe_cells" */
    const double *probe_weights;  /* "probe_weights" */
    uint64_t flow_count;          /* length of "flow_mask": 0 (still air) or nx*ny*nz */
    const float *flow_x, *flow_y; /* "flow_x", "flow_y": the plain form's shifts (cells a step) */
    const uint8_t *flow_mask;     /* "flow_mask" */
    const float *wind[3];         /* "wind_x", "wind_y", "wind_z": the round form's face winds, or NULL */
    const float *loop[3];         /* "loop_x", "loop_y", "loop_z" */
} fdtd_layout;

typedef struct fdtd_solver fdtd_solver;

/* Counts of a created solver, for reports (wave.py:1225-1259's info) and memory planning. */
typedef struct fdtd_info {
    uint64_t cells;          /* nx * ny * nz */
    uint64_t air_cells;      /* interior + special + layer cells (the reference's air_cells) */
    uint64_t interior_cells; /* cells the bulk sweep updates */
    uint64_t special_cells;
    uint64_t links;
    uint64_t branch_states;
    uint64_t layer_cells;
    uint64_t probes;
    uint64_t steps_done;     /* steps since creation or the last reset */
    uint64_t device_bytes;   /* device memory the handle holds */
    int32_t precision;       /* FDTD_FP32, FDTD_FP64 or FDTD_FP32_COMPENSATED */
    int32_t device;          /* CUDA ordinal */
} fdtd_info;

/*
 * Replaces engine/gpu.py:GpuWaveSolver.__init__ (engine/gpu.py:449-540), which packs
 * solver.layout() into WebGPU buffers: copies `layout` to device `device` and creates a solver at
 * rest (both pressure levels, branch velocities and matched-layer state zero).
 * precision: FDTD_FP32, FDTD_FP64 or FDTD_FP32_COMPENSATED. On failure *out is NULL and
 * fdtd_global_error() says why.
 */
int fdtd_create(const fdtd_layout *layout, int precision, int device, fdtd_solver **out);

/*
 * Replaces GpuWaveSolver.run (engine/gpu.py:546-557) and WaveSolver::run (fdtd.hpp:786-904):
 * advances `steps` steps, adding signal[k] at the source on step k, and writes each probe's
 * pressure before each step to out[p * steps + k] (probes x steps, row-major). `signal` and `out`
 * are host buffers (pageable or pinned). The state persists across calls: runs of any lengths
 * concatenate to one run. Synchronous. Returns FDTD_ENONFINITE (after writing `out`) when a
 * probe's pressure is not finite, as wave.py:1220-1224 refuses such a run.
 */
int fdtd_run(fdtd_solver *solver, const float *signal, uint64_t steps, double *out);

/*
 * The same as fdtd_run with device buffers, asynchronous on the handle's stream: d_signal holds
 * `steps` floats, probe p's pressure before step k goes to d_out[p * out_stride + k]
 * (out_stride >= steps). Nothing is checked for finiteness. fdtd_synchronize waits for it.
 */
int fdtd_run_device(fdtd_solver *solver, const float *d_signal, uint64_t steps, double *d_out,
                    uint64_t out_stride);
int fdtd_synchronize(fdtd_solver *solver);

/* The handle's CUDA stream (a cudaStream_t), for callers that order their own work or events
   with fdtd_run_device; NULL for a NULL handle. */
void *fdtd_stream(const fdtd_solver *solver);

/*
 * Per-kernel timing of fdtd_run_device (no counterpart in the reference): with `enable` set, each
 * step's kernels run one after another on the handle's stream, each bracketed by CUDA events, and
 * fdtd_get_timing adds up, since the last call, the milliseconds each kind took — ms[0] the
 * interior sweep, ms[1] the matched layer, ms[2] the special rows, ms[3] the probe records — over
 * *steps steps. The work done is the same.
 */
int fdtd_set_timing(fdtd_solver *solver, int enable);
int fdtd_get_timing(fdtd_solver *solver, double ms[4], uint64_t *steps);

/*
 * The gradient of a loss of the probes' series by the reverse-time (adjoint) stepper; no
 * counterpart in the reference, whose absorption fit searches by finite differences
 * (engine/impedance.py:379-440). From rest, a run of `steps` steps on `signal` gives the series
 * y (probes x steps); given dloss_dy = dL/dy (host, probes x steps), fdtd_gradient returns dL/d of
 * each special row's coef_b and coef_inv (special_count each) and of each branch state's now,
 * before and gain coefficients (state_count each; the state's branch's, fdtd.hpp:797-805), summed
 * over the run in double; any output may be NULL. The forward pass is recomputed in segments of
 * `segment` steps from checkpoints of the whole state kept at each segment's start (0: one
 * segment), recording each step's values at the special rows (and, with a matched layer, each
 * layer cell's eighteen factors of the layer's update: kLayerFactors x layer_count values a step of
 * the segment); the adjoint then steps back through each segment. Either stencil, with or without
 * a speed field, with or without a matched layer (fdtd.hpp:2219-2264); on a grid with a layer
 * the gradient in its twelve tables follows from fdtd_layer_gradient. The solver is left at rest.
 */
int fdtd_gradient(fdtd_solver *solver, const float *signal, uint64_t steps, const double *dloss_dy,
                  uint64_t segment, double *grad_coef_b, double *grad_coef_inv, double *grad_now,
                  double *grad_before, double *grad_gain);

/*
 * The last fdtd_gradient's (or fdtd_gradient_noalloc's) dL/d of the matched layer's twelve tables
 * (no counterpart in the reference; the tables are layer_coefficients', fdtd.hpp:2219-2238), into
 * `tables`: keep_x, keep_face_x, keep_y, keep_face_y, keep_z, keep_face_z, then push_x,
 * push_face_x, ..., push_face_z, the order of fdtd_layout.keep and .push, each of nx + 1, nx + 1,
 * ny + 1, ny + 1, nz + 1, nz + 1 values (4 (nx + ny + nz + 3) in all). The gradient in the layer's
 * damping follows by the chain rule through the tables (their derivative in the damping).
 * FDTD_EINVAL on a grid without a layer, before a gradient, or after gradients without the tables
 * (fdtd_set_gradient_tables).
 */
int fdtd_layer_gradient(const fdtd_solver *solver, double *tables);

/*
 * Whether the handle's gradients also give the matched layer's tables' gradient (1, the default)
 * or the rows' and branch states' only (0; no counterpart in the reference). Without the tables a
 * gradient records none of the layer's per-step factors (18 values a layer cell a step of the
 * segment) and steps back through the layer on its carried values alone: the walls' gradient is
 * the same, to the bit, at the cost of the layer's adjoint only. It also decides a following
 * taped run's kind (fdtd_set_tape): without the tables, a grid with a matched layer keeps the
 * rows' trajectory where it fits, as grids without one do, and its gradient recomputes nothing.
 */
int fdtd_set_gradient_tables(fdtd_solver *solver, int enable);

/*
 * A tangent of the matched layer's tables (no counterpart in the reference): the derivative of each
 * table entry in one parameter θ — the layer's damping, say (layer_coefficients, fdtd.hpp:2219-2238)
 * — in fdtd_layer_gradient's order and count (4 (nx + ny + nz + 3) values). While it is set,
 * gradients give dL/dθ = sum over the entries of dL/d(entry) d(entry)/dθ (fdtd_layer_tangent_gradient)
 * in place of the twelve tables' gradient: the forward records three factors a step per layer cell
 * and axis along which the tangent moves an entry at the cell's coordinate (or the next one's
 * face), not eighteen, each cell sums its products over the steps, and a taped run (fdtd_set_tape)
 * keeps those factors of every step beside the rows' trajectory where both fit, so that the
 * gradient recomputes nothing. The walls' gradient is the same. NULL clears it. FDTD_EINVAL on a
 * grid without a layer, a count other than the tables', or a value that is not finite. Drops the
 * handle's tape.
 */
int fdtd_set_layer_tangent(fdtd_solver *solver, const double *tangent, uint64_t count);

/* The last gradient's dL/dθ along the layer tables' tangent (fdtd_set_layer_tangent); FDTD_EINVAL
 * when no gradient ran since the tangent was set. */
int fdtd_layer_tangent_gradient(const fdtd_solver *solver, double *out);

/*
 * The tape of a run for a gradient that follows (no counterpart in the reference). With `segment`
 * > 0, each fdtd_run that starts from rest keeps on the device the state at every multiple of
 * `segment` steps before its end, and a copy of its drive; a following fdtd_gradient of the same
 * drive and steps with the same `segment` starts from those states instead of running the forward
 * pass again, so that a fit's forward run and its gradient together step the grid twice rather
 * than three times. The result is the same to the bit. 0 turns the tape off. The states take
 * (steps / segment - 1) x (2 levels + 2 branch-velocity sets, and with a matched layer its
 * state) of device memory, kept by the handle. Where the trajectory fits the budget
 * (fdtd_set_tape_budget) the tape keeps it instead; on a grid with a matched layer only for
 * gradients without the layer's tables (fdtd_set_gradient_tables) or along a tangent of them
 * (fdtd_set_layer_tangent, whose factors the tape then keeps too).
 */
int fdtd_set_tape(fdtd_solver *solver, uint64_t segment);

/*
 * The device memory a tape may take for the trajectory (no counterpart in the reference). A taped
 * run keeps, in place of checkpoints, every level of the special rows' values and branch
 * velocities ((steps + 2) * (special rows + branch states) elements) when that fits in `bytes`;
 * the gradient then recomputes nothing. UINT64_MAX (the default): half the device memory free at
 * the run. 0: always checkpoints.
 */
int fdtd_set_tape_budget(fdtd_solver *solver, uint64_t bytes);

/*
 * Chooses the launch shapes for this grid (no counterpart in the reference): from rest, steps
 * `trial_steps` steps (0: 8) with each candidate and keeps the fastest by CUDA events — first the
 * interior sweep's tile shape (each of the ten shapes of fdtd_tiles that fits a multiprocessor,
 * each with 1/4, 1/2, 1 and 2 times the default planes a tile, within 8 to 64), then, with the best
 * tiles, the count of blocks per multiprocessor of the matched-layer and special-row kernels and
 * the six arrangements of the step's kernels on the streams (fdtd_set_streams), then the tiles again; the
 * best few whole choices are timed three times more and the fastest kept — and resets the state.
 * The chosen counts are written to *layer_per_sm and *special_per_sm when given (0: one thread a
 * cell); fdtd_get_tiles gives the rest. Results do not depend on any of these choices. Refused
 * after steps (fdtd_reset first).
 */
int fdtd_autotune(fdtd_solver *solver, uint64_t trial_steps, int *layer_per_sm, int *special_per_sm);

/* The interior sweep's tiles (no counterpart in the reference). */
typedef struct fdtd_tiles {
    int shape;          /* 0: 64 x 16 cells, 5 stages; 1: 128 x 16, 4; 2: 64 x 32, 4; 3: 32 x 32, 5 (128
                         * threads a block, a column a thread); 4, 5, 6: shapes 0, 1, 2 with 256
                         * threads a block; 7: shape 0 with a pair of columns a thread; 8: 128 x 16,
                         * 4 stages, 256 threads, pairs; 9: 64 x 16, 5 stages, 256 threads, pairs */
    int tile_x, tile_y; /* cells of a tile along x and y */
    int stages;         /* plane stages in a block's shared-memory ring */
    uint64_t planes;    /* planes of a tile, at most (a tile marches them along z) */
    uint32_t tiles;     /* tiles, one block each */
    int blocks_per_sm;  /* resident blocks of the sweep a multiprocessor */
    int concurrent;     /* how a step's kernels share the streams (fdtd_set_streams: 0 to 5) */
    int threads;        /* threads a block of the sweep */
    int cols;           /* adjacent columns a thread (1, or 2: the 7-point stencil a pair at a time) */
} fdtd_tiles;

/*
 * Sets the interior sweep's tile shape (an index of fdtd_tiles.shape) and planes a tile (1 to
 * 1024), as fdtd_autotune would choose them; the state is kept and results are unchanged, to the
 * bit. FDTD_EINVAL for a shape out of range or one whose shared memory does not fit a
 * multiprocessor in the handle's precision. Waits for the handle's work.
 */
int fdtd_set_tiles(fdtd_solver *solver, int shape, uint64_t planes);

/* The interior sweep's present tiles. */
int fdtd_get_tiles(const fdtd_solver *solver, fdtd_tiles *out);

/*
 * How a step's kernels share the streams, as fdtd_autotune may choose (no counterpart in the
 * reference): 1 (the default), the interior sweep on the handle's stream, the matched layer and the
 * special rows (with the probes) on streams of their own; 2, the layer and then the special rows
 * on one stream beside the sweep; 3, the special rows after the sweep on the handle's stream, the
 * layer beside them; 0, all one after another on the handle's stream; 4 and 5, as 1 and 2 with
 * the special rows launched at the device's highest stream priority, so that their blocks run
 * beside the sweep's from the step's start. Results are the same to the bit. FDTD_EINVAL outside
 * 0 to 5. Waits for the handle's work.
 */
int fdtd_set_streams(fdtd_solver *solver, int concurrent);

/*
 * The gradient's reverse step: at most `far_per_sm` blocks an SM for its launch of the special rows
 * and corrected cells far from the matched layer, `near_per_sm` for its launch of the rest and the
 * layer's cells (0: a block for every 128 of them; no counterpart in the reference). Fewer blocks
 * let the launches run beside one another and the interior sweep. Results are the same to the bit.
 */
int fdtd_set_adjoint_launch(fdtd_solver *solver, int far_per_sm, int near_per_sm);

/*
 * The device address and size of plane z of the current (which 0) or previous (1) pressure level
 * between runs (no counterpart in the reference): pitch * ny elements, contiguous, pitch the row
 * length rounded up to 16 cells. A grid split into slabs of planes across ranks exchanges its
 * boundary planes through these after each step; the addresses change with the levels' roles, so
 * ask again after every run.
 */
int fdtd_level_plane(fdtd_solver *solver, uint64_t z, int which, void **ptr, uint64_t *bytes);

/* A plane of one grid of a group copied, after each step, into a plane of another (fdtd_run_linked). */
typedef struct fdtd_plane_link {
    uint32_t from, to;     /* indices of the solvers in the group */
    uint64_t from_plane;   /* plane z of the source's grid (one of its own planes) */
    uint64_t to_plane;     /* plane z of the destination's grid: solid there (a ghost plane) */
} fdtd_plane_link;

/*
 * Steps a group of grids together, `steps` steps, each the z-slab of one larger grid (no
 * counterpart in the reference, whose solver holds one grid on one machine): after every step,
 * each link copies the source's plane of the new pressure into the destination's plane — a slab's
 * first and last planes into its neighbours' ghost planes. The ordering lives on the devices: a
 * solver's step waits for the planes its neighbours sent it, each copy runs on its source's stream
 * after the source's step (cudaMemcpyPeerAsync between devices, with peer access enabled), and the
 * host enqueues the whole run without waiting, so no step costs a round trip to the host. Each
 * solver takes its drive from d_signals[h] and records its probes into d_outs[h] (device memory,
 * as fdtd_run_device; out_stride between probes). The grids' planes must be of one size, a link's
 * destination plane solid, the solvers distinct and of one precision. Returns when the work is
 * enqueued; each solver's stream ends with the run (fdtd_synchronize, or fdtd_stream).
 */
int fdtd_run_linked(fdtd_solver *const *solvers, uint32_t count, const fdtd_plane_link *links, uint32_t link_count,
                    const float *const *d_signals, uint64_t steps, double *const *d_outs, uint64_t out_stride);

/*
 * The failure path of the kernels' bounded waits, on its own (no counterpart in the reference):
 * a kernel polls a device flag that nothing sets, at most `spins` times (1 to 2^24), then reports
 * through the error flag as a kernel whose wait gave up does; returns that status (FDTD_ECUDA
 * and its message). The handle stays usable. No GPU is faulted or hung: the wait is bounded.
 */
int fdtd_test_wait(fdtd_solver *solver, uint32_t spins);

/* Sets those launch shapes directly (0 to 64 blocks per multiprocessor; 0: one thread a cell). */
int fdtd_set_launch(fdtd_solver *solver, int layer_per_sm, int special_per_sm);

/*
 * New material coefficients for the handle's grid (no counterpart in the reference, which builds a
 * new solver for new materials): each non-NULL array replaces the layout's — coef_b and coef_inv
 * one per special row (special_count), branch_now, branch_before and branch_gain one per branch
 * (branch_count, gathered per state as fdtd_create gathers them). The geometry, the state and the
 * adjoint's tables stay (their products with coef_inv are formed anew), so that a fit steps one
 * handle through its iterations; stepping and gradients then equal those of a handle created with
 * the new coefficients, to the bit. Waits for the handle's work; drops the tape.
 */
int fdtd_set_coefficients(fdtd_solver *solver, const float *coef_b, const float *coef_inv, const float *branch_now,
                          const float *branch_before, const float *branch_gain);

/* Bytes of the static device pool of fdtd_gradient_noalloc: 16 MiB, held on every device the
   library runs on until the process exits. */
#define FDTD_GRADIENT_STATIC_BYTES (16ull << 20)

/*
 * fdtd_gradient without a device allocation; it has no counterpart in the reference. It computes
 * the same gradient with the same kernels in the same order, but every device buffer it needs —
 * the adjoint's tables and levels, the drive and dL/dy, the trajectory, the checkpoints, the sums —
 * is carved from a pool of FDTD_GRADIENT_STATIC_BYTES that the library keeps in static device
 * memory, so the call makes no cudaMalloc or cudaFree and keeps nothing on the handle. It is for
 * callers that must not allocate while they run: cudaMalloc and cudaFree can synchronize the whole
 * device and so stall every other stream on it (another solver's steps, a renderer's or a model's
 * kernels), and a process whose device memory belongs to a caching allocator (PyTorch's) may have
 * none left to give. A run whose buffers do not fit the pool is refused with FDTD_EINVAL before any
 * device work, the message giving the bytes it needs (take fewer steps, a longer `segment`, or
 * fdtd_gradient). Every call looks up the pool's device address (cudaGetSymbolAddress) with the
 * handle's device current, so a context destroyed and made again (cudaDeviceReset) leaves no stale
 * address behind; make the first call on a device before any stream capture on it, since that
 * lookup loads the library's device code there. A tape kept by fdtd_set_tape supplies the
 * checkpoints, which then take no room in the pool. There is one pool per device, shared by every handle and kept between calls:
 * what must start at zero is cleared by each call, but calls whose work overlaps on a device — from
 * two threads, or on two handles — race on the pool and give wrong results. A call returns only
 * when its work has ended, so calls made one after another are safe. Arguments, results and
 * refusals are otherwise those of fdtd_gradient.
 */
int fdtd_gradient_noalloc(fdtd_solver *solver, const float *signal, uint64_t steps, const double *dloss_dy,
                          uint64_t segment, double *grad_coef_b, double *grad_coef_inv, double *grad_now,
                          double *grad_before, double *grad_gain);

/* Replaces WaveSolver::reset (fdtd.hpp:906-915): silences the grid. */
int fdtd_reset(fdtd_solver *solver);

/* Frees the handle and its device memory; NULL is accepted. */
int fdtd_destroy(fdtd_solver *solver);

/* Counts of the solver. */
int fdtd_get_info(const fdtd_solver *solver, fdtd_info *info);

/*
 * Copies the state to host buffers, each optional (NULL skips it): the current pressure and the
 * one a step before (nx*ny*nz elements of float in FDTD_FP32, double in FDTD_FP64), the current
 * and the previous branch velocities (state_count each) and the matched layer's state
 * (9 * layer_count, the reference's per-cell order p_x, p_y, p_z, u-_x, u+_x, u-_y, u+_y, u-_z,
 * u+_z, fdtd.hpp:2245). For parity checks of the whole field, not only the probes.
 */
int fdtd_read_state(const fdtd_solver *solver, void *current, void *previous, void *branch_current,
                    void *branch_previous, void *layer_state);

/* The message of the handle's last failure ("" if none). */
const char *fdtd_last_error(const fdtd_solver *solver);

/* The message of the calling thread's last failure without a handle (fdtd_create, queries). */
const char *fdtd_global_error(void);

/*
 * Replaces engine/gpu.py:gpu_name (engine/gpu.py:302-311): the device's name as
 * "<name> (CUDA sm_<major><minor>, <memory> GiB)" into buf. FDTD_ENODEV without a device.
 */
int fdtd_device_name(int device, char *buf, size_t size);

/* CUDA devices of compute capability 10.x visible to the process (0 when none). */
int fdtd_device_count(void);

/* ---- fitted walls: the cut of a convex room by the grid (set-up, not stepping) ---- */

/* Planes of a convex room, and pieces of its walls, at most. */
#define FDTD_CUT_MAX_PLANES 64
#define FDTD_CUT_MAX_PIECES 256

/* A convex room P = {x : normals[f] . x <= offsets[f] for every plane f} (unit normals, pointing
 * out of the room; metres), on a grid of nx x ny x nz cells of `cell` metres whose first cell's
 * corner is `origin` (cell (i, j, k) spans origin + (i, j, k) cell .. + cell, the doubles of the
 * reference's cut_grid, fdtd.hpp:1620-1634). */
typedef struct fdtd_cut_room {
    const double *normals; /* planes x 3 */
    const double *offsets; /* planes */
    const uint8_t *open;   /* planes: nonzero for a face left open (no wall), NULL for none */
    uint32_t planes;
    double origin[3];
    double cell;
    uint64_t nx, ny, nz;
    /* Optional (pieces 0: each wall one piece, its plane's): the walls cut into pieces, as the
     * triangles of a mesh carry materials of their own. Piece k lies on the wall plane
     * piece_plane[k] and is the part of it inside the half-spaces piece_edges[4 e .. 4 e + 3]
     * (normal, offset: n . x <= d) for e in piece_start[k] .. piece_start[k + 1] - 1; the pieces
     * of a plane cover its wall face without overlapping. */
    uint32_t pieces;
    const uint32_t *piece_plane;  /* pieces */
    const uint32_t *piece_start;  /* pieces + 1 */
    const double *piece_edges;    /* 4 per edge */
} fdtd_cut_room;

/* The cells the walls' planes cut, in no particular order (the library allocates the arrays;
 * fdtd_cut_free releases them): each cell's index (x fastest); the volume of its air inside every
 * wall's plane (in cells^3; the rest of the cell is its air outside them), the area of each of its
 * faces (-x, +x, -y, +y, -z, +z; in cell faces, 6 a cell) on that inner side, each wall's area
 * in the cell (`planes` values a cell: one a plane, 0 for an open plane; or, for a room given in
 * pieces, one a piece, `planes` then the count of pieces), and the area of the walls' planes between
 * the inner and the outer air that no wall covers (beyond a face left open: the two sides of the
 * cell's air meet there). */
typedef struct fdtd_cut_cells {
    uint64_t cells;
    uint32_t planes;
    uint64_t *cell;
    double *volume;
    double *face_area;
    double *cap;
    double *bare;
} fdtd_cut_cells;

/*
 * The FP64 fractions of fitted (cut-cell) walls for a convex room, on the GPU (no counterpart
 * for this kind of room in the reference, whose exact fit of a triangle mesh runs on the host:
 * cut_cells.hpp, CutCells, measured per cell in set_up_fitted, fdtd.hpp:970-1217). One thread a
 * cell: each cell that a wall's plane cuts is clipped by every plane that cuts it (a wall's plane
 * splits the cell, an open plane only bounds the walls' faces). Returns FDTD_OK with
 * *out filled, or a status with fdtd_cut_error's message (no device: FDTD_ENODEV).
 */
int fdtd_cut_convex(const fdtd_cut_room *room, int device, fdtd_cut_cells *out);

/* Releases the arrays of a fdtd_cut_cells (NULL and a zeroed struct are accepted). */
void fdtd_cut_free(fdtd_cut_cells *cells);

/* The message of the calling thread's last failed fdtd_cut_convex. */
const char *fdtd_cut_error(void);

/* FDTD_B200_ABI_VERSION of the library. */
int fdtd_abi_version(void);

/* A digest of the sources and flags the library was built from (no counterpart in the
 * reference): the Python loader refuses a library whose digest is not its sources'. */
const char *fdtd_build_id(void);

#ifdef __cplusplus
}
#endif

#endif /* FDTD_B200_H */

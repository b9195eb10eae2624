/*
 * ORACLE / TEST INFRASTRUCTURE ONLY — see fdtd_oracle.h. A restatement, single-threaded and
 * written for reading, of WaveSolver::run (cpp/include/acoustic_spaces/fdtd.hpp:786-904 of
 * naelolaiz/acoustic-spaces). Built with -ffp-contract=off so that no multiply-add is fused.
 */
#define _POSIX_C_SOURCE 200809L
#include "fdtd_oracle.h"
#include "../acoustic_spaces_b200/csrc/fdtd_compensated.h"

#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#if defined(__SSE__) || defined(__x86_64__)
#include <xmmintrin.h>
#define ORACLE_HAS_MXCSR 1
#endif

/*
 * Threads. Within a step every write is to the next level (or a cell's own branch and layer
 * state) and every read of a neighbour is of the current level, so the cells, rows and layer
 * cells split across threads in contiguous ranges with one barrier per step, and no result
 * changes. Grids of ORACLE_PARALLEL_CELLS cells or more use oracle_threads() threads.
 */
#define ORACLE_PARALLEL_CELLS (1u << 16)

int oracle_threads(void) {
    const char *env = getenv("ORACLE_THREADS");
    long t = env ? atol(env) : sysconf(_SC_NPROCESSORS_ONLN);
    return (int)(t < 1 ? 1 : (t > 64 ? 64 : t));
}

typedef struct oracle_job {
    oracle_solver *s;
    const float *signal;
    uint64_t steps;
    double *out;
    int tid, threads;
    pthread_barrier_t *barrier;
} oracle_job;

/* This thread's share [*lo, *hi) of count items. */
static void share(const oracle_job *j, uint64_t count, uint64_t *lo, uint64_t *hi) {
    *lo = count * (uint64_t)j->tid / (uint64_t)j->threads;
    *hi = count * (uint64_t)(j->tid + 1) / (uint64_t)j->threads;
}

static void step_barrier(const oracle_job *j) {
    if (j->threads > 1) pthread_barrier_wait(j->barrier);
}

/* The reference's flush of subnormal single-precision results (fdtd.hpp:316-336) is a per-thread
   flag: every thread that steps float sets it for itself. */
static unsigned flush_enter(int flush) {
#ifdef ORACLE_HAS_MXCSR
    const unsigned saved = _mm_getcsr();
    if (flush) _mm_setcsr(saved | 0x8040u);
    return saved;
#else
    (void)flush;
    return 0;
#endif
}

static void flush_leave(int flush, unsigned saved) {
#ifdef ORACLE_HAS_MXCSR
    if (flush) _mm_setcsr(saved);
#else
    (void)flush, (void)saved;
#endif
}

static char g_error[512];

static int fail(const char *message) {
    snprintf(g_error, sizeof g_error, "%s", message);
    return FDTD_EINVAL;
}

const char *oracle_error(void) { return g_error; }

/* The directions of fdtd.hpp:924-927: six axial, then the twelve edge neighbours. */
static const int kSteps[18][3] = {
    {-1, 0, 0},  {1, 0, 0},  {0, -1, 0}, {0, 1, 0},   {0, 0, -1}, {0, 0, 1},
    {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 1, 0},   {-1, 0, -1}, {1, 0, -1},
    {-1, 0, 1},  {1, 0, 1},  {0, -1, -1}, {0, 1, -1}, {0, -1, 1},  {0, 1, 1}};

struct oracle_solver {
    int precision;
    uint64_t nx, ny, nz, n, sy, sz;
    int wide;
    float axial, diagonal, centre, total;
    int scaled;
    float *scale, *layer_scale;
    uint8_t *types;
    uint64_t specials, links, states, branches, layers, probes;
    int64_t *special;
    uint64_t *link_start, *state_start, *probe_start, *probe_cells;
    uint8_t *link_direction;
    float *link_weight, *coef_a, *coef_b, *coef_inv, *source, *state_weight;
    float *state_now, *state_before, *state_gain; /* each state's branch's, as run() gathers them */
    int64_t *layer_cells;
    float *keep[6], *push[6];
    uint64_t axis_len[3];
    double *probe_weights;
    int64_t offset[18];
    /* the state: u0 the previous level, u1 the current one at the start of a run */
    void *u0, *u1, *w0, *w1;
    void *layer_state; /* 9 per layer cell */
    void *term;        /* each state's term of the step */
    /* ORACLE_FP32C: each cell's increment p_n - p_(n-1) (the previous level is not kept), and
       the residuals of the constant mode (compensated_residuals) */
    float *increment;
    float residual, *row_residual;
    /* moving air (fdtd.hpp:1672-2119): the plain form's shifts and neighbour bits, or the round
       form's face winds and loops (round); the carry's two stage fields (T, zero where solid) */
    int flowing, round;
    float *flow_x, *flow_y, *wind[3], *loop[3];
    uint8_t *flow_mask;
    void *t1, *t2;
};

static void *copy_of(const void *src, size_t bytes) {
    void *p = malloc(bytes ? bytes : 1);
    if (p && src && bytes) memcpy(p, src, bytes);
    return p;
}

int oracle_create(const fdtd_layout *L, int precision, oracle_solver **out) {
    *out = NULL;
    if (precision != ORACLE_FP32 && precision != ORACLE_FP64 && precision != ORACLE_FP32C)
        return fail("precision is FP32, FP64 or FP32 compensated");
    if (L->stencil != 7 && L->stencil != 19) return fail("the stencil has 7 or 19 points");
    if (L->flow_count && L->flow_count != L->nx * L->ny * L->nz) return fail("moving air needs one mask per cell");
    if (L->flow_count && precision == ORACLE_FP32C) return fail("the compensated form steps still air only");
    oracle_solver *s = calloc(1, sizeof *s);
    if (!s) return FDTD_ENOMEM;
    s->precision = precision;
    s->nx = L->nx, s->ny = L->ny, s->nz = L->nz;
    s->n = L->nx * L->ny * L->nz;
    s->sy = L->nx, s->sz = L->nx * L->ny;
    s->wide = L->stencil == 19;
    s->axial = L->weights[0];
    s->diagonal = s->wide ? L->weights[6] : 0.0f;
    s->centre = L->centre, s->total = L->total;
    s->scaled = L->scaled != 0;
    s->specials = L->special_count, s->links = L->link_count, s->states = L->state_count;
    s->branches = L->branch_count, s->layers = L->layer_count, s->probes = L->probe_count;
    s->types = copy_of(L->types, s->n);
    s->scale = s->scaled ? copy_of(L->scale, 4 * s->n) : NULL;
    s->layer_scale = s->scaled ? copy_of(L->layer_scale, 4 * s->layers) : NULL;
    s->special = copy_of(L->special, 8 * s->specials);
    s->link_start = copy_of(L->link_start, 8 * (s->specials + 1));
    s->state_start = copy_of(L->state_start, 8 * (s->specials + 1));
    s->link_direction = copy_of(L->link_direction, s->links);
    s->link_weight = copy_of(L->link_weight, 4 * s->links);
    s->coef_a = copy_of(L->coef_a, 4 * s->specials);
    s->coef_b = copy_of(L->coef_b, 4 * s->specials);
    s->coef_inv = copy_of(L->coef_inv, 4 * s->specials);
    s->source = copy_of(L->source, 4 * s->specials);
    s->state_weight = copy_of(L->state_weight, 4 * s->states);
    s->state_now = malloc(4 * s->states + 4);
    s->state_before = malloc(4 * s->states + 4);
    s->state_gain = malloc(4 * s->states + 4);
    for (uint64_t j = 0; j < s->states; ++j) {
        const int32_t b = L->state_branch[j];
        if (b < 0 || (uint64_t)b >= s->branches) return fail("a branch state has no branch");
        s->state_now[j] = L->branch_now[b];
        s->state_before[j] = L->branch_before[b];
        s->state_gain[j] = L->branch_gain[b];
    }
    s->layer_cells = copy_of(L->layer_cells, 8 * s->layers);
    s->axis_len[0] = s->nx, s->axis_len[1] = s->ny, s->axis_len[2] = s->nz;
    for (int k = 0; k < 6; ++k) {
        const uint64_t len = s->axis_len[k / 2] + 1;
        s->keep[k] = s->layers ? copy_of(L->keep[k], 4 * len) : NULL;
        s->push[k] = s->layers ? copy_of(L->push[k], 4 * len) : NULL;
    }
    s->probe_start = copy_of(L->probe_start, 8 * (s->probes + 1));
    const uint64_t pc = s->probe_start[s->probes];
    s->probe_cells = copy_of(L->probe_cells, 8 * pc);
    s->probe_weights = copy_of(L->probe_weights, 8 * pc);
    for (int k = 0; k < 18; ++k)
        s->offset[k] = kSteps[k][0] + kSteps[k][1] * (int64_t)s->sy + kSteps[k][2] * (int64_t)s->sz;
    const size_t e = precision == ORACLE_FP64 ? 8 : 4;
    if (precision == ORACLE_FP32C) {
        s->increment = calloc(s->n + 1, 4);
        s->row_residual = malloc(4 * s->specials + 4);
        fdtd_compensated_residuals(L, &s->residual, s->row_residual);
    }
    if (L->flow_count) {
        s->flowing = 1;
        s->round = L->wind[0] != NULL;
        s->flow_mask = copy_of(L->flow_mask, s->n);
        if (s->round) {
            for (int d = 0; d < 3; ++d) {
                s->wind[d] = copy_of(L->wind[d], 4 * s->n);
                s->loop[d] = copy_of(L->loop[d], 4 * s->n);
            }
        } else {
            s->flow_x = copy_of(L->flow_x, 4 * s->n);
            s->flow_y = copy_of(L->flow_y, 4 * s->n);
        }
        s->t1 = calloc(s->n + 1, e);
        s->t2 = calloc(s->n + 1, e);
    }
    s->u0 = calloc(s->n + 1, e);
    s->u1 = calloc(s->n + 1, e);
    s->w0 = calloc(s->states + 1, e);
    s->w1 = calloc(s->states + 1, e);
    s->term = calloc(s->states + 1, e);
    s->layer_state = calloc(9 * s->layers + 1, e);
    if (!s->u0 || !s->u1) return FDTD_ENOMEM;
    *out = s;
    return FDTD_OK;
}

/*
 * Moving air (fdtd.hpp:1946-2119): -v . grad q of cell i over a step, and the three stages of the
 * strong-stability-preserving Runge-Kutta method. T float rounds as the reference's float code
 * (its constants 1/12 and 2/3 formed in float); T double promotes them.
 */
#define DEFINE_CARRY(T, SUFFIX)                                                                   \
    /* gradient, fdtd.hpp:1946-1967: along an axis of stride st, the mask's four bits m */       \
    static T gradient_##SUFFIX(const T *q, uint64_t i, uint64_t st, unsigned m, float shift) {   \
        if ((m & 15u) == 15u)                                                                     \
            return ((T)8 * (q[i + st] - q[i - st]) - (q[i + 2 * st] - q[i - 2 * st])) *          \
                   ((T)1 / (T)12);                                                                \
        const int below = (m & 1u) != 0, above = (m & 2u) != 0;                                   \
        const T c = q[i];                                                                         \
        T faces = 0, loops = 0;                                                                   \
        if (above) {                                                                              \
            faces += (T)0.5 * (q[i + st] - c);                                                    \
            if (m & 8u) loops += q[i + st] - q[i + 2 * st];                                       \
        } else if (shift < 0.0f) {                                                                \
            faces -= c;                                                                           \
        }                                                                                         \
        if (below) {                                                                              \
            faces += (T)0.5 * (c - q[i - st]);                                                    \
            if (m & 4u) loops += q[i - 2 * st] - q[i - st];                                       \
        } else if (shift > 0.0f) {                                                                \
            faces += c;                                                                           \
        }                                                                                         \
        if (below && above) loops += q[i + st] - q[i - st];                                       \
        return faces + loops * ((T)1 / (T)12);                                                    \
    }                                                                                             \
    /* carried, fdtd.hpp:1970-1974: the plain way */                                             \
    static T carried_##SUFFIX(const oracle_solver *s, const T *q, uint64_t i) {                  \
        const float sx = s->flow_x[i], sy = s->flow_y[i];                                        \
        const unsigned m = s->flow_mask[i];                                                       \
        return -((T)sx * gradient_##SUFFIX(q, i, 1, m & 15u, sx) +                                \
                 (T)sy * gradient_##SUFFIX(q, i, s->sy, m >> 4, sy));                             \
    }                                                                                             \
    /* carried_round, fdtd.hpp:1978-1991; carried_border, fdtd.hpp:1996-2020 */                  \
    static T carried_round_##SUFFIX(const oracle_solver *s, const T *q, uint64_t i) {            \
        const uint64_t stride[3] = {1, s->sy, s->sz};                                             \
        const int border = s->flow_mask[i] == 2;                                                  \
        const T c = q[i];                                                                         \
        T sum = 0;                                                                                \
        for (int d = 0; d < 3; ++d) {                                                             \
            const uint64_t st = stride[d];                                                        \
            const float *w = s->wind[d], *l = s->loop[d];                                         \
            const T above = q[i + st], below = q[i - st];                                         \
            if (!border) {                                                                        \
                sum += (T)0.5 * ((T)w[i] * (above - c) + (T)w[i - st] * (c - below)) +            \
                       (T)l[i] * (above - q[i + 2 * st]) + (T)l[i - st] * (above - below) +       \
                       (T)l[i - 2 * st] * (q[i - 2 * st] - below);                                \
                continue;                                                                         \
            }                                                                                     \
            if (s->flow_mask[i + st]) {                                                           \
                sum += (T)0.5 * (T)w[i] * (above - c);                                            \
            } else if (w[i] < 0.0f) {                                                             \
                sum -= (T)w[i] * c;                                                               \
            }                                                                                     \
            if (s->flow_mask[i - st]) {                                                           \
                sum += (T)0.5 * (T)w[i - st] * (c - below);                                       \
            } else if (w[i - st] > 0.0f) {                                                        \
                sum += (T)w[i - st] * c;                                                          \
            }                                                                                     \
            sum += (T)l[i] * (above - q[i + 2 * st]) + (T)l[i - st] * (above - below) +           \
                   (T)l[i - 2 * st] * (q[i - 2 * st] - below);                                    \
        }                                                                                         \
        return -sum;                                                                              \
    }                                                                                             \
    static int still_##SUFFIX(const oracle_solver *s, uint64_t i) {                               \
        return s->round ? s->flow_mask[i] == 0 : (s->flow_x[i] == 0.0f && s->flow_y[i] == 0.0f);  \
    }                                                                                             \
    static T moved_##SUFFIX(const oracle_solver *s, const T *q, uint64_t i) {                     \
        return s->round ? carried_round_##SUFFIX(s, q, i) : carried_##SUFFIX(s, q, i);            \
    }                                                                                             \
    /* carry, fdtd.hpp:2049-2097: the three stages over this thread's cells [i0, i1) */          \
    static void carry_##SUFFIX(const oracle_job *job, T *q, uint64_t i0, uint64_t i1) {          \
        const oracle_solver *s = job->s;                                                          \
        T *t1 = (T *)s->t1, *t2 = (T *)s->t2;                                                     \
        for (uint64_t i = i0; i < i1; ++i) {                                                      \
            if (s->types[i] == 0) continue;                                                       \
            t1[i] = still_##SUFFIX(s, i) ? q[i] : q[i] + moved_##SUFFIX(s, q, i);                  \
        }                                                                                         \
        step_barrier(job);                                                                        \
        for (uint64_t i = i0; i < i1; ++i) {                                                      \
            if (s->types[i] == 0) continue;                                                       \
            t2[i] = still_##SUFFIX(s, i) ? q[i]                                                   \
                                         : (T)0.75 * q[i] + (T)0.25 * (t1[i] + moved_##SUFFIX(s, t1, i)); \
        }                                                                                         \
        step_barrier(job);                                                                        \
        for (uint64_t i = i0; i < i1; ++i) {                                                      \
            if (s->types[i] == 0 || still_##SUFFIX(s, i)) continue;                               \
            q[i] = q[i] + ((T)2 / (T)3) * ((t2[i] + moved_##SUFFIX(s, t2, i)) - q[i]);            \
        }                                                                                         \
        step_barrier(job);                                                                        \
    }

DEFINE_CARRY(float, f32)
DEFINE_CARRY(double, f64)

/*
 * One instantiation per arithmetic type T. Each expression keeps the reference's operands in the
 * reference's order; with T float every operation rounds to float as the reference's does.
 */
#define DEFINE_STEPPER(T, NAME, FLUSH, SUFFIX)                                                    \
    static void NAME(const oracle_job *job) {                                                    \
        oracle_solver *s = job->s;                                                               \
        const float *signal = job->signal;                                                       \
        const uint64_t steps = job->steps;                                                       \
        double *out = job->out;                                                                  \
        T *term = (T *)s->term, *lstate = (T *)s->layer_state;                                   \
        const uint64_t sy = s->sy, sz = s->sz;                                                   \
        const T axial = (T)s->axial, diagonal = (T)s->diagonal, centre = (T)s->centre;           \
        const T total = (T)s->total;                                                             \
        uint64_t i0, i1, k0, k1, c0, c1;                                                         \
        share(job, s->n, &i0, &i1);                                                              \
        share(job, s->specials, &k0, &k1);                                                       \
        share(job, s->layers, &c0, &c1);                                                         \
        const unsigned csr = flush_enter(FLUSH);                                                 \
        for (uint64_t step = 0; step < steps; ++step) {                                          \
            /* the levels' roles by the step's parity (the swap of fdtd.hpp:884-885) */          \
            T *a = (T *)(step & 1 ? s->u1 : s->u0), *b = (T *)(step & 1 ? s->u0 : s->u1);        \
            T *wa = (T *)(step & 1 ? s->w1 : s->w0), *wb = (T *)(step & 1 ? s->w0 : s->w1);      \
            /* record (fdtd.hpp:3525-3533) */                                                    \
            for (uint64_t p = 0; job->tid == 0 && p < s->probes; ++p) {                          \
                double value = 0.0;                                                              \
                for (uint64_t k = s->probe_start[p]; k < s->probe_start[p + 1]; ++k)             \
                    value += s->probe_weights[k] * (double)b[s->probe_cells[k]];                 \
                out[p * steps + step] = value;                                                   \
            }                                                                                    \
            /* moving air: both levels carried along (fdtd.hpp:833-840) */                       \
            if (s->flowing) {                                                                    \
                carry_##SUFFIX(job, b, i0, i1);                                                  \
                carry_##SUFFIX(job, a, i0, i1);                                                  \
            }                                                                                    \
            /* interior (fdtd.hpp:242-288) */                                                    \
            for (uint64_t i = i0; i < i1; ++i) {                                                 \
                if (s->types[i] != 1) continue;                                                  \
                const T sum = b[i - 1] + b[i + 1] + b[i - sy] + b[i + sy] + b[i - sz] + b[i + sz]; \
                T edges = 0;                                                                     \
                if (s->wide)                                                                     \
                    edges = b[i - 1 - sy] + b[i + 1 - sy] + b[i - 1 + sy] + b[i + 1 + sy] +      \
                            b[i - 1 - sz] + b[i + 1 - sz] + b[i - 1 + sz] + b[i + 1 + sz] +      \
                            b[i - sy - sz] + b[i + sy - sz] + b[i - sy + sz] + b[i + sy + sz];   \
                if (s->scaled) {                                                                 \
                    const T sc = (T)s->scale[i];                                                 \
                    if (s->wide)                                                                 \
                        a[i] = ((T)2 - total * sc) * b[i] + (sc * axial) * sum +                 \
                               (sc * diagonal) * edges - a[i];                                   \
                    else                                                                         \
                        a[i] = ((T)2 - total * sc) * b[i] + (sc * axial) * sum - a[i];           \
                } else if (s->wide) {                                                            \
                    a[i] = centre * b[i] + axial * sum + diagonal * edges - a[i];                \
                } else {                                                                         \
                    a[i] = centre * b[i] + axial * sum - a[i];                                   \
                }                                                                                \
            }                                                                                    \
            /* special cells (fdtd.hpp:860-881) */                                               \
            const T sig = (T)signal[step];                                                       \
            for (uint64_t k = k0; k < k1; ++k) {                                                 \
                const uint64_t i = (uint64_t)s->special[k];                                      \
                T sum = 0;                                                                       \
                for (uint64_t l = s->link_start[k]; l < s->link_start[k + 1]; ++l)               \
                    sum += (T)s->link_weight[l] * b[(int64_t)i + s->offset[s->link_direction[l]]]; \
                T flow = 0;                                                                      \
                for (uint64_t j = s->state_start[k]; j < s->state_start[k + 1]; ++j) {           \
                    const T own = (T)s->state_now[j] * wb[j] - (T)s->state_before[j] * wa[j];    \
                    term[j] = own;                                                               \
                    flow += (T)s->state_weight[j] * own;                                         \
                }                                                                                \
                const T previous = a[i];                                                         \
                const T next = ((T)s->coef_a[k] * b[i] + sum - (T)s->coef_b[k] * previous - flow + \
                                (T)s->source[k] * sig) * (T)s->coef_inv[k];                      \
                a[i] = next;                                                                     \
                for (uint64_t j = s->state_start[k]; j < s->state_start[k + 1]; ++j)             \
                    wa[j] += (next - previous) * (T)s->state_gain[j] + term[j];                  \
            }                                                                                    \
            /* matched layer (fdtd.hpp:2242-2264) */                                             \
            for (uint64_t c = c0; c < c1; ++c) {                                                 \
                const uint64_t i = (uint64_t)s->layer_cells[c];                                  \
                const uint64_t at[3] = {i % s->nx, (i / s->nx) % s->ny, i / sz};                 \
                T *st = lstate + 9 * c;                                                          \
                T tot = 0;                                                                       \
                for (int axis = 0; axis < 3; ++axis) {                                           \
                    const uint64_t stride = axis == 0 ? 1 : (axis == 1 ? sy : sz);               \
                    const uint64_t x = at[axis];                                                 \
                    const float *fk = s->keep[2 * axis + 1], *fp = s->push[2 * axis + 1];        \
                    T *below = &st[3 + 2 * axis], *above = &st[4 + 2 * axis];                    \
                    *below = (T)fk[x] * *below - (T)fp[x] * (b[i] - b[i - stride]);              \
                    *above = (T)fk[x + 1] * *above - (T)fp[x + 1] * (b[i + stride] - b[i]);      \
                    T *part = &st[axis];                                                         \
                    if (!s->scaled)                                                              \
                        *part = (T)s->keep[2 * axis][x] * *part -                                \
                                (T)s->push[2 * axis][x] * (*above - *below);                     \
                    else                                                                         \
                        *part = (T)s->keep[2 * axis][x] * *part -                                \
                                ((T)s->push[2 * axis][x] * (T)s->layer_scale[c]) * (*above - *below); \
                    tot += *part;                                                                \
                }                                                                                \
                a[i] = tot;                                                                      \
            }                                                                                    \
            step_barrier(job);                                                                   \
        }                                                                                        \
        flush_leave(FLUSH, csr);                                                                 \
    }

DEFINE_STEPPER(float, step_fp32, 1, f32)
DEFINE_STEPPER(double, step_fp64, 0, f64)

/*
 * ORACLE_FP32C: the same scheme in exact arithmetic, stepped in float on the pressure p_n and its
 * increment d_n = p_n - p_(n-1), kept in place of the previous level. Substituting p_(n-1) =
 * p_n - d_n into the updates above gives d_(n+1) as a sum of neighbour differences (p_m - p_n),
 * d_n and the drive, plus the constant mode's residual times p_n (zero when the coefficients
 * hold a constant pressure still, and worked out in double from the stored coefficients);
 * p_(n+1) = p_n + d_(n+1). The increment, the velocity of the scheme, is then rounded relative to
 * itself rather than to the pressure, so that rounding no longer drives the slow modes of a long
 * run. The operation order here is the GPU's compensated kernels' (fdtd_kernels.cuh).
 */
static void step_fp32c(const oracle_job *job) {
    oracle_solver *s = job->s;
    const float *signal = job->signal;
    const uint64_t steps = job->steps;
    double *out = job->out;
    float *term = (float *)s->term, *lstate = (float *)s->layer_state, *d = s->increment;
    const uint64_t sy = s->sy, sz = s->sz;
    const float axial = s->axial, diagonal = s->diagonal, residual = s->residual;
    uint64_t i0, i1, k0, k1, c0, c1;
    share(job, s->n, &i0, &i1);
    share(job, s->specials, &k0, &k1);
    share(job, s->layers, &c0, &c1);
    const unsigned csr = flush_enter(1);
    for (uint64_t step = 0; step < steps; ++step) {
        float *a = (float *)(step & 1 ? s->u1 : s->u0), *b = (float *)(step & 1 ? s->u0 : s->u1);
        float *wa = (float *)(step & 1 ? s->w1 : s->w0), *wb = (float *)(step & 1 ? s->w0 : s->w1);
        for (uint64_t p = 0; job->tid == 0 && p < s->probes; ++p) {
            double value = 0.0;
            for (uint64_t k = s->probe_start[p]; k < s->probe_start[p + 1]; ++k)
                value += s->probe_weights[k] * (double)b[s->probe_cells[k]];
            out[p * steps + step] = value;
        }
        for (uint64_t i = i0; i < i1; ++i) {
            if (s->types[i] != 1) continue;
            const float here = b[i];
            const float sum = (b[i - 1] - here) + (b[i + 1] - here) + (b[i - sy] - here) + (b[i + sy] - here) +
                              (b[i - sz] - here) + (b[i + sz] - here);
            float edges = 0.0f;
            if (s->wide)
                edges = (b[i - 1 - sy] - here) + (b[i + 1 - sy] - here) + (b[i - 1 + sy] - here) +
                        (b[i + 1 + sy] - here) + (b[i - 1 - sz] - here) + (b[i + 1 - sz] - here) +
                        (b[i - 1 + sz] - here) + (b[i + 1 + sz] - here) + (b[i - sy - sz] - here) +
                        (b[i + sy - sz] - here) + (b[i - sy + sz] - here) + (b[i + sy + sz] - here);
            float next;
            if (s->scaled) {
                const float sc = s->scale[i];
                next = s->wide ? d[i] + (sc * axial) * sum + (sc * diagonal) * edges + (sc * residual) * here
                               : d[i] + (sc * axial) * sum + (sc * residual) * here;
            } else {
                next = s->wide ? d[i] + axial * sum + diagonal * edges + residual * here
                               : d[i] + axial * sum + residual * here;
            }
            a[i] = here + next;
            d[i] = next;
        }
        const float sig = signal[step];
        for (uint64_t k = k0; k < k1; ++k) {
            const uint64_t i = (uint64_t)s->special[k];
            const float here = b[i];
            float sum = 0.0f;
            for (uint64_t l = s->link_start[k]; l < s->link_start[k + 1]; ++l)
                sum += s->link_weight[l] * (b[(int64_t)i + s->offset[s->link_direction[l]]] - here);
            float flow = 0.0f;
            for (uint64_t j = s->state_start[k]; j < s->state_start[k + 1]; ++j) {
                const float own = s->state_now[j] * wb[j] - s->state_before[j] * wa[j];
                term[j] = own;
                flow += s->state_weight[j] * own;
            }
            const float before = d[i];
            const float next = (sum + s->coef_b[k] * before - flow + s->source[k] * sig) * s->coef_inv[k] +
                               s->row_residual[k] * here;
            a[i] = here + next;
            d[i] = next;
            for (uint64_t j = s->state_start[k]; j < s->state_start[k + 1]; ++j)
                wa[j] += (next + before) * s->state_gain[j] + term[j];
        }
        /* The matched layer: the parts and faces as the reference updates them, but the cell's
           pressure carried on from its own, p + sum over axes of (keep - 1) * part - push * (above -
           below), the parts' sum in exact arithmetic: a part along an undamped axis (keep 1) then
           drops out, and with it the rounding of parts that grow far beyond the pressure. */
        for (uint64_t c = c0; c < c1; ++c) {
            const uint64_t i = (uint64_t)s->layer_cells[c];
            const uint64_t at[3] = {i % s->nx, (i / s->nx) % s->ny, i / sz};
            float *st = lstate + 9 * c;
            const float here = b[i];
            float change = 0.0f;
            for (int axis = 0; axis < 3; ++axis) {
                const uint64_t stride = axis == 0 ? 1 : (axis == 1 ? sy : sz);
                const uint64_t x = at[axis];
                const float *fk = s->keep[2 * axis + 1], *fp = s->push[2 * axis + 1];
                float *below = &st[3 + 2 * axis], *above = &st[4 + 2 * axis];
                *below = fk[x] * *below - fp[x] * (here - b[i - stride]);
                *above = fk[x + 1] * *above - fp[x + 1] * (b[i + stride] - here);
                float *part = &st[axis];
                const float keep = s->keep[2 * axis][x];
                const float push = s->scaled ? s->push[2 * axis][x] * s->layer_scale[c] : s->push[2 * axis][x];
                const float flux = push * (*above - *below);
                change += (keep - 1.0f) * *part - flux;
                *part = keep * *part - flux;
            }
            a[i] = here + change;
            d[i] = change;
        }
        step_barrier(job);
    }
    flush_leave(1, csr);
}

static void step_job(const oracle_job *job) {
    if (job->s->precision == ORACLE_FP32C)
        step_fp32c(job);
    else if (job->s->precision == ORACLE_FP32)
        step_fp32(job);
    else
        step_fp64(job);
}

/* Workers start when every one of them exists (go), or return at once (abort). */
typedef struct start_gate {
    pthread_mutex_t mutex;
    pthread_cond_t cond;
    int state; /* 0 waiting, 1 go, -1 abort */
} start_gate;

typedef struct worker {
    oracle_job job;
    start_gate *gate;
} worker;

static void *run_worker(void *arg) {
    worker *w = (worker *)arg;
    pthread_mutex_lock(&w->gate->mutex);
    while (w->gate->state == 0) pthread_cond_wait(&w->gate->cond, &w->gate->mutex);
    const int state = w->gate->state;
    pthread_mutex_unlock(&w->gate->mutex);
    if (state > 0) step_job(&w->job);
    return NULL;
}

int oracle_run(oracle_solver *s, const float *signal, uint64_t steps, double *out) {
    int threads = s->n >= ORACLE_PARALLEL_CELLS ? oracle_threads() : 1;
    worker workers[64];
    pthread_t ids[64];
    pthread_barrier_t barrier;
    start_gate gate = {PTHREAD_MUTEX_INITIALIZER, PTHREAD_COND_INITIALIZER, 0};
    int started = 1;
    for (; started < threads; ++started) {
        workers[started].job = (oracle_job){s, signal, steps, out, started, threads, &barrier};
        workers[started].gate = &gate;
        if (pthread_create(&ids[started], NULL, run_worker, &workers[started]) != 0) break;
    }
    int go = started == threads && (threads == 1 || pthread_barrier_init(&barrier, NULL, (unsigned)threads) == 0);
    pthread_mutex_lock(&gate.mutex);
    gate.state = go ? 1 : -1;
    pthread_cond_broadcast(&gate.cond);
    pthread_mutex_unlock(&gate.mutex);
    /* (without all of them, the workers return and this thread steps alone) */
    const oracle_job mine = go ? (oracle_job){s, signal, steps, out, 0, threads, &barrier}
                               : (oracle_job){s, signal, steps, out, 0, 1, NULL};
    step_job(&mine);
    for (int t = 1; t < started; ++t) pthread_join(ids[t], NULL);
    if (go && threads > 1) pthread_barrier_destroy(&barrier);
    /* the parity swap (fdtd.hpp:900-903): u1 stays the current level between runs */
    if (steps % 2 == 1) {
        void *t = s->u0; s->u0 = s->u1; s->u1 = t;
        t = s->w0; s->w0 = s->w1; s->w1 = t;
    }
    return FDTD_OK;
}

int oracle_reset(oracle_solver *s) {
    const size_t e = s->precision == ORACLE_FP64 ? 8 : 4;
    if (s->increment) memset(s->increment, 0, 4 * s->n);
    memset(s->u0, 0, e * s->n);
    memset(s->u1, 0, e * s->n);
    memset(s->w0, 0, e * s->states);
    memset(s->w1, 0, e * s->states);
    memset(s->layer_state, 0, e * 9 * s->layers);
    return FDTD_OK;
}

void *oracle_level(oracle_solver *s, int which) { return which ? s->u0 : s->u1; }

int oracle_read_state(const oracle_solver *s, void *current, void *previous, void *branch_current,
                      void *branch_previous, void *layer_state) {
    const size_t e = s->precision == ORACLE_FP64 ? 8 : 4;
    if (current) memcpy(current, s->u1, e * s->n);
    if (previous && s->increment) {
        /* the level before, as the pressure less its increment */
        for (uint64_t i = 0; i < s->n; ++i) ((float *)previous)[i] = ((const float *)s->u1)[i] - s->increment[i];
    } else if (previous) {
        memcpy(previous, s->u0, e * s->n);
    }
    if (branch_current) memcpy(branch_current, s->w1, e * s->states);
    if (branch_previous) memcpy(branch_previous, s->w0, e * s->states);
    if (layer_state) memcpy(layer_state, s->layer_state, e * 9 * s->layers);
    return FDTD_OK;
}

void oracle_destroy(oracle_solver *s) {
    if (!s) return;
    void *ptrs[] = {s->scale, s->layer_scale, s->types, s->special, s->link_start, s->state_start,
                    s->probe_start, s->probe_cells, s->link_direction, s->link_weight, s->coef_a,
                    s->coef_b, s->coef_inv, s->source, s->state_weight, s->state_now,
                    s->state_before, s->state_gain, s->layer_cells, s->probe_weights, s->u0,
                    s->u1, s->w0, s->w1, s->layer_state, s->term, s->increment, s->row_residual};
    for (size_t k = 0; k < sizeof ptrs / sizeof ptrs[0]; ++k) free(ptrs[k]);
    for (int k = 0; k < 6; ++k) free(s->keep[k]), free(s->push[k]);
    free(s);
}

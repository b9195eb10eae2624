/*
 * ORACLE / TEST INFRASTRUCTURE ONLY — see fdtd_oracle.h. A restatement, single-threaded and
 * written for reading, of WaveSolver::run (cpp/include/acoustic_spaces/fdtd.hpp:786-904 of
 * naelolaiz/acoustic-spaces). Built with -ffp-contract=off so that no multiply-add is fused.
 */
#include "fdtd_oracle.h"
#include "../acoustic_spaces_b200/csrc/fdtd_compensated.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#if defined(__SSE__) || defined(__x86_64__)
#include <xmmintrin.h>
#define ORACLE_HAS_MXCSR 1
#endif

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
};

static void *dup(const void *src, size_t bytes) {
    void *p = malloc(bytes ? bytes : 1);
    if (p && src && bytes) memcpy(p, src, bytes);
    return p;
}

int oracle_create(const fdtd_layout *L, int precision, oracle_solver **out) {
    *out = NULL;
    if (precision != ORACLE_FP32 && precision != ORACLE_FP64 && precision != ORACLE_FP32C)
        return fail("precision is FP32, FP64 or FP32 compensated");
    if (L->stencil != 7 && L->stencil != 19) return fail("the stencil has 7 or 19 points");
    if (L->flow_count) return fail("moving air is stepped on the CPU only");
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
    s->types = dup(L->types, s->n);
    s->scale = s->scaled ? dup(L->scale, 4 * s->n) : NULL;
    s->layer_scale = s->scaled ? dup(L->layer_scale, 4 * s->layers) : NULL;
    s->special = dup(L->special, 8 * s->specials);
    s->link_start = dup(L->link_start, 8 * (s->specials + 1));
    s->state_start = dup(L->state_start, 8 * (s->specials + 1));
    s->link_direction = dup(L->link_direction, s->links);
    s->link_weight = dup(L->link_weight, 4 * s->links);
    s->coef_a = dup(L->coef_a, 4 * s->specials);
    s->coef_b = dup(L->coef_b, 4 * s->specials);
    s->coef_inv = dup(L->coef_inv, 4 * s->specials);
    s->source = dup(L->source, 4 * s->specials);
    s->state_weight = dup(L->state_weight, 4 * s->states);
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
    s->layer_cells = dup(L->layer_cells, 8 * s->layers);
    s->axis_len[0] = s->nx, s->axis_len[1] = s->ny, s->axis_len[2] = s->nz;
    for (int k = 0; k < 6; ++k) {
        const uint64_t len = s->axis_len[k / 2] + 1;
        s->keep[k] = s->layers ? dup(L->keep[k], 4 * len) : NULL;
        s->push[k] = s->layers ? dup(L->push[k], 4 * len) : NULL;
    }
    s->probe_start = dup(L->probe_start, 8 * (s->probes + 1));
    const uint64_t pc = s->probe_start[s->probes];
    s->probe_cells = dup(L->probe_cells, 8 * pc);
    s->probe_weights = dup(L->probe_weights, 8 * pc);
    for (int k = 0; k < 18; ++k)
        s->offset[k] = kSteps[k][0] + kSteps[k][1] * (int64_t)s->sy + kSteps[k][2] * (int64_t)s->sz;
    const size_t e = precision == ORACLE_FP64 ? 8 : 4;
    if (precision == ORACLE_FP32C) {
        s->increment = calloc(s->n + 1, 4);
        s->row_residual = malloc(4 * s->specials + 4);
        fdtd_compensated_residuals(L, &s->residual, s->row_residual);
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
 * One instantiation per arithmetic type T. Each expression keeps the reference's operands in the
 * reference's order; with T float every operation rounds to float as the reference's does.
 */
#define DEFINE_STEPPER(T, NAME)                                                                   \
    static void NAME(oracle_solver *s, const float *signal, uint64_t steps, double *out) {       \
        T *a = (T *)s->u0, *b = (T *)s->u1, *wa = (T *)s->w0, *wb = (T *)s->w1;                  \
        T *term = (T *)s->term, *lstate = (T *)s->layer_state;                                   \
        const uint64_t sy = s->sy, sz = s->sz, n = s->n;                                         \
        const T axial = (T)s->axial, diagonal = (T)s->diagonal, centre = (T)s->centre;           \
        const T total = (T)s->total;                                                             \
        for (uint64_t step = 0; step < steps; ++step) {                                          \
            /* record (fdtd.hpp:3525-3533) */                                                    \
            for (uint64_t p = 0; p < s->probes; ++p) {                                           \
                double value = 0.0;                                                              \
                for (uint64_t k = s->probe_start[p]; k < s->probe_start[p + 1]; ++k)             \
                    value += s->probe_weights[k] * (double)b[s->probe_cells[k]];                 \
                out[p * steps + step] = value;                                                   \
            }                                                                                    \
            /* interior (fdtd.hpp:242-288) */                                                    \
            for (uint64_t i = 0; i < n; ++i) {                                                   \
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
            for (uint64_t k = 0; k < s->specials; ++k) {                                         \
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
            for (uint64_t c = 0; c < s->layers; ++c) {                                           \
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
            T *t = a; a = b; b = t;                                                              \
            t = wa; wa = wb; wb = t;                                                             \
        }                                                                                        \
    }

DEFINE_STEPPER(float, step_fp32)
DEFINE_STEPPER(double, step_fp64)

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
static void step_fp32c(oracle_solver *s, const float *signal, uint64_t steps, double *out) {
    float *a = (float *)s->u0, *b = (float *)s->u1, *wa = (float *)s->w0, *wb = (float *)s->w1;
    float *term = (float *)s->term, *lstate = (float *)s->layer_state, *d = s->increment;
    const uint64_t sy = s->sy, sz = s->sz, n = s->n;
    const float axial = s->axial, diagonal = s->diagonal, residual = s->residual;
    for (uint64_t step = 0; step < steps; ++step) {
        for (uint64_t p = 0; p < s->probes; ++p) {
            double value = 0.0;
            for (uint64_t k = s->probe_start[p]; k < s->probe_start[p + 1]; ++k)
                value += s->probe_weights[k] * (double)b[s->probe_cells[k]];
            out[p * steps + step] = value;
        }
        for (uint64_t i = 0; i < n; ++i) {
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
        for (uint64_t k = 0; k < s->specials; ++k) {
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
        for (uint64_t c = 0; c < s->layers; ++c) {
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
        float *t = a; a = b; b = t;
        t = wa; wa = wb; wb = t;
    }
}

int oracle_run(oracle_solver *s, const float *signal, uint64_t steps, double *out) {
    if (s->precision != ORACLE_FP64) {
#ifdef ORACLE_HAS_MXCSR
        const unsigned saved = _mm_getcsr();
        _mm_setcsr(saved | 0x8040u); /* flush to zero, denormals are zero (fdtd.hpp:316-336) */
#endif
        if (s->precision == ORACLE_FP32C)
            step_fp32c(s, signal, steps, out);
        else
            step_fp32(s, signal, steps, out);
#ifdef ORACLE_HAS_MXCSR
        _mm_setcsr(saved);
#endif
    } else {
        step_fp64(s, signal, steps, out);
    }
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

// Device code of the reverse-time (adjoint) stepper: the gradient of a loss of the probes'
// series with respect to the special rows' coefficients, for grids without a matched layer (either
// stencil, with or without a speed field).
//
// A forward step maps the levels (u_n, u_{n-1}) and branch velocities (w_n, w_{n-1}) to u_{n+1},
// w_{n+1}: z_{n+1} = G z_n - H z_{n-1} (+ the source), z = (u, w). For a special row (cell i,
// states j; fdtd.hpp:860-881):
//   x = ca u_n[i] + sum_l wl u_n[i + o_l] - cb u_{n-1}[i] - sum_j W_j (now_j w_n[j] - before_j w_{n-1}[j]) + src s
//   u_{n+1}[i] = ci x,   w_{n+1}[j] = w_{n-1}[j] + gain_j (u_{n+1}[i] - u_{n-1}[i]) + now_j w_n[j] - before_j w_{n-1}[j]
// and interior cells have G = centre on the diagonal, axial to each face neighbour and (19 points)
// diagonal to each edge neighbour, H = 1.
// The adjoint z~_n = dL/dz_n obeys z~_n = G^T z~_{n+1} - H^T z~_{n+2} + P_n (P_n the probes'
// terms), a leapfrog run backwards in time with the transposed operator. With a row's effective
// adjoint L~ = lam[i] + sum_j gain_j om[j] (lam, om: the adjoints of u and w):
//   lam_n[i] = sum over the cells r reading u_i of G_{r,i} L~_{n+1}[r]  -  (ci cb L~_{n+2}[i] + sum_j gain_j om_{n+2}[j])
//   om_n[j]  = -ci W_j now_j L~_{n+1}[i] + now_j om_{n+1}[j] + ci W_j before_j L~_{n+2}[i] + (1 - before_j) om_{n+2}[j]
// (an interior cell's L~ is its lam). Interior cells take the forward bulk sweep on the adjoint
// levels (their readers are interior and axial), except the cells that special rows read, which
// correct_kernel forms whole; special rows a gather over their readers (a transposed list).
// With a speed field an interior cell's adjoint is carried as s lam (s its scale): the forward
// scaled sweep steps it, and a corrected cell forms it with its own scale (the host folds s into
// its rows' coefficients and probe weights; a special row's gather takes axial x s lam from an
// interior reader, which is its coefficient a s times lam).
// The gradient of step n, with U = L~_{n+1}[i] and own~_j = om_{n+1}[j] - W_j ci U:
//   dL/dci += U x,  dL/dcb += -U ci u_{n-1}[i],  dL/dnow_j += own~_j w_n[j],
//   dL/dbefore_j += -own~_j w_{n-1}[j],  dL/dgain_j += om_{n+1}[j] (u_{n+1}[i] - u_{n-1}[i])
// needs only the special rows' own forward values, recorded as a trajectory per step; the sums
// over steps are kept in double.
#pragma once

#include "fdtd_kernels.cuh"

namespace fdtd {

struct AdjointTables {
    uint32_t specials, states;
    const uint32_t *special;  // pitched cell of each row
    const uint32_t *state_start;
    const float *state_weight, *state_now, *state_before, *state_gain;
    const float *coef_b, *coef_inv;
    // Readers of each special row's cell (transposed links): reader_start[k] .. reader_start[k+1];
    // an entry's index is a special row (its L~) when the kind bit is set, else a pitched cell
    // (interior: its lam), and its coefficient G_{reader, cell}.
    const uint32_t *reader_start, *reader_index;
    const uint8_t *reader_kind;
    const double *reader_coef;
    // Interior cells that special rows read: corrected_start .. per cell, entries (special row,
    // its coefficient on the cell), and which of the cell's neighbours (6, or 18 with the wide
    // stencil) are special rows (bit d, in the order of the stencil's directions). The adjoint
    // sweep leaves these cells to correct_kernel.
    uint32_t corrected;
    const uint32_t *corrected_cell, *corrected_start, *corrected_row;
    const uint32_t *corrected_mask;
    const double *corrected_coef;
    const float *corrected_scale;  // with a speed field: each corrected cell's scale (else null)
    float axial, diagonal, centre, total;
    uint32_t wide;  // 1: the 19-point stencil
    int32_t offset[18];
    // The probes' terms dL/dy_p x weight on the cells they read, by cell: a special row's at
    // special_read_start[k] .. [k + 1], a corrected cell's at corrected_read_start[c] .. [c + 1], of
    // (read_probe, read_weight). (Probes read no other cells that the adjoint carries: a solid
    // cell's pressure never changes.)
    const uint32_t *special_read_start, *corrected_read_start, *read_probe;
    const double *read_weight;
};

// The trajectory of a run: level l of the special rows' pressure at traj_u[l * specials + k] and
// of the branch velocities at traj_w[l * states + j].
template <typename T>
__global__ void __launch_bounds__(kBlock) record_kernel(const AdjointTables t, const T *u, const T *w, T *traj_u,
                                                        T *traj_w) {
    const uint32_t k = blockIdx.x * kBlock + threadIdx.x;
    if (k < t.specials) traj_u[k] = u[t.special[k]];
    if (k < t.states) traj_w[k] = w[k];
}

// The probes' terms of step n at a cell: sum over (probe, weight) of weight x dL/dy_p^n, in double,
// in a fixed order.
__device__ __forceinline__ double probe_terms(const AdjointTables &t, uint32_t begin, uint32_t end, const double *dloss,
                                              uint64_t stride, uint64_t step) {
    double sum = 0.0;
    for (uint32_t e = begin; e < end; ++e) sum += t.read_weight[e] * dloss[(uint64_t)t.read_probe[e] * stride + step];
    return sum;
}

// An interior cell that special rows read, or that probes read, whole: the transposed stencil of
// its interior (and solid) neighbours, as the sweep forms it, plus each reading row's
// coefficient times its L~, minus the level two steps on (lam_out holds it on entry), plus the
// probes' terms of step n. The sweep leaves these cells alone.
template <typename T>
__device__ __forceinline__ void correct_cell(const AdjointTables &t, uint32_t c, const T *lam_next, const T *tilde,
                                             T *lam_out, const double *dloss, uint64_t stride, uint64_t step) {
    if (c >= t.corrected) return;
    const uint32_t cell = t.corrected_cell[c];
    const uint32_t special = t.corrected_mask[c];
    T sum = 0, edges = 0;
#pragma unroll
    for (int d = 0; d < 6; ++d)
        if (!(special & (1u << d))) sum += lam_next[(uint32_t)((int64_t)cell + t.offset[d])];
    if (t.wide) {
#pragma unroll
        for (int d = 6; d < 18; ++d)
            if (!(special & (1u << d))) edges += lam_next[(uint32_t)((int64_t)cell + t.offset[d])];
    }
    T centre = (T)t.centre, axial = (T)t.axial, diagonal = (T)t.diagonal;
    if (t.corrected_scale) {  // as the forward scaled sweep forms its cells
        const T sc = (T)t.corrected_scale[c];
        centre = (T)2 - (T)t.total * sc;
        axial = sc * (T)t.axial;
        diagonal = sc * (T)t.diagonal;
    }
    T value = centre * lam_next[cell] + axial * sum + diagonal * edges - lam_out[cell];
    for (uint32_t e = t.corrected_start[c], end = t.corrected_start[c + 1]; e < end; ++e)
        value += (T)t.corrected_coef[e] * tilde[t.corrected_row[e]];
    const double probed = probe_terms(t, t.corrected_read_start[c], t.corrected_read_start[c + 1], dloss, stride, step);
    if (probed != 0.0) value += (T)probed;
    lam_out[cell] = value;
}

// A special row: the adjoint of its cell (with the probes' terms of step n) and branch states,
// their L~ of level n for the next reverse step (tilde_out), and the gradient of step n.
// lam_next/om_next: level n+1 (complete), tilde its L~; lam_out/om_out: hold level n+2 on entry
// (own row only) and level n on exit; traj levels of u_{n-1}, u_n... at l0 = n - s0, then l0 + 1,
// l0 + 2.
template <typename T>
__device__ __forceinline__ void special_adjoint_row(const AdjointTables &t, uint32_t k, const T *lam_next,
                                                   const T *om_next, const T *tilde, T *lam_out, T *om_out,
                                                   const T *traj_u, const T *traj_w, uint32_t level, double *g_ci,
                                                   double *g_cb, double *g_now, double *g_before, double *g_gain,
                                                   T *tilde_out, const double *dloss, uint64_t stride, uint64_t step) {
    if (k >= t.specials) return;
    const uint32_t i = t.special[k];
    const T ci = (T)t.coef_inv[k], cb = (T)t.coef_b[k];
    T gathered = 0;
    for (uint32_t e = t.reader_start[k], end = t.reader_start[k + 1]; e < end; ++e) {
        const uint32_t idx = t.reader_index[e];
        gathered += (T)t.reader_coef[e] * (t.reader_kind[e] ? tilde[idx] : lam_next[idx]);
    }
    const uint32_t s0 = t.state_start[k], s1 = t.state_start[k + 1];
    const T lam2 = lam_out[i];  // level n+2
    T tilde2 = lam2, gain_om2 = 0;
    for (uint32_t j = s0; j < s1; ++j) {
        const T term = (T)t.state_gain[j] * om_out[j];
        tilde2 += term;
        gain_om2 += term;
    }
    const T U = tilde[k];
    T lam = gathered - (ci * cb * tilde2 + gain_om2);
    const double probed = probe_terms(t, t.special_read_start[k], t.special_read_start[k + 1], dloss, stride, step);
    if (probed != 0.0) lam += (T)probed;
    lam_out[i] = lam;
    T next_tilde = lam;
    // The gradient of step n (forward values: u_{n-1}, u_n, u_{n+1} at levels l, l+1, l+2).
    const T u_prev = traj_u[(uint64_t)level * t.specials + k];
    const T u_next = traj_u[(uint64_t)(level + 2) * t.specials + k];
    g_ci[k] += (double)U * ((double)u_next / (double)ci);
    g_cb[k] += -(double)U * (double)ci * (double)u_prev;
    for (uint32_t j = s0; j < s1; ++j) {
        const T W = (T)t.state_weight[j], now = (T)t.state_now[j], before = (T)t.state_before[j];
        const T om1 = om_next[j], om2 = om_out[j];
        const T om = -ci * W * now * U + now * om1 + ci * W * before * tilde2 + ((T)1 - before) * om2;
        om_out[j] = om;
        next_tilde += (T)t.state_gain[j] * om;
        const double own_bar = (double)om1 - (double)W * (double)ci * (double)U;
        const double w_n = (double)traj_w[(uint64_t)(level + 1) * t.states + j];
        const double w_prev = (double)traj_w[(uint64_t)level * t.states + j];
        g_now[j] += own_bar * w_n;
        g_before[j] += -own_bar * w_prev;
        g_gain[j] += (double)om1 * ((double)u_next - (double)u_prev);
    }
    tilde_out[k] = next_tilde;
}

// The special rows' adjoint (blocks 0 .. special_blocks - 1) and correct_kernel's cells (the
// blocks after) in one launch: they read the same complete level and write disjoint memory.
template <typename T>
__global__ void __launch_bounds__(kBlock) rows_adjoint_kernel(const AdjointTables t, uint32_t special_blocks,
                                                              const T *lam_next, const T *om_next, const T *tilde,
                                                              T *lam_out, T *om_out, const T *traj_u, const T *traj_w,
                                                              uint32_t level, double *g_ci, double *g_cb, double *g_now,
                                                              double *g_before, double *g_gain, T *tilde_out,
                                                              const double *dloss, uint64_t stride, uint64_t step) {
    if (blockIdx.x < special_blocks)
        special_adjoint_row<T>(t, blockIdx.x * kBlock + threadIdx.x, lam_next, om_next, tilde, lam_out, om_out, traj_u,
                               traj_w, level, g_ci, g_cb, g_now, g_before, g_gain, tilde_out, dloss, stride, step);
    else
        correct_cell<T>(t, (blockIdx.x - special_blocks) * kBlock + threadIdx.x, lam_next, tilde, lam_out, dloss, stride,
                        step);
}

}  // namespace fdtd

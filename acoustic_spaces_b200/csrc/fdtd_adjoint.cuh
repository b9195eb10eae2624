// Device code of the reverse-time (adjoint) stepper: the gradient of a loss of the probes'
// series with respect to the special rows' coefficients and the matched layer's tables (either
// stencil, with or without a speed field; a matched layer comes with the 7-point stencil).
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
    // The matched layer (fdtd.hpp:2242-2264): its cells (pitched), the packed per-axis tables
    // {keep, push, keep_face, push_face} by grid coordinate, each cell's scale with a speed field.
    uint32_t layers;
    const uint32_t *layer_cells;
    const float4 *layer_coef[3];
    const float *layer_scale;
    uint32_t pitch, plane;
    FastDiv by_plane, by_pitch;
    uint64_t cells;  // pitched cells of a level (the stride of the hat arrays)
    // Rows linking to each layer cell (layer_from_start[c] .. [c + 1] of row and coefficient), the
    // probes' terms of each layer cell (layer_read_start[c] .. [c + 1] into read_probe, read_weight),
    // and which of each layer cell's axial neighbours are interior (bit d, direction d).
    const uint32_t *layer_from_start, *layer_from_row, *layer_read_start;
    const double *layer_from_coef;
    const uint8_t *layer_interior;
    // The layer's terms on a cell's adjoint (layer_terms): bit 2a, the cell below along axis a is a
    // layer cell; bit 2a + 1, the cell above; bit 6, the cell itself. Per special row, per
    // corrected cell (0 where no layer cell is near) and per layer cell (whose bit 7 says that rows
    // link to it or probes read it).
    const uint8_t *special_layer_mask, *corrected_layer_mask, *layer_mask;
    // The special rows and the corrected cells in an order that puts first those whose update
    // gathers none of the layer's terms (special_far of the rows, corrected_far of the cells):
    // those step back beside the layer's kernels, the others after the layer's hats.
    const uint32_t *special_order, *corrected_order;
    uint32_t special_far, corrected_far;
    // A gradient along a tangent of the layer's tables (fdtd_set_layer_tangent): each layer cell's
    // axes of tangent factors and its first factor in a step's (as the forward's Tables holds them).
    const uint8_t *tangent_axes;
    const uint32_t *tangent_start;
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
__device__ __forceinline__ T layer_terms(const AdjointTables &t, const T *hat, uint32_t j, uint32_t mask);

template <typename T>
__device__ __forceinline__ void correct_cell(const AdjointTables &t, uint32_t c, const T *lam_next, const T *tilde,
                                             const T *hat, T *lam_out, const double *dloss, uint64_t stride,
                                             uint64_t step) {
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
    T centre = (T)t.centre, axial = (T)t.axial, diagonal = (T)t.diagonal, sc = (T)1;
    if (t.corrected_scale) {  // as the forward scaled sweep forms its cells
        sc = (T)t.corrected_scale[c];
        centre = (T)2 - (T)t.total * sc;
        axial = sc * (T)t.axial;
        diagonal = sc * (T)t.diagonal;
    }
    T value = centre * lam_next[cell] + axial * sum + diagonal * edges - lam_out[cell];
    for (uint32_t e = t.corrected_start[c], end = t.corrected_start[c + 1]; e < end; ++e)
        value += (T)t.corrected_coef[e] * tilde[t.corrected_row[e]];
    // the matched layer's terms, times the cell's own scale as the rows' are
    if (t.layers && t.corrected_layer_mask[c]) value += sc * layer_terms<T>(t, hat, cell, t.corrected_layer_mask[c]);
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
                                                   const T *om_next, const T *tilde, const T *hat, T *lam_out, T *om_out,
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
    if (t.layers && t.special_layer_mask[k]) gathered += layer_terms<T>(t, hat, i, t.special_layer_mask[k]);
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

// ---- the matched layer ------------------------------------------------------------------------
//
// Per layer cell and axis the forward step is (fdtd.hpp:2242-2264; s the cell's speed scale, 1
// without a speed field)
//   lo' = kf[x] lo - pf[x] (b_i - b_(i-st)),  hi' = kf[x+1] hi - pf[x+1] (b_(i+st) - b_i),
//   q' = k[x] q - p[x] s (hi' - lo'),  b'_i = sum over axes of q'.
// Going back, the adjoints of step n's new states, from the level after and the values carried
// from the step after (primed):
//   Q^ = lam_(n+1)[i] + k Q^',  H^ = -p s Q^ + kf[x+1] H^',  L^ = p s Q^ + kf[x] L^'.
// Their terms on the pressures the states read: -pf[x+1] H^ on b_(i+st), pf[x] L^ on b_(i-st), and
// pf[x+1] H^ - pf[x] L^ on b_i; the cells those land on gather them (layer_terms). The tables'
// gradient, from the forward's factors of step n (layer_cell records them):
//   dk[x] += Q^ q,  dp[x] -= Q^ s (hi' - lo'),  dkf[x+1] += H^ hi,  dpf[x+1] -= H^ (b_(i+st) - b_i),
//   dkf[x] += L^ lo,  dpf[x] -= L^ (b_i - b_(i-st)).

// The six factors per axis a layer cell records per forward step, at factor f of cell c:
// traj[f * layers + c]: q, hi' - lo', hi, b_(i+st) - b_i, lo, b_i - b_(i-st) for axis 0, then 1, 2.
constexpr int kLayerFactors = 18;

// The carried values (9 per cell, together: Q^' x3, L^' x3, H^' x3 at carried[kCarried c + v]) are
// updated in place; the hats, together per pitched cell too, hat[kHats i + 2a] = pf[x] L^ and
// hat[kHats i + 2a + 1] = pf[x+1] H^, are the terms' factors its neighbours gather (a cell's state in
// one stream of memory, not fifteen). A cell's hats of step n depend only on its own adjoint
// of level n + 1 and its carried values, so the thread that forms that adjoint (the layer cell's
// reverse step n + 1, layer_adjoint_cell) forms the hats of step n right after, into the other of
// two hat buffers: the layer takes one launch a reverse step, not two. The tables' gradient sums
// g[(6a + f) * layers + c] the products of Q^, H^, L^ with the forward's factors of step n (`traj`,
// layer_cell's records); where step n's factors are not recorded yet (step n ends the segment
// before, recomputed later), Q^, L^, H^ wait in `pending` (9 per cell) for layer_pending_kernel.
constexpr int kCarried = 10;  // a layer cell's carried values, padded to an even count (vector loads)
constexpr int kHats = 6;      // a pitched cell's hats

// Along a tangent of the tables (d/dθ of each entry, θ a parameter such as the layer's damping) the
// gradient's step is the tables' products summed with the tangent:
//   dL/dθ += Q^ (q k'[x] - s (hi' - lo') p'[x]) + H^ (hi kf'[x+1] - (b_(i+st) - b_i) pf'[x+1])
//          + L^ (lo kf'[x] - (b_i - b_(i-st)) pf'[x])
// per axis along which the tangent touches the cell: the forward records the three bracketed
// factors (layer_cell's traj_tangent); each cell sums a segment's products in the last slot of its
// carried values, then into its own double sum (`acc`, layer_tangent_flush_kernel), and the cells'
// sums are summed in a fixed order at the end (layer_tangent_sum_kernel).
template <typename T>
__device__ __forceinline__ double tangent_products(const AdjointTables &t, uint32_t c, const T *factors, const T (&q)[3],
                                                   const T (&lo)[3], const T (&hi)[3]) {
    const uint32_t axes = t.tangent_axes[c];
    uint32_t slot = t.tangent_start[c];
    double sum = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (!(axes & (1u << a))) continue;
        const T *ff = factors + slot;
        slot += 3;
        sum += (double)q[a] * (double)ff[0] + (double)hi[a] * (double)ff[1] + (double)lo[a] * (double)ff[2];
    }
    return sum;
}

template <typename T>
__device__ __forceinline__ void layer_hat_cell(const AdjointTables &t, uint32_t c, uint32_t i, T lam, T *carried, T *hat,
                                               const T *traj, double *g, T *pending, const T *tangent = nullptr) {
    const uint32_t L = t.layers;
    const uint32_t z = t.by_plane(i), r = i - z * t.plane, y = t.by_pitch(r);
    const uint32_t at[3] = {r - y * t.pitch, y, z};
    const T s = t.layer_scale ? (T)t.layer_scale[c] : (T)1;
    using V2 = typename Pair<T>::type;
    V2 *own = reinterpret_cast<V2 *>(carried + (uint64_t)kCarried * c);
    T cv[kCarried];
#pragma unroll
    for (int v = 0; v < kCarried / 2; ++v) {
        const V2 p = own[v];
        cv[2 * v] = p.x, cv[2 * v + 1] = p.y;
    }
    T hv[kHats];
    T qs[3], los[3], his[3];  // (the tangent's products)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float4 c0 = __ldg(t.layer_coef[a] + at[a]), c1 = __ldg(t.layer_coef[a] + at[a] + 1);
        const T ps = t.layer_scale ? (T)c0.y * s : (T)c0.y;
        const T q_hat = lam + cv[a];
        const T lo_hat = ps * q_hat + cv[3 + a];
        const T hi_hat = -ps * q_hat + cv[6 + a];
        qs[a] = q_hat, los[a] = lo_hat, his[a] = hi_hat;
        cv[a] = (T)c0.x * q_hat;
        cv[3 + a] = (T)c0.z * lo_hat;
        cv[6 + a] = (T)c1.z * hi_hat;
        hv[2 * a] = (T)c0.w * lo_hat;
        hv[2 * a + 1] = (T)c1.w * hi_hat;
        if (g && traj) {
            const T *f = traj + (uint64_t)(6 * a) * L + c;
            double *gg = g + (uint64_t)(6 * a) * L + c;
            gg[0] += (double)q_hat * (double)f[0];
            gg[(uint64_t)1 * L] += -(double)q_hat * (double)s * (double)f[(uint64_t)1 * L];
            gg[(uint64_t)2 * L] += (double)hi_hat * (double)f[(uint64_t)2 * L];
            gg[(uint64_t)3 * L] += -(double)hi_hat * (double)f[(uint64_t)3 * L];
            gg[(uint64_t)4 * L] += (double)lo_hat * (double)f[(uint64_t)4 * L];
            gg[(uint64_t)5 * L] += -(double)lo_hat * (double)f[(uint64_t)5 * L];
        } else if (pending) {
            pending[(uint64_t)(3 * a) * L + c] = q_hat;
            pending[(uint64_t)(3 * a + 1) * L + c] = lo_hat;
            pending[(uint64_t)(3 * a + 2) * L + c] = hi_hat;
        }
    }
    // (Along a tangent the carried values' last slot, read and written anyway, sums the products of
    // the segment's steps; layer_tangent_flush_kernel adds it to the cell's double sum after each
    // segment.)
    if (tangent) cv[kCarried - 1] += (T)tangent_products<T>(t, c, tangent, qs, los, his);
#pragma unroll
    for (int v = 0; v < kCarried / 2; ++v) {
        V2 p;
        p.x = cv[2 * v], p.y = cv[2 * v + 1];
        own[v] = p;
    }
    V2 *hats = reinterpret_cast<V2 *>(hat + (uint64_t)kHats * i);
#pragma unroll
    for (int v = 0; v < kHats / 2; ++v) {
        V2 p;
        p.x = hv[2 * v], p.y = hv[2 * v + 1];
        hats[v] = p;
    }
}

// The tables' products of a step whose Q^, L^, H^ waited in `pending` (layer_hat_cell), once its
// forward factors are recorded.
template <typename T>
__global__ void __launch_bounds__(kBlock) layer_pending_kernel(const AdjointTables t, const T *pending, const T *traj,
                                                               double *g) {
    const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
    const uint32_t L = t.layers;
    if (c >= L) return;
    const T s = t.layer_scale ? (T)t.layer_scale[c] : (T)1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const T q_hat = pending[(uint64_t)(3 * a) * L + c], lo_hat = pending[(uint64_t)(3 * a + 1) * L + c];
        const T hi_hat = pending[(uint64_t)(3 * a + 2) * L + c];
        const T *f = traj + (uint64_t)(6 * a) * L + c;
        double *gg = g + (uint64_t)(6 * a) * L + c;
        gg[0] += (double)q_hat * (double)f[0];
        gg[(uint64_t)1 * L] += -(double)q_hat * (double)s * (double)f[(uint64_t)1 * L];
        gg[(uint64_t)2 * L] += (double)hi_hat * (double)f[(uint64_t)2 * L];
        gg[(uint64_t)3 * L] += -(double)hi_hat * (double)f[(uint64_t)3 * L];
        gg[(uint64_t)4 * L] += (double)lo_hat * (double)f[(uint64_t)4 * L];
        gg[(uint64_t)5 * L] += -(double)lo_hat * (double)f[(uint64_t)5 * L];
    }
}

// The tangent's products of a step whose Q^, L^, H^ waited in `pending`, once its factors are
// recorded.
template <typename T>
__global__ void __launch_bounds__(kBlock) layer_pending_tangent_kernel(const AdjointTables t, const T *pending,
                                                                       const T *factors, double *acc) {
    const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
    const uint32_t L = t.layers;
    if (c >= L) return;
    T q[3], lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        q[a] = pending[(uint64_t)(3 * a) * L + c];
        lo[a] = pending[(uint64_t)(3 * a + 1) * L + c];
        hi[a] = pending[(uint64_t)(3 * a + 2) * L + c];
    }
    acc[c] += tangent_products<T>(t, c, factors, q, lo, hi);
}

// After a segment's reverse steps along a tangent: each cell's products of the segment (the last
// slot of its carried values) into its double sum, and the slot back to 0.
template <typename T>
__global__ void __launch_bounds__(kBlock) layer_tangent_flush_kernel(uint32_t layers, T *carried, double *acc) {
    const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
    if (c >= layers) return;
    T &slot = carried[(uint64_t)kCarried * c + kCarried - 1];
    acc[c] += (double)slot;
    slot = (T)0;
}

// The cells' sums along the tangent, summed in a fixed order: block b sums cells b * span ..
// (b + 1) * span - 1, each thread a strided share in order, then the shares in a fixed tree, into
// out[b]; a last launch of one block with `span` = the first's blocks sums those.
__global__ void __launch_bounds__(kBlock) layer_tangent_sum_kernel(const double *acc, uint64_t count, uint64_t span,
                                                                   double *out) {
    __shared__ double part[kBlock];
    const uint64_t begin = (uint64_t)blockIdx.x * span, end = begin + span < count ? begin + span : count;
    double sum = 0.0;
    for (uint64_t e = begin + threadIdx.x; e < end; e += kBlock) sum += acc[e];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int half = kBlock / 2; half > 0; half /= 2) {
        if ((int)threadIdx.x < half) part[threadIdx.x] += part[threadIdx.x + half];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = part[0];
}

// The tables' gradient per coordinate, in a fixed order: block b sums the six products of the
// layer cells whose coordinate along its axis is its own (cells by_coord[start[b]] ..
// by_coord[start[b + 1]] - 1, the cells sorted by that coordinate), each thread a strided share in
// order, then the shares in a fixed tree; out[6 b + f] takes sum f. Blocks 0 .. of axis 0's
// coordinates first, then axis 1's, then axis 2's (axis_block[a] the first block of axis a).
__global__ void __launch_bounds__(kBlock) layer_table_sums_kernel(const double *g, uint32_t layers,
                                                                  const uint32_t *by_coord, const uint32_t *start,
                                                                  uint32_t axis1_block, uint32_t axis2_block,
                                                                  double *out) {
    __shared__ double part[6][kBlock];
    const uint32_t b = blockIdx.x;
    const int a = b >= axis2_block ? 2 : (b >= axis1_block ? 1 : 0);
    double sum[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t e = start[b] + threadIdx.x; e < start[b + 1]; e += kBlock) {
        const uint32_t c = by_coord[e];
#pragma unroll
        for (int f = 0; f < 6; ++f) sum[f] += g[(uint64_t)(6 * a + f) * layers + c];
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) part[f][threadIdx.x] = sum[f];
    __syncthreads();
    for (int half = kBlock / 2; half > 0; half /= 2) {
        if ((int)threadIdx.x < half)
#pragma unroll
            for (int f = 0; f < 6; ++f) part[f][threadIdx.x] += part[f][threadIdx.x + half];
        __syncthreads();
    }
    if (threadIdx.x < 6) out[6 * (uint64_t)b + threadIdx.x] = part[threadIdx.x][0];
}

// The layer's terms on the adjoint of cell j, from the hats of its layer neighbours and its own
// (mask as AdjointTables' layer masks).
template <typename T>
__device__ __forceinline__ T layer_terms(const AdjointTables &t, const T *hat, uint32_t j, uint32_t mask) {
    T sum = 0;
    if (!mask) return sum;
    const uint32_t strides[3] = {1u, t.pitch, t.plane};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (mask & (1u << (2 * a))) sum -= hat[(uint64_t)kHats * (j - strides[a]) + 2 * a + 1];
        if (mask & (1u << (2 * a + 1))) sum += hat[(uint64_t)kHats * (j + strides[a]) + 2 * a];
    }
    if (mask & 64u) {
#pragma unroll
        for (int a = 0; a < 3; ++a) sum += hat[(uint64_t)kHats * j + 2 * a + 1] - hat[(uint64_t)kHats * j + 2 * a];
    }
    return sum;
}

// The layer's part of a reverse step: where its hats of the step before go (`next`, the other hat
// buffer), its carried values, and the tables' sums with the factors of that step (`traj`, or null
// with `pending` where they are not recorded yet; both null for a gradient without the tables).
// Along a tangent (`tangent_base` not null): the factors of that step at *tangent_base +
// tangent_offset (the base in device memory, so that a captured reverse step serves every
// segment), or with `pending` none yet.
template <typename T>
struct LayerNext {
    T *hat, *carried, *pending;
    const T *traj;
    double *g;
    const T *const *tangent_base = nullptr;
    uint64_t tangent_offset = 0;
};

// A layer cell's adjoint: its interior neighbours' axial x lam (with a speed field their stored
// s lam), the rows linking to it, the layer's terms and the probes' terms (a layer cell's update
// reads no level before the last, so no level two steps on enters); then, from it, the cell's hats
// of the step before (layer_hat_cell).
template <typename T>
__device__ __forceinline__ void layer_adjoint_cell(const AdjointTables &t, uint32_t c, const T *lam_next, const T *tilde,
                                                   const T *hat, T *lam_out, const double *dloss, uint64_t stride,
                                                   uint64_t step, const LayerNext<T> &next) {
    if (c >= t.layers) return;
    const uint32_t i = t.layer_cells[c];
    const uint32_t inner = t.layer_interior[c];
    T sum = 0;
#pragma unroll
    for (int d = 0; d < 6; ++d)
        if (inner & (1u << d)) sum += lam_next[(uint32_t)((int64_t)i + t.offset[d])];
    T value = (T)t.axial * sum;
    const uint32_t mask = t.layer_mask[c];
    if (mask & 128u)  // rows linking to the cell, or probes reading it
        for (uint32_t e = t.layer_from_start[c], end = t.layer_from_start[c + 1]; e < end; ++e)
            value += (T)t.layer_from_coef[e] * tilde[t.layer_from_row[e]];
    value += layer_terms<T>(t, hat, i, mask & 127u);
    if (mask & 128u) {
        const double probed = probe_terms(t, t.layer_read_start[c], t.layer_read_start[c + 1], dloss, stride, step);
        if (probed != 0.0) value += (T)probed;
    }
    lam_out[i] = value;
    const T *tangent = next.tangent_base && !next.pending ? *next.tangent_base + next.tangent_offset : nullptr;
    layer_hat_cell<T>(t, c, i, value, next.carried, next.hat, next.traj, next.g, next.pending, tangent);
}

// One launch of the special rows' adjoint (the rows special_order[begin .. end), on the first
// blocks), of correct_kernel's cells (corrected_order[begin .. end), the next blocks) and, with
// `layer`, of the matched layer's cells (the blocks after): they read the same complete level (and
// the layer's hats of the step) and write disjoint memory. The rows and cells far from the layer
// take one launch, the rest and the layer's cells another, beside it on a stream of its own.
struct RowsPart {
    uint32_t special_begin, special_end, special_blocks;
    uint32_t corrected_begin, corrected_end, corrected_blocks;
    uint32_t layer_blocks;  // 0: no layer cells in this launch
    __host__ __device__ uint32_t blocks() const { return special_blocks + corrected_blocks + layer_blocks; }
};

template <typename T>
__global__ void __launch_bounds__(kBlock) rows_adjoint_kernel(const AdjointTables t, const RowsPart part,
                                                              const T *lam_next, const T *om_next, const T *tilde,
                                                              const T *hat, T *lam_out, T *om_out, const T *traj_u,
                                                              const T *traj_w, uint32_t level, double *g_ci,
                                                              double *g_cb, double *g_now, double *g_before,
                                                              double *g_gain, T *tilde_out, const double *dloss,
                                                              uint64_t stride, uint64_t step, const LayerNext<T> next) {
    // (The launch may hold fewer blocks than the part's work: each takes blocks' worth in turn.)
    for (uint32_t b = blockIdx.x; b < part.blocks(); b += gridDim.x) {
    if (b < part.special_blocks) {
        const uint32_t e = part.special_begin + b * kBlock + threadIdx.x;
        if (e < part.special_end)
            special_adjoint_row<T>(t, t.special_order[e], lam_next, om_next, tilde, hat, lam_out, om_out, traj_u,
                                   traj_w, level, g_ci, g_cb, g_now, g_before, g_gain, tilde_out, dloss, stride, step);
    } else if (b < part.special_blocks + part.corrected_blocks) {
        const uint32_t e = part.corrected_begin + (b - part.special_blocks) * kBlock + threadIdx.x;
        if (e < part.corrected_end)
            correct_cell<T>(t, t.corrected_order[e], lam_next, tilde, hat, lam_out, dloss, stride, step);
    } else {
        layer_adjoint_cell<T>(t, (b - part.special_blocks - part.corrected_blocks) * kBlock + threadIdx.x, lam_next,
                              tilde, hat, lam_out, dloss, stride, step, next);
    }
    }
}

}  // namespace fdtd

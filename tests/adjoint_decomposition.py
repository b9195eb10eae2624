"""Test infrastructure: the reverse-time stepper's decomposition of the adjoint by kind of cell, as
the CUDA adjoint (acoustic_spaces_b200/csrc/fdtd_adjoint.cuh) forms it, restated in float64 numpy,
with the matched layer's part that the CUDA adjoint does not take yet.

Per reverse step (level n from levels n+1 and n+2):

* the matched layer first: per cell and axis the adjoints of step n's new states, Q^ = lam_(n+1)
  + k Q^', H^ = -p s Q^ + kf_hi H^', L^ = p s Q^ + kf_lo L^' (the primed values carried from the
  step after; s the cell's speed scale, 1 without a speed field), and their terms on the
  pressures the states read, -pf_hi H^ on the cell a face above, pf_lo L^ on the cell a face
  below, pf_hi H^ - pf_lo L^ on the cell itself;
* interior cells that touch no special row, layer cell or probe: the forward sweep of the grid's
  own kind on the adjoint levels; with a speed field on v = s lam, which that sweep steps;
* corrected cells (interior cells next to a special row or a layer cell, linked by a row, or
  probed): the same stencil over their interior neighbours, plus their rows' terms, the layer's
  terms and the probes' terms, those times their own s;
* special rows: a gather over their readers (the row itself, rows linking to it, interior
  neighbours at a v, the layer's terms), their branch states as the CUDA kernel forms them;
* layer cells: their interior neighbours' a v, the rows linking to them, the layer's terms, the
  probes' terms (a layer cell's update reads no level before the last).

The gradient of the special rows' and branch states' coefficients is the CUDA adjoint's; the layer's
twelve tables take dk += Q^ q, dp -= Q^ s (hi' - lo'), dkf_hi += H^ hi, dpf_hi -= H^ (b_(i+s) - b_i),
dkf_lo += L^ lo, dpf_lo -= L^ (b_i - b_(i-s)), with q, hi, lo the states before the step and hi',
lo' after. It is checked against the autograd checker (adjoint_reference.py), which differentiates
the forward scheme without this decomposition.
"""

from __future__ import annotations

import numpy as np

from adjoint_reference import _DIRECTIONS, KEEP, PUSH


def _take(layout, name, dtype=np.float64):
    return np.asarray(layout.get(name, np.zeros(0)), dtype)


def gradient(layout, signal, dloss_dy, tables: bool = False) -> dict[str, np.ndarray]:
    """dL/d(coef_b, coef_inv; now, before, gain per state; with ``tables`` and a matched layer,
    every entry of its twelve tables) for dL/dy = ``dloss_dy`` (probes, steps)."""
    signal = np.asarray(signal, np.float64)
    dloss = np.asarray(dloss_dy, np.float64)
    nx, ny, nz = (int(v) for v in layout["shape"])
    n, strides = nx * ny * nz, (1, nx, nx * ny)
    off = np.array([x + y * nx + z * nx * ny for x, y, z in _DIRECTIONS])
    wide = int(np.asarray(layout["stencil"]).reshape(-1)[0]) == 19
    D = 18 if wide else 6
    weights = _take(layout, "weights")
    a, dg = float(weights[0]), (float(weights[6]) if wide else 0.0)
    centre, total = float(_take(layout, "centre")[0]), float(_take(layout, "total")[0])
    types = np.asarray(layout["types"])
    interior = types == 1
    scaled = len(_take(layout, "scale")) > 0
    scale = _take(layout, "scale") if scaled else np.ones(n)
    special = _take(layout, "special", np.int64)
    K = len(special)
    link_start, link_dir = _take(layout, "link_start", np.int64), _take(layout, "link_direction", np.int64)
    link_row = np.repeat(np.arange(K), np.diff(link_start))
    link_cell = special[link_row] + off[link_dir]
    link_w = _take(layout, "link_weight")
    ca, cb, ci, src = (_take(layout, k) for k in ("coef_a", "coef_b", "coef_inv", "source"))
    state_start = _take(layout, "state_start", np.int64)
    state_row = np.repeat(np.arange(K), np.diff(state_start))
    S = len(state_row)
    sw = _take(layout, "state_weight")
    branch = _take(layout, "state_branch", np.int64)
    now, before, gain = (_take(layout, k)[branch] for k in ("branch_now", "branch_before", "branch_gain"))
    probe_start = _take(layout, "probe_start", np.int64)
    P = len(probe_start) - 1
    probe_of = np.repeat(np.arange(P), np.diff(probe_start))
    probe_cell, probe_w = _take(layout, "probe_cells", np.int64), _take(layout, "probe_weights")
    layer = _take(layout, "layer_cells", np.int64)
    C = len(layer)
    coord = (layer % nx, (layer // nx) % ny, layer // (nx * ny))
    tab = {k: _take(layout, k) for k in KEEP + PUSH} if C else {}
    lscale = _take(layout, "layer_scale") if (C and scaled) else np.ones(C)
    # per axis: k, p s, kf and pf of the - face, kf and pf of the + face
    lc = [(tab[KEEP[2 * x]][coord[x]], tab[PUSH[2 * x]][coord[x]] * lscale, tab[KEEP[2 * x + 1]][coord[x]],
           tab[PUSH[2 * x + 1]][coord[x]], tab[KEEP[2 * x + 1]][coord[x] + 1], tab[PUSH[2 * x + 1]][coord[x] + 1])
          for x in range(3 if C else 0)]  # fmt: skip
    steps = len(signal)

    # ---- forward: every level, the branch velocities, the layer's states before each step
    u = np.zeros((steps + 2, n))  # u[m + 1] = u_m (u[0] = u_-1 = 0, u[1] = u_0 = 0)
    w = np.zeros((steps + 2, S))
    history = np.zeros((steps + 1, 9, C)) if (tables and C) else None
    state = np.zeros((9, C))  # q per axis (0..2), then per axis the - face and the + face
    inner = np.nonzero(interior)[0]
    for m in range(steps):
        b, prev, wb, wa = u[m + 1], u[m], w[m + 1], w[m]
        new = np.zeros(n)
        faces = sum(b[inner + o] for o in off[:6])
        edges = sum(b[inner + o] for o in off[6:]) if wide else 0.0
        if scaled:
            sc = scale[inner]
            new[inner] = (2 - total * sc) * b[inner] + sc * (a * faces + dg * edges) - prev[inner]
        else:
            new[inner] = centre * b[inner] + a * faces + dg * edges - prev[inner]
        own = now * wb - before * wa
        links = np.bincount(link_row, link_w * b[link_cell], K)
        flow = np.bincount(state_row, sw * own, K)
        rows = (ca * b[special] + links - cb * prev[special] - flow + src * signal[m]) * ci
        new[special] = rows
        w[m + 2] = wa + (rows - prev[special])[state_row] * gain + own
        if C:
            if history is not None:
                history[m] = state
            state = state.copy()
            for x in range(3):
                k_, ps, kf_lo, pf_lo, kf_hi, pf_hi = lc[x]
                st = strides[x]
                state[3 + 2 * x] = kf_lo * state[3 + 2 * x] - pf_lo * (b[layer] - b[layer - st])
                state[4 + 2 * x] = kf_hi * state[4 + 2 * x] - pf_hi * (b[layer + st] - b[layer])
                state[x] = k_ * state[x] - ps * (state[4 + 2 * x] - state[3 + 2 * x])
            new[layer] = state[:3].sum(0)
        u[m + 2] = new
    if history is not None:
        history[steps] = state

    # ---- the lists
    is_special = np.zeros(n, bool)
    is_special[special] = True
    is_layer = np.zeros(n, bool)
    is_layer[layer] = True
    row_of = np.full(n, -1, np.int64)
    row_of[special] = np.arange(K)
    # readers of each row's cell: (row, index, is-a-row, coefficient)
    r_row, r_idx, r_kind, r_coef = [np.arange(K)], [np.arange(K)], [np.ones(K, bool)], [ca * ci]
    corrected = np.zeros(n, bool)
    for d in range(D):
        j = special + off[d]
        ok = (j >= 0) & (j < n)
        ok[ok] &= interior[j[ok]]
        r_row.append(np.nonzero(ok)[0]), r_idx.append(j[ok]), r_kind.append(np.zeros(ok.sum(), bool))
        r_coef.append(np.full(ok.sum(), a if d < 6 else dg))
        corrected[j[ok]] = True
    to_row = is_special[link_cell]
    r_row.append(row_of[link_cell[to_row]]), r_idx.append(link_row[to_row]), r_kind.append(np.ones(to_row.sum(), bool))
    r_coef.append(link_w[to_row] * ci[link_row[to_row]])
    r_row, r_idx, r_kind, r_coef = (np.concatenate(v) for v in (r_row, r_idx, r_kind, r_coef))
    to_layer = is_layer[link_cell]
    to_cell = ~to_row & ~to_layer  # interior cells the rows read: corrected
    corrected[link_cell[to_cell]] = True
    for x in range(3 if C else 0):
        for side in (1, -1):
            j = layer + side * strides[x]
            corrected[j[interior[j]]] = True
    corrected[probe_cell[interior[probe_cell]]] = True
    corrected &= interior
    swept = np.nonzero(interior & ~corrected)[0]
    corr = np.nonzero(corrected)[0]
    left_out = is_special | is_layer  # neighbours a corrected cell leaves out of its sums
    # each probe term lands on its cell times the cell's scale where the cell is interior
    p_factor = np.where(interior[probe_cell], scale[probe_cell], 1.0)

    # ---- reverse
    lam_next, lam_after = np.zeros(n), np.zeros(n)  # levels n+1 and n+2
    om_next, om_after = np.zeros(S), np.zeros(S)
    til = np.zeros(K)  # the rows' L~ of level n+1
    carried = np.zeros((9, C))
    g = {"coef_b": np.zeros(K), "coef_inv": np.zeros(K), "now": np.zeros(S), "before": np.zeros(S), "gain": np.zeros(S)}
    if history is not None:
        for name in KEEP + PUSH:
            g[name] = np.zeros(len(tab[name]))
    for m in range(steps - 1, -1, -1):
        b = u[m + 1]
        out = np.zeros(n)
        # the layer's adjoints of step m's new states, and their terms on the pressures
        terms = np.zeros(n)
        hats = []
        new_carried = np.zeros((9, C))
        for x in range(3 if C else 0):
            k_, ps, kf_lo, pf_lo, kf_hi, pf_hi = lc[x]
            st = strides[x]
            q_hat = lam_next[layer] + carried[x]
            hi_hat = -ps * q_hat + carried[4 + 2 * x]
            lo_hat = ps * q_hat + carried[3 + 2 * x]
            hats.append((q_hat, hi_hat, lo_hat))
            new_carried[x], new_carried[3 + 2 * x], new_carried[4 + 2 * x] = k_ * q_hat, kf_lo * lo_hat, kf_hi * hi_hat
            np.add.at(terms, layer + st, -pf_hi * hi_hat)
            np.add.at(terms, layer - st, pf_lo * lo_hat)
            np.add.at(terms, layer, pf_hi * hi_hat - pf_lo * lo_hat)
            if history is not None:
                old, after = history[m], history[m + 1]
                xs = coord[x]
                np.add.at(g[KEEP[2 * x]], xs, q_hat * old[x])
                np.add.at(g[PUSH[2 * x]], xs, -q_hat * lscale * (after[4 + 2 * x] - after[3 + 2 * x]))
                np.add.at(g[KEEP[2 * x + 1]], xs + 1, hi_hat * old[4 + 2 * x])
                np.add.at(g[PUSH[2 * x + 1]], xs + 1, -hi_hat * (b[layer + st] - b[layer]))
                np.add.at(g[KEEP[2 * x + 1]], xs, lo_hat * old[3 + 2 * x])
                np.add.at(g[PUSH[2 * x + 1]], xs, -lo_hat * (b[layer] - b[layer - st]))
        probed = np.zeros(n)
        np.add.at(probed, probe_cell, p_factor * probe_w * dloss[probe_of, m])
        # interior cells the sweep steps
        faces = sum(lam_next[swept + o] for o in off[:6])
        edges = sum(lam_next[swept + o] for o in off[6:]) if wide else 0.0
        if scaled:
            sc = scale[swept]
            out[swept] = (2 - total * sc) * lam_next[swept] + sc * (a * faces + dg * edges) - lam_after[swept]
        else:
            out[swept] = centre * lam_next[swept] + a * faces + dg * edges - lam_after[swept]
        # corrected cells
        nb = lambda o: np.where(left_out[corr + o], 0.0, lam_next[corr + o])  # noqa: E731
        faces = sum(nb(o) for o in off[:6])
        edges = sum(nb(o) for o in off[6:]) if wide else 0.0
        sc = scale[corr]
        from_rows = np.zeros(n)
        np.add.at(from_rows, link_cell[to_cell], link_w[to_cell] * ci[link_row[to_cell]] * til[link_row[to_cell]])
        if scaled:
            value = (2 - total * sc) * lam_next[corr] + sc * (a * faces + dg * edges) - lam_after[corr]
        else:
            value = centre * lam_next[corr] + a * faces + dg * edges - lam_after[corr]
        out[corr] = value + sc * (from_rows[corr] + terms[corr]) + probed[corr]
        # layer cells
        if C:
            own = np.zeros(C)
            for o in off[:6]:
                j = layer + o
                own += np.where(interior[j], a * lam_next[j], 0.0)
            by = link_row[to_layer]
            np.add.at(from_rows, link_cell[to_layer], link_w[to_layer] * ci[by] * til[by])
            out[layer] = own + from_rows[layer] + terms[layer] + probed[layer]
        # special rows and their branch states
        gathered = np.bincount(r_row, r_coef * np.where(r_kind, til[np.minimum(r_idx, K - 1)] if K else 0.0,
                                                        lam_next[r_idx]), K)  # fmt: skip
        gain_om2 = np.bincount(state_row, gain * om_after, K)
        tilde2 = lam_after[special] + gain_om2
        U = til
        lam_rows = gathered + terms[special] - (ci * cb * tilde2 + gain_om2) + probed[special]
        out[special] = lam_rows
        u_prev, u_next = u[m][special], u[m + 2][special]
        g["coef_inv"] += U * (u_next / ci)
        g["coef_b"] += -U * ci * u_prev
        Ur, t2r, cir = U[state_row], tilde2[state_row], ci[state_row]
        om = -cir * sw * now * Ur + now * om_next + cir * sw * before * t2r + (1 - before) * om_after
        own_bar = om_next - sw * cir * Ur
        g["now"] += own_bar * w[m + 1]
        g["before"] += -own_bar * w[m]
        g["gain"] += om_next * (u_next - u_prev)[state_row]
        til = lam_rows + np.bincount(state_row, gain * om, K)
        lam_next, lam_after = out, lam_next
        om_next, om_after = om, om_next
        carried = new_carried
    return g

"""Fitting wall admittances to impulse responses with the adjoint gradient.

The reference fits a material's admittance to band absorption targets by least squares over
finite-difference slopes (src/acoustic_spaces/engine/impedance.py:379-440) and never
differentiates the wave solver. Here the misfit is of the impulse responses themselves,
L = sum over receivers and steps of (y - t)^2, and its gradient with respect to every material's
parameters comes from one forward and one reverse-time pass on the B200
(:meth:`~acoustic_spaces_b200.solver.B200WaveSolver.gradient`), whatever the number of materials.

The layout's coefficients depend on the materials as the reference builds them (fdtd.hpp:544-625,
3499-3517, 396-411): a boundary row k takes g_k = sum_m W_km (beta_m + sum_{j in m} 1 / (2 a_j))
+ W_k,edge * edge admittance over the weights W of its cut links, coef_b = 1 - r g,
coef_inv = 1 / (1 + r g); a branch (m, r, q) has a = m + r/2 + q/2 and coefficients now = 2m/a,
before = (2m + q)/a, gain = 1/(2a). :class:`AdjointFit` rebuilds those coefficients for new
parameters (the geometry stays) and carries the gradient with respect to them back to the
parameters. A relaxation branch (a 1-pole admittance: conductance gamma, corner frequency f_c) is
(m, r, q) = (0, 1/gamma, 2 pi f_c T / gamma) (engine/impedance.py:199-211).
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from acoustic_spaces_b200 import layouts
from acoustic_spaces_b200.solver import B200WaveSolver


def relaxation_branch(conductance: float, corner_hz: float, rate: float) -> np.ndarray:
    """(m, r, q) of a relaxation branch at ``rate`` steps a second."""
    r = 1.0 / conductance
    return np.array([[0.0, r, r * 2.0 * math.pi * corner_hz / rate]])


@dataclass
class Relaxation:
    """Each material's admittance: a fixed real ``beta`` and one relaxation branch of
    ``conductance`` and ``corner_hz`` (2 parameters a material)."""

    beta: np.ndarray
    conductance: np.ndarray
    corner_hz: np.ndarray

    def vector(self) -> np.ndarray:
        return np.concatenate([self.conductance, self.corner_hz])

    @staticmethod
    def from_vector(beta: np.ndarray, v: np.ndarray) -> Relaxation:
        m = len(beta)
        return Relaxation(beta, np.asarray(v[:m], float), np.asarray(v[m:], float))


class AdjointFit:
    """The misfit of a room's responses and its gradient with respect to its materials'
    relaxation parameters. ``built`` comes from :func:`layouts.cell_face_layout` (it carries the
    rows' material weights); ``target`` is (receivers, steps)."""

    def __init__(self, built: layouts.Built, signal: np.ndarray, target: np.ndarray, rate: float,
                 beta: np.ndarray, precision: str = "fp32", segment: int = 250) -> None:  # fmt: skip
        if built.sensitivity is None:
            raise ValueError("the layout carries no material weights: build it with layouts.cell_face_layout")
        self.built, self.sens = built, built.sensitivity
        self.signal = np.ascontiguousarray(signal, np.float32)
        self.target = np.asarray(target, np.float64)
        self.rate = rate
        self.beta = np.asarray(beta, float)
        self.precision, self.segment = precision, segment
        self.materials = self.sens["materials"]
        owner = np.asarray(self.sens["branch_material"], np.int64)
        if len(owner) != self.materials or not np.array_equal(np.sort(owner), np.arange(self.materials)):
            raise ValueError("one relaxation branch per material is expected")
        self.branch_of_material = np.argsort(owner)  # branch index of each material
        self.forward_s = self.gradient_s = 0.0

    # -- coefficients ---------------------------------------------------------------------------

    def _branches(self, params: Relaxation) -> np.ndarray:
        rows = np.zeros((self.materials, 3))
        for mat in range(self.materials):
            rows[self.branch_of_material[mat]] = relaxation_branch(params.conductance[mat], params.corner_hz[mat], self.rate)
        return rows

    def _g(self, params: Relaxation, mrq: np.ndarray) -> np.ndarray:
        a = mrq[:, 0] + 0.5 * mrq[:, 1] + 0.5 * mrq[:, 2]
        per_material = params.beta.copy()
        owner = np.asarray(self.sens["branch_material"], np.int64)
        np.add.at(per_material, owner, 0.5 / a)
        g = self.sens["edge_weight"] * self.sens["edge_admittance"]
        g = g + np.bincount(self.sens["row"], self.sens["weight"] * per_material[self.sens["material"]],
                            minlength=self.sens["boundary_rows"])  # fmt: skip
        return g

    def coefficients(self, params: Relaxation) -> dict[str, np.ndarray]:
        """The coefficients that depend on the materials, in float64: the boundary rows' coef_b and
        coef_inv (the first ``boundary_rows`` special rows) and each branch's now, before, gain."""
        mrq = self._branches(params)
        a = mrq[:, 0] + 0.5 * mrq[:, 1] + 0.5 * mrq[:, 2]
        r = self.sens["r"]
        g = self._g(params, mrq)
        return {
            "coef_b": 1.0 - r * g,
            "coef_inv": 1.0 / (1.0 + r * g),
            "branch_now": 2.0 * mrq[:, 0] / a,
            "branch_before": (2.0 * mrq[:, 0] + mrq[:, 2]) / a,
            "branch_gain": 0.5 / a,
        }

    def coefficient_tensors(self, conductance, corner_hz) -> dict:
        """:meth:`coefficients` as a differentiable torch map of the relaxation parameters (float64
        tensors of one value a material), extended to every special row with the rows that no
        material touches held at the layout's values: the arguments of
        :func:`acoustic_spaces_b200.autograd.responses`."""
        import torch

        d = torch.float64
        owner = torch.as_tensor(np.asarray(self.sens["branch_material"], np.int64))
        r_branch = (1.0 / conductance)[owner]
        q_branch = r_branch * (2.0 * math.pi / self.rate) * corner_hz[owner]
        a = 0.5 * r_branch + 0.5 * q_branch  # m = 0 for a relaxation branch
        per_material = torch.as_tensor(self.beta, dtype=d).index_add(0, owner, 0.5 / a)
        B = self.sens["boundary_rows"]
        weight = torch.as_tensor(np.asarray(self.sens["weight"], np.float64))
        g = torch.as_tensor(np.asarray(self.sens["edge_weight"] * self.sens["edge_admittance"], np.float64))
        g = g.index_add(0, torch.as_tensor(np.asarray(self.sens["row"], np.int64)),
                        weight * per_material[torch.as_tensor(np.asarray(self.sens["material"], np.int64))])  # fmt: skip
        r = torch.as_tensor(np.asarray(self.sens["r"], np.float64))
        lay = self.built.layout
        rest_b = torch.as_tensor(np.asarray(lay["coef_b"], np.float64)[B:])
        rest_inv = torch.as_tensor(np.asarray(lay["coef_inv"], np.float64)[B:])
        return {
            "coef_b": torch.cat([1.0 - r * g, rest_b]),
            "coef_inv": torch.cat([1.0 / (1.0 + r * g), rest_inv]),
            "branch_now": torch.zeros_like(a),
            "branch_before": q_branch / a,
            "branch_gain": 0.5 / a,
        }

    def _with(self, values: dict[str, np.ndarray]) -> dict[str, np.ndarray]:
        B = self.sens["boundary_rows"]
        lay = dict(self.built.layout)
        for name in ("coef_b", "coef_inv"):
            column = np.asarray(lay[name], np.float32).copy()
            column[:B] = np.asarray(values[name]).astype(np.float32)
            lay[name] = column
        for name in ("branch_now", "branch_before", "branch_gain"):
            lay[name] = np.asarray(values[name]).astype(np.float32)
        return lay

    def layout(self, params: Relaxation) -> dict[str, np.ndarray]:
        """The room's layout with the materials of ``params`` (coefficients rounded to float32,
        the layout's type)."""
        return self._with(self.coefficients(params))

    # -- misfit and gradient ----------------------------------------------------------------------

    def responses(self, params: Relaxation, precision: str | None = None) -> np.ndarray:
        solver = B200WaveSolver(self.layout(params), precision=precision or self.precision)
        t0 = time.perf_counter()
        y = solver.run(self.signal)
        self.forward_s = time.perf_counter() - t0
        return y

    def loss(self, params: Relaxation, precision: str | None = None) -> float:
        y = self.responses(params, precision)
        return float(np.sum((y - self.target) ** 2))

    def loss_and_gradient(self, params: Relaxation, precision: str | None = None,
                          coefficients: bool = False):  # fmt: skip
        """L and dL/d(conductance, corner_hz) (2 M values, conductances first); with
        ``coefficients``, also the gradient with respect to the layout's coefficients."""
        precision = precision or self.precision
        lay = self.layout(params)
        solver = self._solver(lay, precision)
        t0 = time.perf_counter()
        y = solver.run(self.signal)
        self.forward_s = time.perf_counter() - t0
        solver.reset()
        t0 = time.perf_counter()
        G = solver.gradient(self.signal, 2.0 * (y - self.target), segment=self.segment)
        self.gradient_s = time.perf_counter() - t0
        loss = float(np.sum((y - self.target) ** 2))
        if coefficients:
            return loss, self.chain(params, lay, G), G
        return loss, self.chain(params, lay, G)

    def central_difference(self, params: Relaxation, index: int, G: dict[str, np.ndarray],
                           relative: float = 1e-4) -> tuple[float, float]:  # fmt: skip
        """The gradient ``G`` (with respect to the coefficients, as the adjoint gives it) against the
        central difference of L in the coefficients along the tangent of parameter ``index``:
        (G . d, (L(c + d) - L(c - d)) / 2), L from the FP64 stepper. The step d is the coefficients'
        change for a relative change ``relative`` of the parameter, rounded per coefficient to a whole
        number of float32 units in the last place so that c + d and c - d are both exact float32
        values; a step that is not symmetric leaves a second-order term in the central difference."""
        v = params.vector()
        h = relative * v[index]
        up, down = v.copy(), v.copy()
        up[index] += h
        down[index] -= h
        cu = self.coefficients(Relaxation.from_vector(params.beta, up))
        cd = self.coefficients(Relaxation.from_vector(params.beta, down))
        base = self.layout(params)
        B = self.sens["boundary_rows"]
        branch = np.asarray(base["state_branch"], np.int64)
        plus, minus = dict(base), dict(base)
        predicted = 0.0
        for name, key in (("coef_b", "coef_b"), ("coef_inv", "coef_inv"), ("branch_now", "now"),
                          ("branch_before", "before"), ("branch_gain", "gain")):  # fmt: skip
            rows = name.startswith("coef")  # per special row (boundary rows), else per branch
            c0 = np.asarray(base[name], np.float32)
            part = slice(0, B) if rows else slice(None)
            unit = np.spacing(np.abs(c0[part])).astype(np.float64)
            d = np.round((cu[name] - cd[name]) / 2.0 / unit) * unit
            hi = c0[part].astype(np.float64) + d
            lo = c0[part].astype(np.float64) - d
            if not (np.array_equal(hi.astype(np.float32), hi) and np.array_equal(lo.astype(np.float32), lo)):
                raise ArithmeticError("a symmetric step is not exact in float32; take a smaller relative step")
            plus[name], minus[name] = c0.copy(), c0.copy()
            plus[name][part], minus[name][part] = hi.astype(np.float32), lo.astype(np.float32)
            predicted += float(np.sum(G[key][:B] * d) if rows else np.sum(G[key] * d[branch]))
        measured = 0.0
        for lay, sign in ((plus, 0.5), (minus, -0.5)):
            solver = B200WaveSolver(lay, precision="fp64")
            measured += sign * float(np.sum((solver.run(self.signal) - self.target) ** 2))
            solver.close()
        return predicted, measured

    def _solver(self, lay: dict, precision: str) -> B200WaveSolver:
        """The fit's solver of this precision, built once and given each iteration's coefficients
        (the geometry, the adjoint's tables and the tape's buffers stay), at rest, taping."""
        cache = self.__dict__.setdefault("_solvers", {})
        solver = cache.get(precision)
        if solver is None:
            solver = cache[precision] = B200WaveSolver(lay, precision=precision)
            solver.set_tape(self.segment)  # the run keeps its tape for the gradient
        else:
            solver.set_coefficients(*(lay[k] for k in ("coef_b", "coef_inv", "branch_now", "branch_before", "branch_gain")))
            solver.set_tape(self.segment)
            solver.reset()
        return solver

    def chain(self, params: Relaxation, lay: dict, G: dict[str, np.ndarray]) -> np.ndarray:
        """dL/d(conductance, corner_hz) from dL/d of the layout's coefficients."""
        mrq = self._branches(params)
        m, r_, q = mrq[:, 0], mrq[:, 1], mrq[:, 2]
        a = m + 0.5 * r_ + 0.5 * q
        r = self.sens["r"]
        B = self.sens["boundary_rows"]
        g = self._g(params, mrq)
        ci = 1.0 / (1.0 + r * g)
        dg = G["coef_b"][:B] * (-r) + G["coef_inv"][:B] * (-r * ci * ci)  # dL/dg per boundary row
        # per material: sum over rows of dL/dg * W_km
        per_material = np.bincount(self.sens["material"], dg[self.sens["row"]] * self.sens["weight"], minlength=self.materials)
        owner = np.asarray(self.sens["branch_material"], np.int64)
        dL_da = per_material[owner] * (-0.5 / (a * a))
        branch = np.asarray(lay["state_branch"], np.int64)
        nb = len(a)
        s_now = np.bincount(branch, G["now"], minlength=nb)
        s_before = np.bincount(branch, G["before"], minlength=nb)
        s_gain = np.bincount(branch, G["gain"], minlength=nb)
        dL_da = dL_da + s_now * (-2.0 * m / (a * a)) + s_before * (-(2.0 * m + q) / (a * a)) + s_gain * (-0.5 / (a * a))
        dL_dr = 0.5 * dL_da
        dL_dq = 0.5 * dL_da + s_before / a
        out = np.zeros(2 * self.materials)
        T = 1.0 / self.rate
        for mat in range(self.materials):
            j = self.branch_of_material[mat]
            gamma, fc = params.conductance[mat], params.corner_hz[mat]
            wc = 2.0 * math.pi * fc
            out[mat] = dL_dr[j] * (-1.0 / gamma**2) + dL_dq[j] * (-wc * T / gamma**2)
            out[self.materials + mat] = dL_dq[j] * (2.0 * math.pi * T / gamma)
        return out


# ---- the adjoint fit's room ----------------------------------------------------------------------


@dataclass
class FitProblem:
    fit: AdjointFit
    truth: Relaxation
    start: Relaxation
    description: dict
    # the room as built (room, grid, source, receivers, and the patches' cuts and materials), for
    # handing the same scene to the reference's own solver
    scene: dict = field(default_factory=dict)


def patched_room(seed: int = 0, *, size=(10.0, 8.0, 4.0), cell: float = 0.05, receivers: int = 4,
                 steps: int = 3000, precision: str = "fp32", segment: int = 250, perturbation: float = 0.3,
                 speed_of_sound: float = 343.0, split: bool = True, drive: str = "ricker") -> FitProblem:  # fmt: skip
    """A box room of ``size`` metres on cells of ``cell`` with 8 materials on seeded patches (the
    floor cut in two along x and the ceiling along y at seeded places, and the four side walls;
    with ``split`` false, 6 materials, one a face), each a 1-pole admittance (a relaxation branch:
    conductance uniform in [0.05, 0.5], corner frequency log-uniform in [50, 500] Hz); one source
    and ``receivers`` receivers at seeded places 0.5 m from the walls; the drive a 0.5 ms Ricker
    wavelet (``drive="gaussian"``: a Gaussian pulse, which adds net mass, so that the closed room's
    pressure drifts and the drift, which the walls barely change, dominates the misfit); the target
    is the room's responses at the seeded true parameters, and the fit starts from them each
    perturbed by a seeded factor within +-``perturbation``."""
    rng = np.random.default_rng(seed)
    size = np.asarray(size, float)
    rate = speed_of_sound / (layouts.COURANT * cell)
    materials = 8 if split else 6
    conductance = rng.uniform(0.05, 0.5, materials)
    corner = np.exp(rng.uniform(math.log(50.0), math.log(500.0), materials))
    truth = Relaxation(np.zeros(materials), conductance, corner)
    x_cut = rng.uniform(0.3, 0.7) * size[0]
    y_cut = rng.uniform(0.3, 0.7) * size[1]
    order = rng.permutation(materials)

    def patches(planes, points):
        planes = np.asarray(planes)
        if not split:
            return order[planes]
        patch = np.where(planes == 4, np.where(points[:, 0] < x_cut, 0, 1),
                 np.where(planes == 5, np.where(points[:, 1] < y_cut, 2, 3),
                          4 + np.clip(planes, 0, 3)))  # fmt: skip
        return order[patch]

    mats = [layouts.Material(0.0, relaxation_branch(conductance[k], corner[k], rate)) for k in range(materials)]
    room = layouts.shoebox(size, [layouts.Material(0.0)] * 6)
    room.patches, room.patch_materials = patches, mats
    points = layouts.inside_points(rng, room, size, 1 + receivers, 0.5, apart=4 * cell)
    grid = layouts.room_grid(size, cell)
    built = layouts.cell_face_layout(room, grid, points[0], points[1:], rate=rate)
    signal = layouts.ricker_drive(rate, steps) if drive == "ricker" else layouts.gaussian_drive(rate, steps)
    fit = AdjointFit(built, signal, np.zeros((receivers, steps)), rate, truth.beta, precision, segment)
    fit.target = fit.responses(truth, "fp64")
    factors = 1.0 + rng.uniform(-perturbation, perturbation, 2 * materials)
    start = Relaxation.from_vector(truth.beta, truth.vector() * factors)
    description = {
        "room": f"box {size[0]:g}x{size[1]:g}x{size[2]:g} m, {materials} materials on "
        + ("patches" if split else "its faces") + ", 1-pole each",
        "grid": "x".join(str(v) for v in grid.shape),
        "cell_m": cell,
        "air_cells": built.air_cells,
        "special_rows": len(built.layout["special"]),
        "branch_states": len(built.layout["state_branch"]),
        "receivers": receivers,
        "steps": steps,
        "parameters": 2 * materials,
        "drive": "0.5 ms Ricker wavelet" if drive == "ricker" else "0.5 ms Gaussian pulse",
        "checkpoint_every": segment,
        "seed": seed,
    }
    scene = {"room": room, "grid": grid, "source": points[0], "receivers": points[1:], "x_cut": x_cut,
             "y_cut": y_cut, "order": order, "split": split, "materials": mats}  # fmt: skip
    return FitProblem(fit, truth, start, description, scene)


def adam(problem: FitProblem, *, iterations: int = 300, rate: float = 0.05, final_rate: float | None = None,
         tolerance: float = 0.01, precision: str | None = None) -> dict:  # fmt: skip
    """Adam on the logarithms of the parameters from ``problem.start`` until every parameter is
    within ``tolerance`` of the truth (or ``iterations`` are spent). The step decays geometrically
    from ``rate`` to ``final_rate`` (``rate / 100`` by default) over the iterations: with a fixed
    step, Adam's normalised updates keep every parameter moving by about the step near the
    optimum."""
    fit = problem.fit
    beta = problem.truth.beta
    theta = np.log(problem.start.vector())
    truth = problem.truth.vector()
    final_rate = rate / 100.0 if final_rate is None else final_rate
    m = np.zeros_like(theta)
    v = np.zeros_like(theta)
    history = []
    b1, b2, eps = 0.9, 0.999, 1e-12
    errors = np.abs(np.exp(theta) / truth - 1.0)
    loss = float("nan")
    for it in range(1, iterations + 1):
        params = Relaxation.from_vector(beta, np.exp(theta))
        loss, grad = fit.loss_and_gradient(params, precision)
        grad_log = grad * np.exp(theta)
        m = b1 * m + (1 - b1) * grad_log
        v = b2 * v + (1 - b2) * grad_log**2
        step = rate * (final_rate / rate) ** ((it - 1) / max(1, iterations - 1))
        theta = theta - step * (m / (1 - b1**it)) / (np.sqrt(v / (1 - b2**it)) + eps * max(1e-300, np.sqrt(np.mean(v))))
        errors = np.abs(np.exp(theta) / truth - 1.0)
        history.append((loss, float(np.max(errors))))
        if np.max(errors) <= tolerance:
            break
    worst = float(np.max(errors))
    return {"iterations": it, "converged": worst <= tolerance, "worst_relative_error": worst, "loss": loss,
            "parameter_errors": errors.tolist(), "history": history}  # fmt: skip


def lbfgs(problem: FitProblem, *, iterations: int = 200, tolerance: float = 0.01, precision: str | None = None,
          memory: int = 20) -> dict:  # fmt: skip
    """L-BFGS (scipy's L-BFGS-B, no bounds) on the logarithms of the parameters from
    ``problem.start``, each evaluation one forward and one reverse-time pass; it builds the
    misfit's curvature from the gradients, which the correlated parameters of an admittance need
    (a valley along which Adam's per-parameter steps crawl). Stops when every parameter is within
    ``tolerance`` of the truth, or after ``iterations`` iterations."""
    from scipy.optimize import minimize

    fit = problem.fit
    beta = problem.truth.beta
    truth = problem.truth.vector()
    history: list[tuple[float, float]] = []
    state = {"evaluations": 0, "errors": np.abs(problem.start.vector() / truth - 1.0)}

    class _Done(Exception):
        pass

    def objective(theta):
        state["evaluations"] += 1
        loss, grad = fit.loss_and_gradient(Relaxation.from_vector(beta, np.exp(theta)), precision)
        state["last"] = (theta.copy(), loss)
        return loss, grad * np.exp(theta)

    def check(theta):
        errors = np.abs(np.exp(theta) / truth - 1.0)
        state["errors"] = errors
        seen, loss = state.get("last", (None, None))
        if seen is None or not np.array_equal(seen, theta):
            loss = fit.loss(Relaxation.from_vector(beta, np.exp(theta)), precision)
        history.append((float(loss), float(np.max(errors))))
        if np.max(errors) <= tolerance:
            raise _Done

    try:
        minimize(objective, np.log(problem.start.vector()), jac=True, method="L-BFGS-B", callback=check,
                 options={"maxiter": iterations, "maxcor": memory, "ftol": 0.0, "gtol": 0.0})  # fmt: skip
    except _Done:
        pass
    worst = float(np.max(state["errors"]))
    return {"iterations": len(history), "evaluations": state["evaluations"], "converged": worst <= tolerance,
            "worst_relative_error": worst, "loss": history[-1][0] if history else float("nan"),
            "parameter_errors": state["errors"].tolist(), "history": history}  # fmt: skip

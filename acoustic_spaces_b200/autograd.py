"""The wave solver's responses as a differentiable torch function of the layout's coefficients.

:func:`responses` runs a grid from rest on a drive and returns the probes' series (probes, steps)
as a float64 tensor; its backward pass is the B200 reverse-time stepper
(:meth:`~acoustic_spaces_b200.solver.B200WaveSolver.gradient`), which gives the gradient with
respect to every special row's ``coef_b``, ``coef_inv`` and every branch's ``now``, ``before``,
``gain`` (fdtd.hpp:860-881 are the rows these coefficients enter) in one pass, whatever their
number. A map from material parameters to coefficients written in torch composes with it, so the
gradient with respect to the parameters comes from torch's own chain rule.

The coefficients are float32 in the layout (the reference's type); the values given are rounded to
float32 before the run, and the gradient returned is the gradient at those rounded values. Grids of
either stencil without a matched layer, with or without a speed field.
"""

from __future__ import annotations

from collections.abc import Mapping

import numpy as np
import torch

from acoustic_spaces_b200.solver import B200WaveSolver

COEFFICIENTS = ("coef_b", "coef_inv", "branch_now", "branch_before", "branch_gain")


class _Responses(torch.autograd.Function):
    @staticmethod
    def forward(ctx, layout, signal, precision, segment, *coefs):  # noqa: D401
        lay = dict(layout)
        for name, value in zip(COEFFICIENTS, coefs):
            lay[name] = value.detach().cpu().numpy().astype(np.float32)
        solver = B200WaveSolver(lay, precision=precision)
        try:
            y = solver.run(signal)
        except BaseException:
            solver.close()
            raise
        ctx.solver, ctx.signal, ctx.segment = solver, signal, segment
        ctx.branch = np.asarray(lay["state_branch"], np.int64)
        ctx.branches = len(lay["branch_now"])
        ctx.devices = [c.device for c in coefs]
        return torch.from_numpy(y)

    @staticmethod
    def backward(ctx, dy):
        solver = ctx.solver
        try:
            G = solver.gradient(ctx.signal, dy.detach().cpu().numpy().astype(np.float64), segment=ctx.segment)
        finally:
            solver.close()
        per_branch = [np.bincount(ctx.branch, G[k], minlength=ctx.branches) for k in ("now", "before", "gain")]
        grads = [G["coef_b"], G["coef_inv"], *per_branch]
        out = [torch.from_numpy(np.ascontiguousarray(g)).to(device) for g, device in zip(grads, ctx.devices)]
        return (None, None, None, None, *out)


def responses(layout: Mapping[str, np.ndarray], signal, *, coef_b: torch.Tensor, coef_inv: torch.Tensor,
              branch_now: torch.Tensor, branch_before: torch.Tensor, branch_gain: torch.Tensor,
              precision: str = "fp32", segment: int = 250) -> torch.Tensor:  # fmt: skip
    """The probes' series (probes, steps, float64) of ``layout`` run from rest on ``signal`` with
    the given coefficients (one per special row for ``coef_b``/``coef_inv``, one per branch for the
    branch terms), differentiable in them; the backward pass recomputes the forward from checkpoints
    every ``segment`` steps. Each call steps on a fresh solver (the grid is uploaded once per
    call)."""
    signal = np.ascontiguousarray(signal, np.float32).reshape(-1)
    coefs = (coef_b, coef_inv, branch_now, branch_before, branch_gain)
    for name, value in zip(COEFFICIENTS, coefs):
        if value.shape != (len(layout[name]),):
            raise ValueError(f"{name} has shape {tuple(value.shape)}, the layout has {len(layout[name])}")
    return _Responses.apply(layout, signal, precision, int(segment), *coefs)

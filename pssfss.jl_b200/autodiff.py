"""Sweep objectives as differentiable functions of geometry and layer parameters.

``SweepObjective`` is a ``torch.autograd.Function`` (the Python counterpart of a
ChainRulesCore ``rrule``): its forward runs the sweep through the adjoint entry of the CUDA
library (``pss_partial_gsms_adj``: per point one factorisation, forward and transposed
solves on it, and per perturbed input set a fused assemble-and-contract pass that recomputes
the set's Green's-function values instead of storing its matrix) and returns the objective;
its backward hands out the gradient that forward computed, scaled by the incoming gradient.

The reference has no gradients; its objective functions are built on ``getsijmn``
(``src/Outputs.jl:73-89``), as ``gradient.te_tm_transmission_objective`` is here.
"""
import functools

import numpy as np
import torch

from . import engine
from .gradient import linearized_gradient, meander_strata, meander_topology, te_tm_transmission_objective


def adjoint_partial(precision="fp32r", device=0):
    """The ``partial_lin`` callable of ``gradient.linearized_gradient`` through the adjoint
    entry point."""
    return functools.partial(engine.partial_gsms_adjoint, precision=precision, device=device)


class SweepObjective(torch.autograd.Function):
    """f(p) = objective(analyze(build(p), flist, steering)) with df/dp from the adjoint path.

    ``forward(ctx, params, names, build, flist, steering, objective, precision, rel_step,
    topology)``: ``params`` a 1-D float64 tensor (one entry per name).  The gradient is the
    central difference (relative step ``rel_step``) of the first-order partial GSMs, which
    is exact to O(h^2) and needs no extra factorisation."""

    @staticmethod
    def forward(ctx, params, names, build, flist, steering, objective, precision="fp32r", rel_step=1e-4,
                topology=None):
        p = {k: float(v) for k, v in zip(names, params.detach().cpu().tolist())}
        f, g = linearized_gradient(build, p, flist, steering, objective, adjoint_partial(precision),
                                   rel_step=rel_step, topology=topology)
        ctx.save_for_backward(torch.tensor([g[k] for k in names], dtype=torch.float64, device=params.device))
        return torch.tensor(f, dtype=torch.float64, device=params.device)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return (grad_out * g,) + (None,) * 8


def meander_objective(params, flist, *, ntri=4000, precision="fp32r", rel_step=1e-4):
    """Σ_f (|S21_TE|² − |S21_TM|²) of the meanderline workload at normal incidence as a
    differentiable function of ``params = tensor([w, a, epsr])`` (trace width and cell pitch
    in mm, substrate permittivity)."""
    names = ("w", "a", "epsr")
    return SweepObjective.apply(params, names, lambda p: meander_strata(p, ntri=ntri),
                                np.asarray(flist, float), {"θ": 0.0, "ϕ": 0.0}, te_tm_transmission_objective,
                                precision, rel_step, lambda p: meander_topology(p, ntri=ntri))

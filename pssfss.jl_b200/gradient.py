"""Central finite-difference gradients of a sweep objective.

The differentiation workload is a meanderline on a substrate whose objective is
Σ_f (|S21_TE|² − |S21_TM|²) over a frequency sweep, differentiated with respect to the trace
width, the meander pitch and the substrate permittivity.  `fd_gradient` takes central
differences with a relative step (1e-4 by default): two whole sweeps per parameter, each
through `analyze` (the CUDA path), so it is the finite-difference check an adjoint gradient is
held to and a gradient in its own right.

Geometry steps must leave the mesh topology unchanged, so that vertices move affinely and the
difference is smooth: `topology(params)` returns a key (for the meander, its segment counts,
`Elements.jl:634-646`) that must agree at p − h, p and p + h, else `fd_gradient` raises.
"""
import numpy as np

from .analyze import analyze
from .elements import meander, meander_counts
from .layers import TE, TM, Layer
from .outputs import getsijmn
from .units import Length, mm


def fd_gradient(build, params, flist, steering, objective, *, rel_step=1e-4, topology=None,
                analyze_fn=None, **kw):
    """Objective value and its central-difference gradient.

    ``build(params) -> strata``; ``params``: dict name -> float; ``objective(results) ->
    float``.  The step of parameter p is ``rel_step * |p|`` (``rel_step`` when p is 0).
    ``analyze_fn`` defaults to this package's `analyze`; ``kw`` goes to it (e.g.
    ``precision="fp32r"``).  Returns ``(f(params), {name: df/dp})``.
    """
    run = analyze_fn or analyze
    p0 = {k: float(v) for k, v in params.items()}
    key0 = topology(p0) if topology is not None else None

    def f(p):
        if topology is not None and topology(p) != key0:
            raise ValueError(f"step changes the mesh topology: {topology(p)} != {key0} at {p}")
        return float(objective(run(build(p), flist, steering, **kw)))

    f0 = f(p0)
    grad = {}
    for name, v in p0.items():
        h = rel_step * abs(v) if v != 0 else rel_step
        fp = f({**p0, name: v + h})
        fm = f({**p0, name: v - h})
        grad[name] = (fp - fm) / (2 * h)
    return f0, grad


def te_tm_transmission_objective(results):
    """Σ over results of |S21(TE, TE)|² − |S21(TM, TM)|²."""
    return sum(abs(getsijmn(2, 1, TE, TE, r)) ** 2 - abs(getsijmn(2, 1, TM, TM, r)) ** 2
               for r in results)


def meander_strata(params, *, b=10.0, h=6.0, ntri=4000, sub_width_mm=1.0):
    """Layers and sheet of the meander workload: ``params`` has ``w`` (trace width, both
    w1 and w2, mm), ``a`` (cell period along the meander, mm) and ``epsr`` (substrate)."""
    sheet = meander(a=params["a"], b=b, h=h, w1=params["w"], w2=params["w"], ntri=ntri, units=mm)
    return [Layer(), sheet, Layer(epsr=params["epsr"], width=Length(sub_width_mm, mm)), Layer()]


def meander_topology(params, *, b=10.0, h=6.0, ntri=4000):
    """Segment counts of the meander mesh at ``params`` (equal counts: same topology)."""
    return meander_counts(params["a"], b, h, params["w"], params["w"], ntri)[:4]


def meander_gradient(params, flist, *, ntri=4000, rel_step=1e-4, analyze_fn=None, **kw):
    """Objective Σ_f (|S21_TE|² − |S21_TM|²) of the meander at normal incidence and its
    gradient with respect to ``w``, ``a`` and ``epsr``."""
    return fd_gradient(lambda p: meander_strata(p, ntri=ntri), params, np.asarray(flist, float),
                       {"θ": 0.0, "ϕ": 0.0}, te_tm_transmission_objective,
                       rel_step=rel_step, topology=lambda p: meander_topology(p, ntri=ntri),
                       analyze_fn=analyze_fn, **kw)

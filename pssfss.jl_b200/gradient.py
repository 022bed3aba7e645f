"""Central finite-difference gradients of a sweep objective.

The differentiation workload is a meanderline on a substrate whose objective is
Σ_f (|S21_TE|² − |S21_TM|²) over a frequency sweep, differentiated with respect to the trace
width, the meander pitch and the substrate permittivity.  `fd_gradient` takes central
differences with a relative step (1e-4 by default): two whole sweeps per parameter, each
through `analyze` (the CUDA path), so it is the finite-difference check an adjoint gradient is
held to and a gradient in its own right.

`linearized_gradient` needs one factorisation per point instead of 2·P: the partial GSM at
p ± h is taken to first order from the factors at p (the perturbed matrices enter only through
Λᵀ (Z± − Z) X with Λ = Z⁻ᵀ Pᵀ, and the perturbed sources through extra right-hand sides), while
the cheap host parts (modes, incident GSMs, cascade) are recomputed at p ± h.  The
linearised partial GSM comes from ``partial_lin``, by default the CUDA library's
(``engine.partial_gsms_linearized``, forward solves on the factors of Z).

Geometry steps must leave the mesh topology unchanged, so that vertices move affinely and the
difference is smooth: `topology(params)` returns a key (for the meander, its segment counts,
`Elements.jl:634-646`) that must agree at p − h, p and p + h, else `fd_gradient` raises.
"""
import numpy as np

from .analyze import add_scattered, analyze, assemble, make_plan, sheet_gblocks, sheet_io
from .elements import meander_counts
from .layers import TE, TM
from .outputs import getsijmn


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


def meander_strata(params, *, ntri=4000):
    """Layers and sheet of the meander workload (``workloads.meander_strata``): ``params`` has
    ``w`` (trace width, both w1 and w2, mm), ``a`` (cell period along the meander, mm) and
    ``epsr`` (the 1 mm substrate)."""
    from .workloads import meander_strata as build
    return build(w=params["w"], a=params["a"], epsr=params["epsr"], ntri=ntri)


def meander_topology(params, *, ntri=4000):
    """Segment counts of the meander mesh at ``params`` (equal counts: same topology)."""
    return meander_counts(params["a"], 10.0, 6.0, params["w"], params["w"], ntri)[:4]


def meander_gradient(params, flist, *, ntri=4000, rel_step=1e-4, analyze_fn=None, **kw):
    """Objective Σ_f (|S21_TE|² − |S21_TM|²) of the meander at normal incidence and its
    gradient with respect to ``w``, ``a`` and ``epsr``."""
    return fd_gradient(lambda p: meander_strata(p, ntri=ntri), params, np.asarray(flist, float),
                       {"θ": 0.0, "ϕ": 0.0}, te_tm_transmission_objective,
                       rel_step=rel_step, topology=lambda p: meander_topology(p, ntri=ntri),
                       analyze_fn=analyze_fn, **kw)


def linearized_gradient(build, params, flist, steering, objective, partial_lin=None, *, rel_step=1e-4,
                        topology=None, plan_flist=None):
    """Objective and central-difference gradient with one factorisation per point.

    ``partial_lin(sheet, rwg, points, (i1, i2), s, u, ios, perturbed)`` returns the scattered
    partial GSMs of one sheet Gblock at ``points`` and, for each entry (sheet_k, rwg_k,
    points_k, u_k, ios_k) of ``perturbed``, their first-order values at that perturbation
    from the unperturbed factorisation.  Every perturbed plan must keep the points, Gblocks,
    modes and mesh topology of the unperturbed one.  ``plan_flist``: the band that chooses
    modes and Gblocks when ``flist`` is one shard of a sweep.  Returns ``(f(params), {name:
    df/dp})``.
    """
    if partial_lin is None:
        from .engine import partial_gsms_linearized as partial_lin
    p0 = {k: float(v) for k, v in params.items()}
    key0 = topology(p0) if topology is not None else None
    steps = []
    for name, v in p0.items():
        h = rel_step * abs(v) if v != 0 else rel_step
        for sgn in (1.0, -1.0):
            p = {**p0, name: v + sgn * h}
            if topology is not None and topology(p) != key0:
                raise ValueError(f"step changes the mesh topology: {topology(p)} != {key0} at {p}")
            steps.append((name, h, p))
    cache = {}  # steps of layer parameters keep the sheet's geometry: one RWG setup serves them
    strata0 = build(p0)
    stratas = [build(p) for _, _, p in steps]
    _prefill_rwg(cache, [strata0] + stratas)
    plan0 = make_plan(strata0, flist, steering, plan_flist, rwg_cache=cache)
    plans = [make_plan(st, flist, steering, plan_flist, rwg_cache=cache) for st in stratas]
    blocks = sheet_gblocks(plan0)
    for pl in plans:
        if (sheet_gblocks(pl) != blocks or len(pl.points) != len(plan0.points)
                or any(len(a.layers[0].P) != len(b.layers[0].P) or len(a.layers[-1].P) != len(b.layers[-1].P)
                       for a, b in zip(pl.points, plan0.points))):
            raise ValueError("a step changes the points, Gblocks or modes of the sweep")
    partial0, partials = {}, [{} for _ in steps]
    for ig, (i1, i2), isht, s in blocks:
        sheet, rwg = plan0.sheets[isht - 1], plan0.rwgdat[isht - 1]
        ios0 = [sheet_io(pt.layers[i1 - 1:i2], sheet, s, pt.k0, pt.beta00) for pt in plan0.points]
        pert = []
        for pl in plans:
            sh_k = pl.sheets[isht - 1]
            if pl.rwgdat[isht - 1].nbf != rwg.nbf:
                raise ValueError("a step changes the number of basis functions")
            ios_k = [sheet_io(pt.layers[i1 - 1:i2], sh_k, s, pt.k0, pt.beta00) for pt in pl.points]
            pert.append((sh_k, pl.rwgdat[isht - 1], pl.points, pl.uvec[isht - 1], ios_k))
        dS0, lin = partial_lin(sheet, rwg, plan0.points, (i1, i2), s, plan0.uvec[isht - 1], ios0, pert)
        partial0[ig] = [add_scattered(io, d) for io, d in zip(ios0, dS0)]
        for k in range(len(steps)):
            partials[k][ig] = [add_scattered(io, d) for io, d in zip(pert[k][4], lin[k])]
    f0 = float(objective(assemble(plan0, partial0)))
    fs = [float(objective(assemble(pl, partials[k]))) for k, pl in enumerate(plans)]
    grad = {}
    for k in range(0, len(steps), 2):
        name, h, _ = steps[k]
        grad[name] = (fs[k] - fs[k + 1]) / (2 * h)
    return f0, grad


def _prefill_rwg(cache, stratas):
    """Basis-function setup (``setup_rwg``) of every distinct sheet geometry of the steps: one
    after another when the face-pair classing runs on the GPU (a fraction of a second each),
    else concurrently, the host classing being a few large numpy sorts that release the GIL."""
    from concurrent.futures import ThreadPoolExecutor
    from . import engine
    from .analyze import _geometry_key
    from .rwg import setup_rwg
    from .sheets import RWGSheet
    todo = {}
    for st in stratas:
        for sh in st:
            if isinstance(sh, RWGSheet) and sh.style != "NULL":
                key = _geometry_key(sh)
                if key not in cache and key not in todo:
                    todo[key] = sh
    if not todo:
        return
    if engine.device_available():
        for key, sh in todo.items():
            cache[key] = setup_rwg(sh)
        return
    with ThreadPoolExecutor(max_workers=min(len(todo), 8)) as ex:
        for key, rwg in zip(todo, ex.map(setup_rwg, todo.values())):
            cache[key] = rwg


def meander_linearized_gradient(params, flist, partial_lin=None, *, ntri=4000, rel_step=1e-4):
    """`meander_gradient` with one factorisation per point (see `linearized_gradient`)."""
    return linearized_gradient(lambda p: meander_strata(p, ntri=ntri), params, np.asarray(flist, float),
                               {"θ": 0.0, "ϕ": 0.0}, te_tm_transmission_objective, partial_lin,
                               rel_step=rel_step, topology=lambda p: meander_topology(p, ntri=ntri))


def linearized_gradient_sharded(build, params, flist, steering, objective, partial_lin=None, *, group=None,
                                **kw):
    """``linearized_gradient`` over the ranks of the default (or given) process group for an
    objective that is a sum over frequency points: rank k takes a contiguous block of
    ``flist`` (planned with the whole band), and one all-reduce of the 1 + P partial sums
    gives every rank the objective and gradient.  Without a process group it is plain
    ``linearized_gradient``."""
    import torch
    import torch.distributed as dist

    from .sweep import shard_range
    flist = [float(f) for f in np.atleast_1d(np.asarray(flist, float))]
    if not (dist.is_available() and dist.is_initialized()):
        return linearized_gradient(build, params, flist, steering, objective, partial_lin, **kw)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo, hi = shard_range(len(flist), rank, world)
    names = list(params)
    if hi > lo:
        f0, g = linearized_gradient(build, params, flist[lo:hi], steering, objective, partial_lin,
                                    plan_flist=flist, **kw)
        part = [f0] + [g[k] for k in names]
    else:
        part = [0.0] * (1 + len(names))
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor(part, dtype=torch.float64, device=dev)
    dist.all_reduce(t, group=group)
    tot = t.cpu().tolist()
    return tot[0], dict(zip(names, tot[1:]))

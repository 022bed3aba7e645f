"""Frequency sweeps and problem batches sharded across GPUs (one process per GPU).

Frequency points are independent given the mesh, layers and the J/K cache, so a sweep
shards with no collective on the data path: each rank analyzes a contiguous block of the
frequency list on its own device, and one ``all_gather_object`` at the end hands every rank
the whole result list in the order ``analyze`` itself returns (steering outer, frequency
inner; src/PSSFSS.jl:199-334).  Mode and Gblock selection depend on the sweep's lowest and
highest frequency (src/PSSFSS.jl:215-221), so every rank plans with the full list.  A batch
of independent problems (``analyze_many``) shards by whole problems instead, balanced by their
estimated cost.
"""
import os

import numpy as np


def shard_range(n, rank, world):
    """Contiguous block [lo, hi) of n items for ``rank`` of ``world`` (sizes differ by <= 1)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def steering_combos(steering):
    """The (outer, inner) steering points in ``analyze``'s loop order."""
    from .analyze import getsttuple

    keys = tuple(steering.keys())
    vals = [[float(v) for v in np.atleast_1d(np.asarray(steering[k], float))] for k in keys]
    return [getsttuple(keys, a, b) for a in vals[0] for b in vals[1]]


def tag_results(results, combos, flist, lo, hi):
    """(steering index, frequency index, result) for one rank's results of flist[lo:hi]."""
    tagged = []
    for r in results:
        s = next(i for i, c in enumerate(combos) if c == r.steering)
        f = lo + next(i for i, v in enumerate(flist[lo:hi]) if v == r.FGHz)
        tagged.append((s, f, r))
    return tagged


def merge_tagged(parts):
    """All ranks' tagged results in analyze's order (points a rank skipped stay skipped)."""
    allr = [t for p in parts for t in p]
    allr.sort(key=lambda t: (t[0], t[1]))
    return [t[2] for t in allr]


def analyze_sharded(strata, flist, steering, *, precision="fp64", group=None, analyze_fn=None, **kw):
    """``analyze`` over the ranks of the default (or given) process group.

    Rank k runs its frequency block on device LOCAL_RANK, planning modes and Gblocks with the
    full frequency list; the results of all ranks are gathered to every rank.  Without an
    initialised process group it is plain ``analyze``."""
    import torch.distributed as dist

    from .analyze import analyze

    fn = analyze_fn or analyze
    flist = [float(f) for f in np.atleast_1d(np.asarray(flist, dtype=float))]
    if not (dist.is_available() and dist.is_initialized()):
        return fn(strata, flist, steering, precision=precision, **kw)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = shard_range(len(flist), rank, world)
    device = int(os.environ.get("LOCAL_RANK", "0"))
    mine = []
    if hi > lo:
        mine = fn(strata, flist[lo:hi], steering, precision=precision, device=device, plan_flist=flist, **kw)
    parts = [None] * world
    dist.all_gather_object(parts, tag_results(mine, steering_combos(steering), flist, lo, hi), group=group)
    return merge_tagged(parts)


def problem_cost(case):
    """Estimated device seconds of one ``analyze_many`` case (strata, flist, steering): per
    point the FP32 factorisation (about 9 nface^3 flops on the tensor cores) and, when the
    phasing changes with frequency (theta != 0), the face-pair integrals (nface^2 pairs, FP64);
    the coefficients are rough B200 rates, used only to balance ranks."""
    from .sheets import RWGSheet
    strata, flist, steering = case
    npts = len(np.atleast_1d(np.asarray(flist, float)))
    for k, v in steering.items():
        npts *= len(np.atleast_1d(np.asarray(v, float)))
    theta = [float(t) for t in np.atleast_1d(np.asarray(steering.get("θ", 0.0), float))]
    oblique = any(t != 0.0 for t in theta)
    cost = 0.0
    for sh in strata:
        if isinstance(sh, RWGSheet) and sh.style != "NULL":
            nf = float(sh.nface)
            cost += npts * (6e-14 * nf ** 3 + (5e-10 * nf ** 2 if oblique else 0.0))
    return cost


def assign_problems(costs, world):
    """Problems to ranks, longest processing time first: each problem, largest cost first, goes
    to the rank with the least cost so far (ties to the lowest rank).  Returns per rank the
    sorted problem indices."""
    if world <= 0:
        raise ValueError("world must be positive")
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(v) for v in out]


def analyze_many_sharded(cases, *, precision="fp32r", group=None, analyze_many_fn=None, **kw):
    """``analyze_many`` over the ranks of the default (or given) process group: the problems
    (independent sheets, each with its own layers, frequencies and steering) are split across
    ranks by ``assign_problems`` on ``problem_cost``; rank k runs its share in one call on
    device LOCAL_RANK, and one ``all_gather_object`` hands every rank all problems' results in
    the input order.  Without an initialised process group it is plain ``analyze_many``."""
    import torch.distributed as dist

    from .analyze import analyze_many

    fn = analyze_many_fn or analyze_many
    cases = list(cases)
    if not (dist.is_available() and dist.is_initialized()):
        return fn(cases, precision=precision, **kw)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mine = assign_problems([problem_cost(c) for c in cases], world)[rank]
    device = int(os.environ.get("LOCAL_RANK", "0"))
    res = fn([cases[i] for i in mine], precision=precision, device=device, **kw) if mine else []
    parts = [None] * world
    dist.all_gather_object(parts, list(zip(mine, res)), group=group)
    out = [None] * len(cases)
    for part in parts:
        for i, r in part:
            out[i] = r
    return out

"""Frequency sweeps sharded across GPUs (one process per GPU).

Frequency points are independent given the mesh, layers and the J/K cache, so a sweep
shards with no collective on the data path: each rank analyzes a contiguous block of the
frequency list on its own device, and one ``all_gather_object`` at the end hands every rank
the whole result list in the order ``analyze`` itself returns (steering outer, frequency
inner; src/PSSFSS.jl:199-334).  Mode and Gblock selection depend on the sweep's lowest and
highest frequency (src/PSSFSS.jl:215-221), so every rank plans with the full list.
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

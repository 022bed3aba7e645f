"""Autotuner of the FP32 + refinement sweep: batch size and LU tile shape per unknown count.

The batched sweep factors ``batch`` matrices of one unknown count together (every LU,
update, solve and refinement kernel takes its matrix from the grid), and its FP32 LU has two
tile-shape knobs: the cluster panel's width (8, 16 or 32 columns) and the outer block (64 or
128 columns, the depth K of each tensor-core trailing update).  Which combination is fastest
depends on N: small matrices are latency-bound and want wide batches; large ones are bound
by the tensor-core update and want the deep outer block.

``tune`` times a representative ring-patch problem (the batched workload's own geometry,
free-standing, normal incidence) per unknown-count bucket on the current device over a staged
search - the tile shape at the default batch, then the batch for the best tile shape - and
stores the winners with every timing in a JSON table.  ``lookup(n)`` returns the stored
choice for an unknown count (the library defaults when no table exists), in the form
``analyze.analyze_many(tuning=...)`` and ``engine.partial_gsms_multi`` take.
"""
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning", "b200_fp32r.json")
DEFAULT = {"batch": 12, "panel_w": 32, "outer_nb": 128}
# upper unknown count of each bucket, and the ring mesh size that lands near its middle
BUCKETS = ((900, 400), (1700, 900), (2500, 1500), (3200, 2000), (4200, 2600), (8192, 3800))
TILES = ((32, 128), (16, 128), (32, 64), (16, 64))
BATCHES = (4, 8, 12, 16, 24, 32)

_cache = {}


def lookup(n, path=None):
    """Batch size and FP32 LU tile shape for unknown count ``n`` from the stored table."""
    path = path or TABLE
    tab = _cache.get(path)
    if tab is None:
        try:
            with open(path) as f:
                tab = json.load(f)
        except (OSError, ValueError):
            tab = {"buckets": []}
        _cache[path] = tab
    for b in tab.get("buckets", []):
        if n <= b["nmax"]:
            return {k: int(b[k]) for k in ("batch", "panel_w", "outer_nb")}
    return dict(DEFAULT)


def _ring_problem(ntri, npts, period=9.0):
    from .analyze import make_plan, sheet_gblocks, sheet_io
    from .elements import polyring
    from .layers import Layer
    from .units import mm
    ro = 0.4 * period
    sheet = polyring(s1=[period, 0], s2=[0, period], a=[ro - 0.05 * period], b=[ro], sides=48, ntri=ntri, units=mm)
    plan = make_plan([Layer(), sheet, Layer()], np.linspace(10, 20, npts), {"θ": 0.0, "ϕ": 0.0})
    (ig, (i1, i2), isht, s), = sheet_gblocks(plan)
    rwg = plan.rwgdat[isht - 1]
    ios = [sheet_io(pt.layers[i1 - 1:i2], sheet, s, pt.k0, pt.beta00) for pt in plan.points]
    return dict(sheet=sheet, rwg=rwg, points=plan.points, region_rng=(i1, i2), s=s, u=plan.uvec[isht - 1], ios=ios)


def _time(problem, cfg, reps, device):
    from . import engine
    best = None
    for _ in range(reps):
        st = {}
        engine.partial_gsms_multi([dict(problem, **cfg)], precision="fp32r", device=device, stats=st)
        t = st["timings_ms"]["total"]
        best = t if best is None else min(best, t)
    return best


def tune(path=None, npts=36, reps=2, device=0, buckets=BUCKETS, log=print):
    """Search every bucket and write the table; returns it."""
    import torch
    path = path or TABLE
    out = {"device": torch.cuda.get_device_name(device), "precision": "fp32r",
           "date": time.strftime("%Y-%m-%d %H:%M:%S"), "points_per_trial": npts, "reps": reps,
           "workload": "polyring ring patch, period 9 mm, 48 sides, free-standing, normal incidence, 10-20 GHz",
           "buckets": []}
    for nmax, ntri in buckets:
        pr = _ring_problem(ntri, npts)
        n = pr["rwg"].nbf
        _time(pr, dict(DEFAULT), 1, device)  # warm-up: buffers sized for this N
        trials = []
        for pw, nb in TILES:
            cfg = {"batch": DEFAULT["batch"], "panel_w": pw, "outer_nb": nb}
            trials.append((_time(pr, cfg, reps, device), cfg))
        best_tile = min(trials, key=lambda t: t[0])[1]
        for bsz in BATCHES:
            if bsz == DEFAULT["batch"]:
                continue
            cfg = dict(best_tile, batch=bsz)
            trials.append((_time(pr, cfg, reps, device), cfg))
        t_best, cfg_best = min(trials, key=lambda t: t[0])
        t_def = next(t for t, c in trials if c == DEFAULT)
        rec = {"nmax": nmax, "n": n, **cfg_best, "ms_per_point": t_best / npts,
               "default_ms_per_point": t_def / npts,
               "trials": [{**c, "ms_per_point": t / npts} for t, c in trials]}
        out["buckets"].append(rec)
        if log:
            log(f"N={n:5d} (<= {nmax}): {cfg_best}  {t_best / npts:.3f} ms/point (default {t_def / npts:.3f})")
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    _cache.pop(path, None)
    return out


if __name__ == "__main__":
    import sys
    sys.exit(0 if tune() else 1)

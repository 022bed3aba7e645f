"""Sharded sweeps across ranks (the multi-GPU path's host logic), on CPU with gloo.

Each rank analyzes a contiguous block of the frequency list; the gathered result list
must equal a single-process run in order and content, including points that ``analyze``
skips (principal modes cut off), and every rank must plan with the whole band.  The
per-point solver is replaced by a host function so no GPU is needed; under these ranks the
GPU path is the same ``analyze`` that the parity tests cover.
"""
import os
import socket
import types

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import conftest  # noqa: F401  (loads the package as pssfss_b200, also in spawned ranks)
from pssfss_b200.sweep import merge_tagged, shard_range, steering_combos, tag_results


def test_shard_range_covers_and_balances():
    for n in (0, 1, 5, 101):
        for world in (1, 2, 3, 8):
            blocks = [shard_range(n, k, world) for k in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
            sizes = [hi - lo for lo, hi in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def fake_analyze(strata, flist, steering, precision="fp64", device=0, plan_flist=None):
    """Stand-in for analyze: one result per (steering, frequency); frequencies above 17 GHz
    are skipped at the second steering point (a cut-off principal mode); echoes the band."""
    out = []
    band = (min(plan_flist or flist), max(plan_flist or flist))
    for i, st in enumerate(steering_combos(steering)):
        for f in flist:
            if i == 1 and f > 17.0:
                continue
            out.append(types.SimpleNamespace(steering=st, FGHz=f, value=(i, f), band=band))
    return out


def _worker(rank, world, port, flist, steering, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pssfss_b200.sweep import analyze_sharded
        res = analyze_sharded(None, flist, steering, analyze_fn=fake_analyze)
        q.put((rank, [(r.value, r.band) for r in res]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_analyze_sharded_gloo_matches_single_process():
    world = 2
    flist = [10.0 + 0.5 * k for k in range(17)]
    steering = {"θ": [0.0, 30.0], "ϕ": 45.0}
    single = [(r.value, r.band) for r in fake_analyze(None, flist, steering, plan_flist=flist)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(k, world, port, flist, steering, q)) for k in range(world)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(240):  # poll: a rank that died ends the wait at once
            while not q.empty() and len(got) < world:
                k, v = q.get()
                got[k] = v
            if len(got) == world or any(p.exitcode not in (None, 0) for p in procs):
                break
            procs[0].join(timeout=0.5)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    for k in range(world):
        assert got[k] == single


def test_merge_tagged_orders_by_steering_then_frequency():
    flist = [1.0, 2.0, 3.0, 4.0]
    steering = {"θ": [0.0, 10.0], "ϕ": 0.0}
    combos = steering_combos(steering)
    mk = lambda s, f: types.SimpleNamespace(steering=combos[s], FGHz=f)
    part0 = tag_results([mk(0, 1.0), mk(0, 2.0), mk(1, 1.0)], combos, flist, 0, 2)
    part1 = tag_results([mk(0, 3.0), mk(1, 3.0), mk(1, 4.0)], combos, flist, 2, 4)
    merged = merge_tagged([part1, part0])
    assert [(combos.index(r.steering), r.FGHz) for r in merged] == [(0, 1.0), (0, 2.0), (0, 3.0), (1, 1.0),
                                                                    (1, 3.0), (1, 4.0)]


def _grad_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import functools
        import oracle
        from pssfss_b200.gradient import (linearized_gradient_sharded, meander_strata, meander_topology,
                                          te_tm_transmission_objective)
        part = functools.partial(oracle.partial_gsms_linearized, tangent=True)
        f, g = linearized_gradient_sharded(lambda p: meander_strata(p, ntri=120), GRAD_P0, GRAD_FREQS,
                                           {"θ": 0.0, "ϕ": 0.0}, te_tm_transmission_objective, part,
                                           topology=lambda p: meander_topology(p, ntri=120))
        q.put((rank, (f, g)))
    finally:
        dist.destroy_process_group()


GRAD_P0 = {"w": 0.3, "a": 5.0, "epsr": 2.2}
GRAD_FREQS = [9.0, 12.0, 15.0]


def test_linearized_gradient_sharded_gloo_matches_single_process():
    # the gradient objective is a sum over frequencies: ranks take blocks of the sweep and one
    # all-reduce of the partial sums gives the single-process objective and gradient
    import functools
    import oracle
    from pssfss_b200.gradient import meander_linearized_gradient
    part = functools.partial(oracle.partial_gsms_linearized, tangent=True)
    f1, g1 = meander_linearized_gradient(GRAD_P0, GRAD_FREQS, part, ntri=120)
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_grad_worker, args=(k, world, port, q)) for k in range(world)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(480):
            while not q.empty() and len(got) < world:
                k, v = q.get()
                got[k] = v
            if len(got) == world or any(p.exitcode not in (None, 0) for p in procs):
                break
            procs[0].join(timeout=0.5)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    for k in range(world):
        f, g = got[k]
        assert abs(f - f1) <= 1e-12 * abs(f1)
        for name in GRAD_P0:
            assert abs(g[name] - g1[name]) <= 1e-9 * abs(g1[name]), (name, g[name], g1[name])


def test_assign_problems_balances_longest_first():
    from pssfss_b200.sweep import assign_problems
    costs = [5.0, 1.0, 4.0, 3.0, 3.0, 2.0, 2.0]
    parts = assign_problems(costs, 2)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs) and loads == [10.0, 10.0]
    assert assign_problems(costs, 1) == [list(range(len(costs)))]
    assert assign_problems([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        assign_problems(costs, 0)


def test_problem_cost_orders_by_size_and_incidence():
    from pssfss_b200.elements import polyring
    from pssfss_b200.layers import Layer
    from pssfss_b200.sweep import problem_cost
    from pssfss_b200.units import mm
    small = polyring(s1=[8, 0], s2=[0, 8], a=[2.8], b=[3.2], sides=24, ntri=200, units=mm)
    big = polyring(s1=[8, 0], s2=[0, 8], a=[2.8], b=[3.2], sides=24, ntri=800, units=mm)
    c = lambda sh, th, nf=5: problem_cost(([Layer(), sh, Layer()], [10.0 + k for k in range(nf)], {"θ": th, "ϕ": 0.0}))
    assert c(small, 0.0) < c(big, 0.0) < c(big, 30.0)
    assert abs(c(big, 0.0, 10) - 2 * c(big, 0.0, 5)) < 1e-12 * c(big, 0.0, 10)


def fake_analyze_many(cases, precision="fp32r", device=0):
    """Stand-in for analyze_many: per case a list of (case tag, frequency) results."""
    return [[(strata, f) for f in flist] for strata, flist, steering in cases]


def _many_worker(rank, world, port, cases, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import pssfss_b200.sweep as sw
        sw.problem_cost = lambda case: float(case[0])  # the tag is the cost: no sheets needed
        q.put((rank, sw.analyze_many_sharded(cases, analyze_many_fn=fake_analyze_many)))
    finally:
        dist.destroy_process_group()


def test_analyze_many_sharded_gloo_matches_single_process():
    world = 2
    cases = [(c, [10.0 + k for k in range(n)], {"θ": 0.0, "ϕ": 0.0})
             for c, n in ((7, 3), (1, 2), (4, 1), (9, 2), (2, 4), (3, 1))]
    single = fake_analyze_many(cases)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_many_worker, args=(k, world, port, cases, q)) for k in range(world)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(240):
            while not q.empty() and len(got) < world:
                k, v = q.get()
                got[k] = v
            if len(got) == world or any(p.exitcode not in (None, 0) for p in procs):
                break
            procs[0].join(timeout=0.5)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    for k in range(world):
        assert got[k] == single

"""CUDA path against the CPU oracle at the benchmark workloads' own sizes.

* meanderline precision sweep: a = 5, b = 10, h = 6, w1 = w2 = 0.3 mm, ntri = 3000 (2840
  faces, N = 3976 unknowns) on 1 mm eps_r = 2.2, normal incidence - 3 of its 101 frequencies
  (8, 13, 18 GHz) through the sweep entry pss_partial_gsms;
* Jerusalem-cross / aperture cascade at its stated size: cross ntri = 1500, aperture
  ntri = 1200, theta = 30, phi = 45 (face-pair integrals recomputed per point) - 2 of its 51
  frequencies through analyze (both sheets, cascade included);
* meanderline gradient workload: ntri = 4000 (3960 faces, N = 5610) - one frequency;
* batched ring workload (64 seeded problems): its largest normal-incidence ring (3046 faces)
  and its largest oblique ring (3202 faces, theta = 15) at 15 GHz, in one multi-problem call.

Bars: the FP64 form within 1e-9 relative of the FP64 oracle (max-abs difference over
max-abs value); the FP32 + FP64-refinement form within |dS| <= 1e-6 absolute of the FP64
oracle (the precision form's target).  The oracle needs a few seconds to a minute per point
at these sizes on the host cores.
"""
import numpy as np
import pytest

import oracle
from pssfss_b200 import engine, workloads
from pssfss_b200.analyze import analyze, make_plan, sheet_gblocks, sheet_io

pytestmark = pytest.mark.gpu


def _sweep_vs_oracle(strata, freqs):
    plan = make_plan(strata, freqs, {"θ": 0.0, "ϕ": 0.0})
    (ig, (i1, i2), isht, s), = sheet_gblocks(plan)
    sheet, rwg, u = plan.sheets[isht - 1], plan.rwgdat[isht - 1], plan.uvec[isht - 1]
    ios = [sheet_io(pt.layers[i1 - 1:i2], sheet, s, pt.k0, pt.beta00) for pt in plan.points]
    args = (sheet, rwg, plan.points, (i1, i2), s, u, ios)
    st64, st32 = {}, {}
    d64 = engine.partial_gsms(*args, precision="fp64", stats=st64)
    d32 = engine.partial_gsms(*args, precision="fp32r", stats=st32)
    ref = [oracle.partial_dS(sheet, rwg, pt.layers[i1 - 1:i2], s, pt.k0, u, io)[0]
           for pt, io in zip(plan.points, ios)]
    return rwg.nbf, d64, d32, ref, st32["status"]


def test_meander_sweep_at_bench_size():
    strata = workloads.meander_strata(ntri=3000)
    nbf, d64, d32, ref, status = _sweep_vs_oracle(strata, [8.0, 13.0, 18.0])
    assert nbf == 3976
    for g64, g32, r in zip(d64, d32, ref):
        assert np.max(np.abs(g64 - r)) / np.max(np.abs(r)) < 1e-9
        assert np.max(np.abs(g32 - r)) <= 1e-6
    assert all(s & ~32 == 0 for s in status), status


def test_meander_gradient_workload_point():
    params, flist, ntri = workloads.meander_gradient_workload()
    strata = workloads.meander_strata(ntri=ntri, **params)
    nbf, d64, d32, ref, status = _sweep_vs_oracle(strata, [13.0])
    assert nbf == 5610
    assert np.max(np.abs(d64[0] - ref[0])) / np.max(np.abs(ref[0])) < 1e-9
    assert np.max(np.abs(d32[0] - ref[0])) <= 1e-6


def test_jerusalem_aperture_cascade_at_stated_size():
    strata, flist, steer = workloads.jerusalem_aperture_cascade()
    freqs = [float(flist[10]), float(flist[40])]  # 9 and 21 GHz of the 51-point sweep
    assert strata[1].nface >= 1400 and strata[4].nface >= 1100
    ref = oracle.analyze(strata, freqs, steer)
    for prec, bar in (("fp64", None), ("fp32r", 1e-6)):
        res = analyze(strata, freqs, steer, precision=prec)
        assert len(res) == len(ref) == 2
        for a, b in zip(res, ref):
            for k in ((1, 1), (1, 2), (2, 1), (2, 2)):
                d = np.max(np.abs(a.gsm[k] - b.gsm[k]))
                if bar is None:
                    assert d / np.max(np.abs(b.gsm[k])) < 1e-9, (prec, k)
                else:
                    assert d <= bar, (prec, k, d)


def test_ring_batch_members_at_stated_size():
    # the batched workload (64 seeded ring problems, 21 frequencies each, theta in {0, 15, 30,
    # 45}): its largest normal-incidence ring and its largest oblique ring, at one frequency
    # each, through one pss_partial_gsms_multi call, against the FP64 oracle
    from pssfss_b200.analyze import make_plan, sheet_gblocks, sheet_io
    batch = workloads.ring_batch()
    normal = max((c for c in batch if c[2]["θ"] == 0.0), key=lambda c: c[0][1].nface)
    oblique = max((c for c in batch if c[2]["θ"] != 0.0), key=lambda c: c[0][1].nface)
    probs, refs = [], []
    for strata, flist, steer in (normal, oblique):
        plan = make_plan(strata, [float(flist[10])], steer)
        (ig, (i1, i2), isht, s), = sheet_gblocks(plan)
        sheet, rwg, u = plan.sheets[isht - 1], plan.rwgdat[isht - 1], plan.uvec[isht - 1]
        ios = [sheet_io(pt.layers[i1 - 1:i2], sheet, s, pt.k0, pt.beta00) for pt in plan.points]
        probs.append(dict(sheet=sheet, rwg=rwg, points=plan.points, region_rng=(i1, i2), s=s, u=u, ios=ios))
        pt = plan.points[0]
        refs.append(oracle.partial_dS(sheet, rwg, pt.layers[i1 - 1:i2], s, pt.k0, u, ios[0])[0])
    assert probs[0]["rwg"].nbf > 4000 and probs[1]["rwg"].nbf > 3000
    d64 = engine.partial_gsms_multi(probs, precision="fp64")
    d32 = engine.partial_gsms_multi(probs, precision="fp32r")
    for g64, g32, r in zip(d64, d32, refs):
        assert np.max(np.abs(g64[0] - r)) / np.max(np.abs(r)) < 1e-9
        assert np.max(np.abs(g32[0] - r)) <= 1e-6

"""Many sweeps in one call (pss_partial_gsms_multi / analyze.analyze_many) on the GPU.

Problems on sheets of different unknown counts (ring patches of the batched workload's
geometry, differing period, radius, mesh size and scan angle) go through one call; the
results must equal those of one call per problem (the same kernels on the same inputs:
1e-12 relative in FP64) and match the FP64 oracle (1e-9 relative in FP64, |dS| <= 1e-6 in the
FP32 + refinement form).  Covered: points of several problems with the same N batched into
one factorisation, a sheet shared by two problems at different incidence (face integrals per
point), and every FP32 LU tile shape the autotuner may pick.
"""
import numpy as np
import pytest

import oracle
from pssfss_b200 import engine
from pssfss_b200.analyze import analyze, analyze_many, make_plan, sheet_gblocks, sheet_io
from pssfss_b200.elements import polyring
from pssfss_b200.layers import Layer
from pssfss_b200.units import mm

pytestmark = pytest.mark.gpu


def ring(period, ro, ntri):
    r = ro * period
    return polyring(s1=[period, 0], s2=[0, period], a=[r - 0.05 * period], b=[r], sides=24, ntri=ntri, units=mm)


def problem(sheet, freqs, theta, phi=0.0, **kw):
    plan = make_plan([Layer(), sheet, Layer()], freqs, {"θ": theta, "ϕ": phi})
    (ig, (i1, i2), isht, s), = sheet_gblocks(plan)
    ios = [sheet_io(pt.layers[i1 - 1:i2], sheet, s, pt.k0, pt.beta00) for pt in plan.points]
    return dict(sheet=sheet, rwg=plan.rwgdat[isht - 1], points=plan.points, region_rng=(i1, i2), s=s,
                u=plan.uvec[isht - 1], ios=ios, **kw)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_multi_equals_single_calls_and_oracle():
    shared = ring(8.0, 0.40, 300)
    probs = [problem(ring(6.0, 0.40, 160), [10.0, 14.0, 19.0], 0.0),
             problem(ring(12.0, 0.44, 360), [11.0, 17.0], 15.0, batch=1),
             problem(ring(6.0, 0.40, 160), [12.0, 16.0], 0.0),     # same N as the first: shared batches
             problem(shared, [10.0, 13.0], 0.0),
             problem(shared, [10.0, 13.0], 30.0)]                 # same sheet at another incidence
    probs[4]["rwg"] = probs[3]["rwg"]  # one uploaded sheet for both: its face integrals per point
    assert len({p["rwg"].nbf for p in probs}) >= 3
    multi = engine.partial_gsms_multi(probs, precision="fp64")
    for pr, got in zip(probs, multi):
        single = engine.partial_gsms(pr["sheet"], pr["rwg"], pr["points"], pr["region_rng"], pr["s"], pr["u"],
                                     pr["ios"], precision="fp64")
        i1, i2 = pr["region_rng"]
        for g, s1, pt, io in zip(got, single, pr["points"], pr["ios"]):
            assert rel(g, s1) < 1e-12
            ref, _, _ = oracle.partial_dS(pr["sheet"], pr["rwg"], pt.layers[i1 - 1:i2], pr["s"], pt.k0, pr["u"], io)
            assert rel(g, ref) < 1e-9


def test_grouped_face_integrals_at_oblique_incidence():
    # the phasing varies with frequency, so every point takes its own face integrals, computed
    # for up to four points of a batch in one launch: batches of 1 (one phasing per launch),
    # 3 (a group with an idle slot) and 6 (a group of four, then two) give the same dS, and
    # that dS matches the oracle
    sheet = ring(8.0, 0.42, 300)
    freqs = [10.0, 11.5, 13.0, 14.5, 16.0, 17.5]
    res = {}
    for batch in (1, 3, 6):
        pr = problem(sheet, freqs, 30.0, 20.0, batch=batch)
        assert len({(io.psi1, io.psi2) for io in pr["ios"]}) == len(freqs)
        res[batch] = engine.partial_gsms_multi([pr], precision="fp64")[0]
    for b in (3, 6):
        for g, r in zip(res[b], res[1]):
            assert rel(g, r) < 1e-12
    i1, i2 = pr["region_rng"]
    for k in (0, 3, 5):
        pt, io = pr["points"][k], pr["ios"][k]
        assert abs(io.psi1) > 0 and abs(io.psi2) > 0
        ref, _, _ = oracle.partial_dS(sheet, pr["rwg"], pt.layers[i1 - 1:i2], pr["s"], pt.k0, pr["u"], io)
        assert rel(res[6][k], ref) < 1e-9


@pytest.mark.parametrize("panel_w,outer_nb,batch", [(32, 128, 12), (16, 128, 5), (32, 64, 3), (16, 64, 32),
                                                    (8, 64, 7)])
def test_multi_fp32_tile_shapes(panel_w, outer_nb, batch):
    probs = [problem(ring(9.0, 0.40, 700), [10.0, 15.0, 20.0], 0.0, panel_w=panel_w, outer_nb=outer_nb, batch=batch),
             problem(ring(7.0, 0.38, 300), [12.0, 18.0], 45.0, panel_w=panel_w, outer_nb=outer_nb, batch=batch)]
    got = engine.partial_gsms_multi(probs, precision="fp32r")
    ref = engine.partial_gsms_multi(probs, precision="fp64")
    for g_p, r_p in zip(got, ref):
        for g, r in zip(g_p, r_p):
            assert np.max(np.abs(g - r)) <= 1e-6


def test_analyze_many_equals_analyze():
    cases = [([Layer(), ring(6.0, 0.40, 160), Layer()], [10.0, 20.0], {"θ": 0.0, "ϕ": 0.0}),
             ([Layer(), ring(10.0, 0.36, 260), Layer()], [12.0], {"θ": 45.0, "ϕ": 0.0})]
    many = analyze_many(cases, precision="fp64")
    for (strata, fl, st), res in zip(cases, many):
        one = analyze(strata, fl, st, precision="fp64")
        assert len(one) == len(res)
        for a, b in zip(one, res):
            for k in ((1, 1), (1, 2), (2, 1), (2, 2)):
                assert np.max(np.abs(a.gsm[k] - b.gsm[k])) <= 1e-12 * max(1.0, np.max(np.abs(a.gsm[k])))

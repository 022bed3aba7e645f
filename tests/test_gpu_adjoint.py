"""The adjoint gradient path on the GPU (pss_partial_gsms_adj, autodiff.SweepObjective).

* first-order partial GSMs against the oracle's adjoint form
  wobs_k (P_k X + Lam^T (R_k - Z_k X)): 1e-11 relative, and the perturbation itself (about
  1e-4 of dS) to 1e-6 of its size;
* the gradient of Σ_f (|S21_TE|² − |S21_TM|²) in trace width, pitch and eps_r against central
  finite differences (relative step 1e-4) of whole sweeps of this solver (analyze, FP64) and
  of the oracle: 1e-5 relative, in both precision forms;
* the autograd Function returns the same gradient through torch.autograd.
"""
import functools

import numpy as np
import pytest

import oracle
from pssfss_b200 import engine
from pssfss_b200.analyze import make_plan, sheet_gblocks, sheet_io
from pssfss_b200.gradient import meander_gradient, meander_linearized_gradient, meander_strata

pytestmark = pytest.mark.gpu

P0 = {"w": 0.3, "a": 5.0, "epsr": 2.2}


def relerr(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b))))


@pytest.mark.parametrize("precision", ["fp64", "fp32r"])
def test_adjoint_partial_gsms_match_oracle(precision):
    steps = [{**P0, "epsr": 2.2 * (1 + 1e-4)}, {**P0, "w": 0.3 * (1 - 1e-4)}, {**P0, "a": 5.0 * (1 + 1e-4)}]
    freqs, st = [9.0, 15.0], {"θ": 0.0, "ϕ": 0.0}
    plan0 = make_plan(meander_strata(P0, ntri=200), freqs, st)
    plans = [make_plan(meander_strata(p, ntri=200), freqs, st) for p in steps]
    (_, (i1, i2), _, s), = sheet_gblocks(plan0)
    sh, rw = plan0.sheets[0], plan0.rwgdat[0]
    ios0 = [sheet_io(pt.layers[i1 - 1:i2], sh, s, pt.k0, pt.beta00) for pt in plan0.points]
    pert = []
    for pl in plans:
        shk = pl.sheets[0]
        pert.append((shk, pl.rwgdat[0], pl.points, pl.uvec[0],
                     [sheet_io(pt.layers[i1 - 1:i2], shk, s, pt.k0, pt.beta00) for pt in pl.points]))
    args = (sh, rw, plan0.points, (i1, i2), s, plan0.uvec[0], ios0, pert)
    ref0, refk = oracle.partial_gsms_linearized(*args, form="adjoint")
    got0, gotk = engine.partial_gsms_adjoint(*args, precision=precision)
    for i in range(len(freqs)):
        assert relerr(got0[i], ref0[i]) < 1e-11
        for k in range(len(pert)):
            assert relerr(gotk[k][i], refk[k][i]) < 1e-11
            d = refk[k][i] - ref0[i]
            assert np.max(np.abs((gotk[k][i] - got0[i]) - d)) <= 1e-6 * np.max(np.abs(d))


@pytest.mark.parametrize("precision", ["fp64", "fp32r"])
def test_adjoint_gradient_matches_central_differences(precision):
    freqs, ntri = [9.0, 13.0, 17.0], 400
    part = functools.partial(engine.partial_gsms_adjoint, precision=precision)
    f_adj, g_adj = meander_linearized_gradient(P0, freqs, part, ntri=ntri)
    f_fd, g_fd = meander_gradient(P0, freqs, ntri=ntri, rel_step=1e-4, precision="fp64")
    f_or, g_or = meander_gradient(P0, freqs, ntri=ntri, rel_step=1e-4, analyze_fn=oracle.analyze)
    assert abs(f_adj - f_fd) <= 1e-9 * abs(f_fd) and abs(f_fd - f_or) <= 1e-9 * abs(f_or)
    for k in P0:
        assert abs(g_adj[k] - g_fd[k]) <= 1e-5 * abs(g_fd[k]), (k, g_adj[k], g_fd[k])
        assert abs(g_adj[k] - g_or[k]) <= 1e-5 * abs(g_or[k]), (k, g_adj[k], g_or[k])


def test_autograd_function_gives_the_adjoint_gradient():
    import torch
    from pssfss_b200.autodiff import meander_objective
    freqs, ntri = [10.0, 16.0], 200
    p = torch.tensor([P0["w"], P0["a"], P0["epsr"]], dtype=torch.float64, requires_grad=True)
    f = meander_objective(p, freqs, ntri=ntri, precision="fp32r")
    (g,) = torch.autograd.grad(2.0 * f, p)
    part = functools.partial(engine.partial_gsms_adjoint, precision="fp32r")
    f_ref, g_ref = meander_linearized_gradient(P0, freqs, part, ntri=ntri)
    assert abs(float(f.detach()) - f_ref) <= 1e-12 * abs(f_ref)
    for i, k in enumerate(("w", "a", "epsr")):
        assert abs(float(g[i]) - 2.0 * g_ref[k]) <= 1e-12 * abs(2.0 * g_ref[k])

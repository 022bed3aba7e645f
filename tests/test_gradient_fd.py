"""Finite-difference gradient driver of the meander differentiation workload, run through
the oracle's analyze on a small mesh (the CUDA sweep is the same call with the default
``analyze_fn``).  Objective Σ_f (|S21_TE|² − |S21_TM|²) with respect to trace width, pitch
and substrate permittivity, central differences with a 1e-4 relative step."""
import pytest

import oracle
from pssfss_b200.gradient import (fd_gradient, meander_gradient, meander_strata, meander_topology,
                                  te_tm_transmission_objective)

P0 = {"w": 0.3, "a": 5.0, "epsr": 2.2}
FREQS = [9.0, 15.0]
NTRI = 120


def test_meander_fd_gradient_converges_in_step():
    f0, g4 = meander_gradient(P0, FREQS, ntri=NTRI, rel_step=1e-4, analyze_fn=oracle.analyze)
    direct = te_tm_transmission_objective(
        oracle.analyze(meander_strata(P0, ntri=NTRI), FREQS, {"θ": 0.0, "ϕ": 0.0}))
    assert abs(f0 - direct) <= 1e-12 * max(1.0, abs(direct))
    _, g3 = meander_gradient(P0, FREQS, ntri=NTRI, rel_step=1e-3, analyze_fn=oracle.analyze)
    for k in P0:
        assert g4[k] != 0.0
        # central differences: O(h^2) truncation, so the two steps agree closely
        assert abs(g4[k] - g3[k]) <= 1e-4 * abs(g4[k]) + 1e-9, (k, g4[k], g3[k])


def test_fd_gradient_rejects_topology_change():
    # a 20% width step changes the meander's segment counts
    assert meander_topology({**P0, "w": 0.36}, ntri=NTRI) != meander_topology(P0, ntri=NTRI)
    with pytest.raises(ValueError, match="topology"):
        fd_gradient(lambda p: meander_strata(p, ntri=NTRI), P0, FREQS, {"θ": 0.0, "ϕ": 0.0},
                    te_tm_transmission_objective, rel_step=0.2,
                    topology=lambda p: meander_topology(p, ntri=NTRI), analyze_fn=oracle.analyze)


def test_linearized_gradient_matches_full_central_differences():
    # One factorisation per point (perturbed matrices enter as Λᵀ ΔZ X, perturbed sources as
    # extra right-hand sides) against two full sweeps per parameter; both are central
    # differences with the same step, so they agree to the O(h²) of the linearisation.
    from pssfss_b200.gradient import meander_linearized_gradient
    f_fd, g_fd = meander_gradient(P0, FREQS, ntri=NTRI, rel_step=1e-4, analyze_fn=oracle.analyze)
    f_lin, g_lin = meander_linearized_gradient(P0, FREQS, oracle.partial_gsms_linearized, ntri=NTRI,
                                               rel_step=1e-4)
    assert abs(f_lin - f_fd) <= 1e-12 * abs(f_fd)
    for k in P0:
        assert abs(g_lin[k] - g_fd[k]) <= 1e-5 * abs(g_fd[k]), (k, g_lin[k], g_fd[k])


def test_tangent_form_equals_adjoint_form():
    # the forward-solve form (perturbed matrices through P Z^-1 (R - Z_k X)) gives the same
    # linearised partial GSMs as the transposed-solve form, to rounding
    import functools
    from pssfss_b200.gradient import meander_linearized_gradient
    _, g_adj = meander_linearized_gradient(P0, FREQS, oracle.partial_gsms_linearized, ntri=NTRI)
    _, g_tan = meander_linearized_gradient(P0, FREQS, functools.partial(oracle.partial_gsms_linearized,
                                                                        tangent=True), ntri=NTRI)
    for k in P0:
        assert abs(g_tan[k] - g_adj[k]) <= 1e-9 * abs(g_adj[k]), (k, g_tan[k], g_adj[k])


def test_fully_adjoint_form_matches_full_central_differences():
    # dS_k = wobs_k (P_k X + Lam^T (R_k - Z_k X)): no solve per perturbed set, only the adjoint
    # solve per point; its central differences match two full sweeps per parameter to 1e-5
    import functools
    from pssfss_b200.gradient import meander_linearized_gradient
    f_fd, g_fd = meander_gradient(P0, FREQS, ntri=NTRI, rel_step=1e-4, analyze_fn=oracle.analyze)
    f_adj, g_adj = meander_linearized_gradient(P0, FREQS, functools.partial(oracle.partial_gsms_linearized,
                                                                            form="adjoint"), ntri=NTRI)
    assert abs(f_adj - f_fd) <= 1e-12 * abs(f_fd)
    for k in P0:
        assert abs(g_adj[k] - g_fd[k]) <= 1e-5 * abs(g_fd[k]), (k, g_adj[k], g_fd[k])

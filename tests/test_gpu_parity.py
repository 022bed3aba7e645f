"""CUDA path (through the C ABI) against the CPU oracle, stage by stage and end to end.

Tolerances: the CUDA kernels restate the same FP64 algorithm in a different summation
order (tree reductions, gather assembly, FFT vs the oracle's recursive DFT) and with
CUDA's transcendental functions, so FP64 results agree to ~1e-13 relative; asserted
bounds are 1e-10 relative (max-abs-difference over max-abs-value) for tables, integrals
and matrices, and 1e-9 for S-parameters.  FP32+refinement results must agree with the
FP64 oracle to |dS| <= 1e-6 absolute (the target of the precision form).
"""
import functools
import math

import numpy as np
import pytest

import oracle
from conftest import golden
from pssfss_b200 import engine
from pssfss_b200.analyze import make_plan, sheet_gblocks, sheet_io
from pssfss_b200.elements import meander, rectstrip
from pssfss_b200.layers import Layer
from pssfss_b200.rwg import setup_rwg
from pssfss_b200.sheets import s1s2_to_b1b2
from pssfss_b200.units import Length, inch, mil, mm

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b))))


def _fillzy_setup(cls, nx=20, ny=20):
    k0 = 2 * math.pi / (11.80285 / 2.0 * 2.54 / 100)
    layers = [Layer(), Layer(epsr=3.4, tandel=0.003, width=Length(1, mil)),
              Layer(epsr=3.4, tandel=0.003, width=Length(1, mil))]
    sheet = rectstrip(Nx=nx, Ny=ny, Lx=20, Ly=50, Px=100, Py=100, units=mil, **{"class": cls})
    u = 0.5 * max(np.linalg.norm(sheet.beta1), np.linalg.norm(sheet.beta2)) * sheet.units.units_per_meter
    return k0, layers, sheet, setup_rwg(sheet), u


@pytest.mark.parametrize("magnetic", [0, 1])
def test_modal_tables_match_oracle(magnetic):
    k0 = 2 * math.pi / (11.80285 / 2.0 * 2.54 / 100)
    layers = [Layer(), Layer(width=Length(20, mil), epsr=3.6, tandel=0.0013, mur=5.0),
              Layer(width=Length(10, mil), epsr=8.0, tandel=0.0013, mur=2.0),
              Layer(width=Length(50, mil), epsr=2.6, tandel=0.0003), Layer()]
    psi1, psi2 = 0.4, -0.6
    s1 = np.array([1.14 * 0.0254, 0.0])
    s2 = np.array([0.5707, 0.9885]) * 0.0254
    b1, b2 = s1s2_to_b1b2(s1, s2)
    b00 = (psi1 * b1 + psi2 * b2) / (2 * math.pi)
    u = 0.5 * max(np.linalg.norm(b1), np.linalg.norm(b2))
    ref = oracle.modal_tables(magnetic, k0, u, psi1, psi2, layers, 2, b1, b2, b00, 1e-7)
    mm_, t1, t2, st = engine.modal_tables(magnetic, k0, u, psi1, psi2, layers, 2, b1, b2, 1e-7)
    assert mm_ == ref.mmax
    assert relerr(t1, ref.t1) < 1e-10 and relerr(t2, ref.t2) < 1e-10


@pytest.mark.parametrize("psi", [(0.0, 0.0), (0.7, -0.3)])
def test_face_integrals_match_oracle(psi):
    k0, layers, sheet, rwg, u = _fillzy_setup("J", 6, 6)
    ul = u / sheet.units.units_per_meter
    ref = oracle.filljk(sheet, rwg, ul, *psi)
    got = engine.face_integrals(sheet, rwg, ul, *psi)
    for k in ("J", "Jxi", "Jeta", "K", "Kxi", "Keta"):
        assert relerr(got[k], getattr(ref, k)) < 1e-11, k
    assert relerr(got["rho_r"], ref.rho_r) < 1e-11
    assert relerr(got["rinv"], ref.rinv) < 1e-11
    assert got["nonconv"] == ref.nonconv == 0


@pytest.mark.parametrize("cls", ["J", "M"])
def test_fill_matches_oracle_and_golden(cls):
    k0, layers, sheet, rwg, u = _fillzy_setup(cls)
    Zr, info = oracle.fill(k0, u, layers, 2, 0.0, 0.0, sheet, rwg)
    Zg, mmax = engine.fill_matrix(sheet, rwg, layers, 2, u, k0, 0.0, 0.0)
    assert mmax == info["mmax"]
    assert relerr(Zg, Zr) < 1e-10
    vals, g = golden("fillz" if cls == "J" else "filly")  # test/FillZY_test.jl:45-46, 77-78
    for (i, j), v in zip(g["index_1based"], vals):
        assert abs(Zg[i - 1, j - 1] - v) / abs(v) < 1e-10


def test_fill_oblique_periodic_strip_with_loss():
    # ψ != 0, cell-spanning strip (periodic boundary basis functions, Floquet flags) and
    # a sheet resistance (surface loading terms): every assembly branch.
    k0 = 2 * math.pi * 12e9 / 299792458.0
    layers = [Layer(), Layer(epsr=2.2, width=Length(1, mm)), Layer()]
    sheet = rectstrip(Nx=4, Ny=6, Lx=10, Ly=3, Px=10, Py=8, units=mm, Rsheet=12.5)
    rwg = setup_rwg(sheet)
    assert (rwg.eci != 0).any()
    u = 0.5 * max(np.linalg.norm(sheet.beta1), np.linalg.norm(sheet.beta2)) * 1000
    Zr, _ = oracle.fill(k0, u, layers, 1, 0.9, -0.4, sheet, rwg)
    Zg, _ = engine.fill_matrix(sheet, rwg, layers, 1, u, k0, 0.9, -0.4)
    assert relerr(Zg, Zr) < 1e-10


def test_basis_transforms_golden():
    # test/RWGData_test.jl:56-58
    sheet = rectstrip(Lx=1, Ly=1, Px=1, Py=1, Nx=2, Ny=1, units=inch, fufp=False)
    rwg = setup_rwg(sheet)
    F = engine.basis_transforms(sheet, rwg, [[20.0, -30.3], [0.0, 0.0]], 0.8, -0.7)
    vals, _ = golden("rwgbfft_inch")
    assert np.allclose(F[0, :3], np.reshape(vals, (3, 2)), rtol=1e-12, atol=0)
    assert relerr(F[1], oracle.rwgbfft(rwg, sheet, [0.0, 0.0], 0.8, -0.7)) < 1e-12


@pytest.mark.parametrize("m,n,k", [(128, 128, 16), (300, 260, 128), (1000, 777, 100), (5, 3, 7)])
def test_schur_update_tensor_cores(m, n, k):
    """C - L U on the tcgen05 3xTF32 kernel against FP64: FP32-level error (a single TF32
    product would be ~1e-3 relative), on full, ragged and sub-tile shapes."""
    rng = np.random.default_rng(m * 7 + n + k)
    cplx = lambda *s: (rng.standard_normal(s) + 1j * rng.standard_normal(s)).astype(np.complex64)
    L, U, C = cplx(m, k), cplx(k, n), cplx(m, n)
    out, st = engine.schur_update(L, U, C)
    ref = C.astype(np.complex128) - L.astype(np.complex128) @ U.astype(np.complex128)
    scale = np.abs(L).astype(np.float64) @ np.abs(U).astype(np.float64) + np.abs(C)
    assert st == 0
    assert float(np.max(np.abs(out - ref) / scale)) < 4e-6


@pytest.mark.parametrize("precision", ["fp64", "fp32r"])
@pytest.mark.parametrize("n", [37, 700, 1300])
def test_lu_solve_matches_lapack(precision, n):
    rng = np.random.default_rng(n)
    Z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3 * np.sqrt(n) * np.eye(n)
    B = rng.standard_normal((n, 5)) + 1j * rng.standard_normal((n, 5))
    X, st = engine.lu_solve(Z, B, precision)
    Xr = oracle.lu_solve(Z, B)
    assert st == 0
    assert relerr(X, Xr) < 1e-11


def _apply_ipiv(A, ipiv):
    P = np.array(A, copy=True)
    for j, p in enumerate(ipiv):
        if p - 1 != j:
            P[[j, p - 1]] = P[[p - 1, j]]
    return P


@pytest.mark.parametrize("n,dominant", [(700, False), (1300, True), (1300, False), (3000, False)])
def test_fp32_factor_against_lapack_cgetrf(n, dominant):
    # The FP32 factorisation of the FP32 + refinement form on its own: P Z = L U with LAPACK's
    # interchange convention, multipliers bounded by the |re|+|im| pivot rule, and a backward
    # error within a small factor of LAPACK cgetrf's on the same complex64 matrix (the
    # trailing updates run as 3xTF32 products on the tensor cores).
    import scipy.linalg as sl
    rng = np.random.default_rng(n + dominant)
    Z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    if dominant:
        Z += 3 * np.sqrt(n) * np.eye(n)
    Z32 = Z.astype(np.complex64).astype(complex)
    lu_l, piv_l = sl.lu_factor(Z.astype(np.complex64))
    L_l = np.tril(lu_l.astype(complex), -1) + np.eye(n)
    back_l = np.linalg.norm(_apply_ipiv(Z32, piv_l + 1) - L_l @ np.triu(lu_l.astype(complex))) / np.linalg.norm(Z32)
    LU, ipiv, info = engine.lu32_factor(Z)
    assert info == 0
    assert ((ipiv >= np.arange(1, n + 1)) & (ipiv <= n)).all()
    L = np.tril(LU.astype(complex), -1) + np.eye(n)
    U = np.triu(LU.astype(complex))
    back = np.linalg.norm(_apply_ipiv(Z32, ipiv) - L @ U) / np.linalg.norm(Z32)
    assert back < 10 * back_l, (back, back_l)
    assert np.max(np.abs(L)) <= np.sqrt(2) + 1e-5
    assert np.max(np.abs(U)) / np.max(np.abs(Z32)) < 100
    if dominant:  # no interchanges are needed, and none are made
        assert (ipiv == np.arange(1, n + 1)).all()


def test_lu_solve_mom_matrix_fp32_refinement():
    # The FillZY_test matrix (1-mil substrates) has cond(Z) ~ 2.2e6: two FP64 LAPACK
    # drivers already differ by ~1.5e-10 on it, and rounding Z to FP32 alone moves the
    # solution by ~4e-3.  Bounds: forward error <= cond * 1e-15, backward error ~eps.
    k0, layers, sheet, rwg, u = _fillzy_setup("J")
    Z, _ = oracle.fill(k0, u, layers, 2, 0.0, 0.0, sheet, rwg)
    B = np.random.default_rng(1).standard_normal((rwg.nbf, 4)) + 0j
    Xr = oracle.lu_solve(Z, B)
    kappa = np.linalg.cond(Z)
    for prec in ("fp64", "fp32r"):
        X, st = engine.lu_solve(Z, B, prec)
        # FP32 refinement contracts by ~cond*eps32 ~ 0.1 per step here; it either
        # converges or the point is redone in FP64 (status bit 32), never returned inaccurate
        assert st in ((0,) if prec == "fp64" else (0, 32)), (prec, st)
        # refinement stops at backward error eps*sqrt(n)*||A|| (LAPACK zcgesv): forward
        # error is then bounded by cond * eps * sqrt(n)
        bound = kappa * 1e-15 if prec == "fp64" else 2 * kappa * 1.1e-16 * np.sqrt(Z.shape[0])
        assert relerr(X, Xr) < bound, prec
        # normwise backward error in the refinement's own norm: ||r||inf / (||Z||inf ||x||inf)
        back = np.max(np.abs(Z @ X - B)) / (np.max(np.sum(np.abs(Z), axis=1)) * np.max(np.abs(X)))
        assert back < 2 * 1.1e-16 * np.sqrt(Z.shape[0]), prec


def _partial_case(strata, freqs, steering, precision):
    plan = make_plan(strata, freqs, steering)
    (ig, (i1, i2), isht, s), = sheet_gblocks(plan)
    sheet, rwg, u = plan.sheets[isht - 1], plan.rwgdat[isht - 1], plan.uvec[isht - 1]
    ios = [sheet_io(pt.layers[i1 - 1:i2], sheet, s, pt.k0, pt.beta00) for pt in plan.points]
    got = engine.partial_gsms(sheet, rwg, plan.points, (i1, i2), s, u, ios, precision=precision)
    ref = []
    for pt in plan.points:
        region = pt.layers[i1 - 1:i2]
        io = sheet_io(region, sheet, s, pt.k0, pt.beta00)
        dS, _, _ = oracle.partial_dS(sheet, rwg, region, s, pt.k0, u, io)
        ref.append(dS)
    return got, ref


@pytest.mark.parametrize("cls", ["J", "M"])
def test_partial_gsm_normal_incidence(cls):
    sheet = rectstrip(Lx=8, Ly=8, Px=10, Py=10, Nx=8, Ny=8, units=mm, **{"class": cls})
    strata = [Layer(), sheet, Layer(epsr=2.2, width=Length(1, mm)), Layer()]
    got, ref = _partial_case(strata, [10.0, 15.0, 20.0], {"θ": 0, "ϕ": 0}, "fp64")
    for g, r in zip(got, ref):
        assert np.max(np.abs(g - r)) / np.max(np.abs(r)) < 1e-9


def test_partial_gsm_oblique_theta_phi():
    # θ steering: ψ changes with frequency, so the face integrals are refreshed per point
    sheet = rectstrip(Lx=6, Ly=2, Px=8, Py=8, Nx=6, Ny=2, units=mm)
    strata = [Layer(), sheet, Layer(epsr=3.0, tandel=0.002, width=Length(0.5, mm)), Layer()]
    got, ref = _partial_case(strata, [5.0, 12.0], {"θ": 30, "ϕ": 45}, "fp64")
    for g, r in zip(got, ref):
        assert np.max(np.abs(g - r)) / np.max(np.abs(r)) < 1e-9


def test_partial_gsm_fp32_refinement_meander():
    sheet = meander(a=5, b=10, h=6, w1=0.3, w2=0.3, ntri=300, units=mm)
    strata = [Layer(), sheet, Layer(epsr=2.2, width=Length(1, mm)), Layer()]
    got, ref = _partial_case(strata, [8.0, 13.0, 18.0], {"θ": 0, "ϕ": 0}, "fp32r")
    for g, r in zip(got, ref):
        assert np.max(np.abs(g - r)) <= 1e-6
        assert np.max(np.abs(g - r)) / np.max(np.abs(r)) < 1e-9


@pytest.mark.parametrize("cls", ["J", "M"])
def test_analyze_strip_grating(cls):
    from pssfss_b200 import analyze
    from test_oracle_golden import _grating
    F = 0.8
    r, t = _grating(2 * math.pi * F)
    ex = {(1, 1): np.array([[r, 0], [0, -t]]), (2, 1): np.array([[t, 0], [0, -r]])}
    ex[(2, 2)], ex[(1, 2)] = ex[(1, 1)], ex[(2, 1)]
    period = 299792458.0 * 100 / 2.54 * 1e-9
    Py, Ly = period, period / 2
    Px = Lx = Ly / 10
    sh = rectstrip(Px=Px, Py=Py, Lx=Lx, Ly=Ly, Nx=4, Ny=40, units=inch, **{"class": cls})
    res = analyze([Layer(), sh, Layer()], F, {"θ": 0, "ϕ": 0})
    ref = oracle.analyze([Layer(), sh, Layer()], F, {"θ": 0, "ϕ": 0})
    for k in ex:
        assert np.abs(res[0].gsm[k] - ex[k]).max() < 0.01   # test/full_test.jl:76,91
        assert np.abs(res[0].gsm[k] - ref[0].gsm[k]).max() < 1e-9


def test_status_flags_singular_matrix():
    Z = np.zeros((8, 8), complex)
    Z[np.arange(7), np.arange(7)] = 1.0
    X, st = engine.lu_solve(Z, np.ones((8, 1)), "fp64")
    assert st & 4


def _gsm_relerr(res, ref):
    worst = 0.0
    assert len(res) == len(ref)
    for a, b in zip(res, ref):
        assert a.FGHz == b.FGHz
        for k in ((1, 1), (1, 2), (2, 1), (2, 2)):
            worst = max(worst, float(np.max(np.abs(a.gsm[k] - b.gsm[k]))))
    return worst


def test_square_patch_sweep():
    """8 mm square patch in a 10 mm cell (structured, 512 triangles,
    N = 736) in free space, normal incidence, 11 frequencies 10-20 GHz; the FP32 form is held
    to |dS| <= 1e-6 of the FP64 oracle on the same sweep."""
    from pssfss_b200 import analyze
    sh = rectstrip(Lx=8, Ly=8, Px=10, Py=10, Nx=16, Ny=16, units=mm)
    strata = [Layer(), sh, Layer()]
    freqs = np.linspace(10, 20, 11)
    ref = oracle.analyze(strata, freqs, {"θ": 0, "ϕ": 0})
    assert _gsm_relerr(analyze(strata, freqs, {"θ": 0, "ϕ": 0}), ref) < 1e-9
    assert _gsm_relerr(analyze(strata, freqs, {"θ": 0, "ϕ": 0}, precision="fp32r"), ref) <= 1e-6


def test_two_sheet_cascade_oblique_scan():
    """Two sheets cascaded through GSMs with a lossy substrate and an air gap: a conductor
    strip sheet and an aperture (M-type) sheet, scan θ=30°, ϕ=45° (ψ changes with frequency,
    so the face-pair integrals are recomputed per point), 3 frequencies 5-25 GHz."""
    from pssfss_b200 import analyze
    j = rectstrip(Lx=6, Ly=0.5, Px=8, Py=8, Nx=12, Ny=2, units=mm)
    m = rectstrip(Lx=6, Ly=6, Px=8, Py=8, Nx=8, Ny=8, units=mm, **{"class": "M"})
    strata = [Layer(), j, Layer(epsr=3.0, tandel=0.002, width=Length(0.5, mm)), Layer(width=Length(2, mm)), m,
              Layer()]
    freqs = [5.0, 15.0, 25.0]
    steer = {"θ": 30, "ϕ": 45}
    ref = oracle.analyze(strata, freqs, steer)
    assert _gsm_relerr(analyze(strata, freqs, steer), ref) < 1e-9
    assert _gsm_relerr(analyze(strata, freqs, steer, precision="fp32r"), ref) <= 1e-6


def test_jerusalem_cross_and_aperture_cascade():
    """Two-sheet cascade: a (solid) Jerusalem-cross
    conductor on 0.5 mm eps_r = 3 (tan d = 0.002), a 2 mm air gap, then a 6 mm square
    aperture (M-type) in an 8 mm cell; scan theta = 30, phi = 45 (face-pair integrals per
    point).  Own structured meshes (the reference meshes these with Triangle), coarse enough
    for the oracle; CUDA vs oracle GSMs to 1e-9."""
    from pssfss_b200 import analyze
    from pssfss_b200.elements import jerusalemcross
    jc = jerusalemcross(P=8, L1=6, L2=0.5, A=3, B=0.5, w=0.5, ntri=300, units=mm)
    ap = rectstrip(Lx=6, Ly=6, Px=8, Py=8, Nx=6, Ny=6, units=mm, **{"class": "M"})
    strata = [Layer(), jc, Layer(epsr=3.0, tandel=0.002, width=Length(0.5, mm)), Layer(width=Length(2, mm)), ap,
              Layer()]
    freqs = [7.0, 16.0]
    steer = {"θ": 30, "ϕ": 45}
    ref = oracle.analyze(strata, freqs, steer)
    assert _gsm_relerr(analyze(strata, freqs, steer), ref) < 1e-9
    assert _gsm_relerr(analyze(strata, freqs, steer, precision="fp32r"), ref) <= 1e-6


@pytest.mark.parametrize("period,ro,ntri,theta", [(6.0, 0.40, 160, 0.0), (9.0, 0.36, 260, 15.0),
                                                  (12.0, 0.44, 360, 45.0)])
def test_ring_patches_of_varied_size(period, ro, ntri, theta):
    """Ring-patch problems of a batch whose members differ (period, outer radius and
    triangle count vary per problem, so do the unknown counts; scan theta in {0, 15, 45}),
    free-standing, 2 frequencies each, FP32 + refinement against the FP64 oracle."""
    from pssfss_b200 import analyze
    from pssfss_b200.elements import polyring
    r_out = ro * period
    sh = polyring(s1=[period, 0], s2=[0, period], a=[r_out - 0.05 * period], b=[r_out], sides=24, ntri=ntri,
                  units=mm)
    strata = [Layer(), sh, Layer()]
    freqs = [10.0, 20.0]
    steer = {"θ": theta, "ϕ": 0}
    ref = oracle.analyze(strata, freqs, steer)
    assert _gsm_relerr(analyze(strata, freqs, steer, precision="fp32r"), ref) <= 1e-6
    assert _gsm_relerr(analyze(strata, freqs, steer), ref) < 1e-9


@pytest.mark.parametrize("precision", ["fp64", "fp32r"])
def test_linearised_partial_gsms_and_gradient(precision):
    """pss_partial_gsms_lin on a small meanderline (two perturbed sets: eps_r of the substrate,
    and the trace width, a second sheet of the same topology) against the oracle's
    forward-solve form, and the one-factorisation gradient through it against the oracle's."""
    from pssfss_b200 import engine
    from pssfss_b200.analyze import make_plan, sheet_gblocks, sheet_io
    from pssfss_b200.gradient import meander_linearized_gradient, meander_strata
    P0 = {"w": 0.3, "a": 5.0, "epsr": 2.2}
    steps = [{**P0, "epsr": 2.2 * (1 + 1e-4)}, {**P0, "w": 0.3 * (1 + 1e-4)}]
    freqs, st = [9.0, 15.0], {"θ": 0.0, "ϕ": 0.0}
    plan0 = make_plan(meander_strata(P0, ntri=120), freqs, st)
    plans = [make_plan(meander_strata(p, ntri=120), freqs, st) for p in steps]
    (_, (i1, i2), _, s), = sheet_gblocks(plan0)
    sh, rw = plan0.sheets[0], plan0.rwgdat[0]
    ios0 = [sheet_io(pt.layers[i1 - 1:i2], sh, s, pt.k0, pt.beta00) for pt in plan0.points]
    pert = []
    for pl in plans:
        shk = pl.sheets[0]
        pert.append((shk, pl.rwgdat[0], pl.points, pl.uvec[0],
                     [sheet_io(pt.layers[i1 - 1:i2], shk, s, pt.k0, pt.beta00) for pt in pl.points]))
    ref0, refk = oracle.partial_gsms_linearized(sh, rw, plan0.points, (i1, i2), s, plan0.uvec[0], ios0, pert,
                                                tangent=True)
    got0, gotk = engine.partial_gsms_linearized(sh, rw, plan0.points, (i1, i2), s, plan0.uvec[0], ios0, pert,
                                                precision=precision)
    for i in range(len(freqs)):
        assert relerr(got0[i], ref0[i]) < 1e-11
        for k in range(len(pert)):
            assert relerr(gotk[k][i], refk[k][i]) < 1e-11
            # the perturbation itself (~1e-4 of dS) to 1e-6 of its size
            d = refk[k][i] - ref0[i]
            assert np.max(np.abs((gotk[k][i] - got0[i]) - d)) <= 1e-6 * np.max(np.abs(d))
    part = functools.partial(engine.partial_gsms_linearized, precision=precision)
    _, g_dev = meander_linearized_gradient(P0, freqs, part, ntri=120)
    _, g_ref = meander_linearized_gradient(P0, freqs, functools.partial(oracle.partial_gsms_linearized, tangent=True),
                                           ntri=120)
    for k in P0:
        assert abs(g_dev[k] - g_ref[k]) <= 1e-6 * abs(g_ref[k]), (k, g_dev[k], g_ref[k])


def test_pipeline_wait_timeout_reports_status_and_context_survives():
    """Bounded waits of the tensor-core update: with a limit of one poll the TMA / MMA /
    epilogue hand-offs run out (the epilogue's first wait spans a whole 128 x 128 x 1024 tile
    of MMAs, far longer than one poll), the call returns PSS_STATUS_DEVICE_TIMEOUT (64) instead of
    hanging, the kernel drains its copies and MMAs at the default limit before it frees its
    tensor memory, and the context stays usable: with the default limit restored the same
    update is exact to FP32 level again."""
    lib = engine.lib()
    rng = np.random.default_rng(5)
    cplx = lambda *s: (rng.standard_normal(s) + 1j * rng.standard_normal(s)).astype(np.complex64)
    L, U, C = cplx(256, 1024), cplx(1024, 256), cplx(256, 256)
    try:
        assert lib.pss_set_wait_limit(1) == 0
        _, st = engine.schur_update(L, U, C)
        assert st == 64
    finally:
        assert lib.pss_set_wait_limit(0) == 0
    out, st = engine.schur_update(L, U, C)
    ref = C.astype(np.complex128) - L.astype(np.complex128) @ U.astype(np.complex128)
    scale = np.abs(L).astype(np.float64) @ np.abs(U).astype(np.float64) + np.abs(C)
    assert st == 0 and float(np.max(np.abs(out - ref) / scale)) < 4e-6
    assert lib.pss_set_wait_limit(-1) == -1

"""The package's host numerics against the oracle's independent restatement (oracle/host.py).

The CUDA library computes only the sheet's scattered partial GSM; the modal constants, the
Gblock's incident GSM and transmission-line Green's functions, the source and projection
factors and the cascade run on the host in the package (modes.py, gsms.py, analyze.py).
oracle/host.py restates the same reference code (Modes.jl:298-322, GSMs.jl:125-176,
213-620, 717-750, PSSFSS.jl:226-312, 362-587) without importing the package, so these
tests compare two separately written host paths, on the CPU:
  * modal constants per layer and point: 1e-13 relative;
  * electric / magnetic Gblock GSMs, TLGFs and incident voltages / currents: 1e-12;
  * a sheet's whole partial GSM (same fill and LU, the package's generic source / projection
    form against the reference's own form): 1e-11;
  * whole analyses (package host + oracle hot path against the all-oracle analyze): 1e-10.
"""
import math

import numpy as np
import pytest

import oracle
from oracle import host
from pssfss_b200.analyze import add_scattered, assemble, make_plan, sheet_gblocks, sheet_io
from pssfss_b200.gsms import gsm_electric_gblock, gsm_magnetic_gblock, gsm_slab_interface
from pssfss_b200.layers import Layer
from pssfss_b200.units import Length, mm


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    d = np.max(np.abs(a - b)) if a.size else 0.0
    return d / max(np.max(np.abs(b)) if b.size else 0.0, 1e-300)


def _base(plan):
    return [host.ModalLayer(l.epsr, l.mur, l.width, list(l.P), list(l.M), list(l.N),
                            np.array(l.beta1, float), np.array(l.beta2, float)) for l in plan.layers]


def _stacks(pkg):
    strip = pkg.rectstrip(Lx=8, Ly=8, Px=10, Py=10, Nx=6, Ny=6, units=mm)
    slot = pkg.rectstrip(Lx=6, Ly=2, Px=8, Py=8, Nx=6, Ny=3, units=mm, **{"class": "M"})
    return {
        "J on substrate, normal": ([Layer(), strip, Layer(epsr=2.2, width=Length(1, mm)), Layer()], [12.0, 19.0],
                                   {"θ": 0.0, "ϕ": 0.0}),
        "J oblique": ([Layer(), strip, Layer(epsr=3.0, tandel=0.002, width=Length(0.5, mm)), Layer()], [14.0],
                      {"θ": [0.0, 30.0], "ϕ": 45.0}),
        "M in a slab": ([Layer(), Layer(epsr=2.5, width=Length(0.8, mm)), slot, Layer(width=Length(2, mm)), Layer()],
                        [11.0], {"θ": 20.0, "ϕ": 10.0}),
        "psi steering": ([Layer(), strip, Layer()], [15.0], {"ψ₁": 30.0, "ψ₂": [0.0, 20.0]}),
    }


@pytest.mark.parametrize("name", ["J on substrate, normal", "J oblique", "M in a slab", "psi steering"])
def test_modal_constants_and_gblocks_match_the_restatement(pkg, name):
    strata, freqs, steer = _stacks(pkg)[name]
    plan = make_plan(strata, freqs, steer)
    base = _base(plan)
    sh0 = plan.sheets[0]
    upm = sh0.units.units_per_meter
    pts = host.steering_points(base, [float(f) for f in freqs], steer, (sh0.beta1 * upm, sh0.beta2 * upm))
    assert len(pts) == len(plan.points) > 0
    for pt, (st, f, k0, b00, ml) in zip(plan.points, pts):
        assert pt.fghz == f and math.isclose(pt.k0, k0, rel_tol=1e-15)
        assert rel(pt.beta00, b00) < 1e-14 or np.max(np.abs(b00)) == 0
        for L, M in zip(pt.layers, ml):
            for a, b in ((L.beta, M.beta), (L.gamma, M.gamma), (L.Y, M.Y), (L.c, M.c), (L.tvec, M.tvec)):
                assert rel(a, b) < 1e-13, name
        for ig, (i1, i2), isht, s in sheet_gblocks(plan):
            sheet = plan.sheets[isht - 1]
            fn, fo = ((gsm_electric_gblock, host.electric_gblock) if sheet.cls == "J"
                      else (gsm_magnetic_gblock, host.magnetic_gblock))
            g, tl, vi = fn(pt.layers[i1 - 1:i2], s, pt.k0)
            go, tlo, vio = fo(ml[i1 - 1:i2], s, k0)
            for blk in ("s11", "s12", "s21", "s22"):
                assert rel(getattr(g, blk), go[blk]) < 1e-12, (name, blk)
            assert rel(tl, tlo) < 1e-12 and rel(vi, vio) < 1e-12, name
        for g in plan.gbls:
            if g.j == 0:
                a = gsm_slab_interface(pt.layers[g.first - 1], pt.layers[g.first], pt.k0)
                b = host.slab_interface(ml[g.first - 1], ml[g.first], k0)
                for blk in ("s11", "s12", "s21", "s22"):
                    assert rel(getattr(a, blk), b[blk]) < 1e-12


@pytest.mark.parametrize("name", ["J on substrate, normal", "M in a slab"])
def test_sheet_partial_gsm_generic_form_matches_reference_form(pkg, name):
    # The package hands the library generic source vectors and projection weights
    # (sheet_io); the oracle's host restates calculate_*type_gsm in the reference's own terms.
    # With the same fill and LU, the two partial GSMs agree.
    import scipy.linalg as sl
    strata, freqs, steer = _stacks(pkg)[name]
    plan = make_plan(strata, freqs, steer)
    (ig, (i1, i2), isht, s), = sheet_gblocks(plan)
    sheet, rwg, u = plan.sheets[isht - 1], plan.rwgdat[isht - 1], plan.uvec[isht - 1]
    base = _base(plan)
    upm = sheet.units.units_per_meter
    pts = host.steering_points(base, [float(f) for f in freqs], steer, (sheet.beta1 * upm, sheet.beta2 * upm))
    for pt, (st, f, k0, b00, ml) in zip(plan.points, pts):
        region = pt.layers[i1 - 1:i2]
        io = sheet_io(region, sheet, s, pt.k0, pt.beta00)
        dS, Z, _ = oracle.partial_dS(sheet, rwg, region, s, pt.k0, u, io)
        g = add_scattered(io, dS)
        lu = sl.lu_factor(Z)
        area = abs(sheet.s1[0] * sheet.s2[1] - sheet.s1[1] * sheet.s2[0]) / upm ** 2
        mreg = ml[i1 - 1:i2]
        ends = (mreg[0], mreg[-1])
        go = host.sheet_partial_gsm(sheet.cls, mreg, s, k0, area, lambda b: sl.lu_solve(lu, b),
                                    lambda r, q: oracle.rwgbfft(rwg, sheet, ends[r].beta[q], io.psi1, io.psi2))
        for blk in ("s11", "s12", "s21", "s22"):
            assert rel(getattr(g, blk), go[blk]) < 1e-11, (name, blk, rel(getattr(g, blk), go[blk]))


@pytest.mark.parametrize("name", ["J oblique", "M in a slab", "psi steering"])
def test_whole_analysis_host_paths_agree(pkg, name):
    # the package's host path (plan, sheet_io, cascade) around the oracle's hot path, against
    # oracle.analyze (all numerics restated independently)
    strata, freqs, steer = _stacks(pkg)[name]
    plan = make_plan(strata, freqs, steer)
    partial = {}
    for ig, (i1, i2), isht, s in sheet_gblocks(plan):
        sheet = plan.sheets[isht - 1]
        out = []
        for pt in plan.points:
            region = pt.layers[i1 - 1:i2]
            io = sheet_io(region, sheet, s, pt.k0, pt.beta00)
            dS, _, _ = oracle.partial_dS(sheet, plan.rwgdat[isht - 1], region, s, pt.k0, plan.uvec[isht - 1], io)
            out.append(add_scattered(io, dS))
        partial[ig] = out
    mine = assemble(plan, partial)
    ref = oracle.analyze(strata, freqs, steer)
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        assert a.FGHz == b.FGHz and a.steering == b.steering
        for blk in ("s11", "s12", "s21", "s22"):
            assert rel(getattr(a.gsm, blk), getattr(b.gsm, blk)) < 1e-10, (name, blk)


def test_cascade_identities_of_the_restatement():
    # GSMs_test.jl:17-95 style: cascading with an identity GSM changes nothing, and a
    # zero-width layer propagates nothing
    rng = np.random.default_rng(3)
    n = 4
    a = {k: rng.normal(size=(n, n)) * 0.3 + 1j * rng.normal(size=(n, n)) * 0.3 for k in ("s11", "s12", "s21", "s22")}
    c = host.cascade(a, host.new_gsm(n, n))
    for blk in a:
        assert rel(c[blk], a[blk]) < 1e-15
    c = host.cascade(host.new_gsm(n, n), a)
    for blk in a:
        assert rel(c[blk], a[blk]) < 1e-15

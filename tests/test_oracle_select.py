"""The oracle's restatements of the steps before the numerics - Gblocks, layer modes and
duplicate Gblocks (oracle/select.py), the basis-function topology (oracle/rwg.py) - against
the reference's golden values, then against the package on the CPU.

Neither oracle file imports the package, so the second group compares two separately
written restatements of choose_gblocks (GSMs.jl:771-868), choose_layer_modes! (Modes.jl:49-275,
with fill_mmax_pmn! and select_pmn!, :367-431), get_gbldup (PSSFSS.jl:675-704) and setup_rwg
(RWG.jl:90-324): the Gblock ranges and sheet junctions, every layer's mode list (p, m, n in
order) and reciprocal lattice, the duplicate map, the basis functions, boundary codes and
face-pair classes must be identical.
"""
import math

import numpy as np
import pytest

from conftest import golden
from oracle import select as S
from pssfss_b200.analyze import make_plan
from pssfss_b200.layers import Layer
from pssfss_b200.units import Length, cm, inch, mil, mm


def _is_layer(x):
    return isinstance(x, Layer)


def _ring(p):
    from pssfss_b200.elements import polyring
    return polyring(sides=4, orient=45, a=[0.1902], b=[0.2169], units=inch, s1=[p, 0], s2=[0, p], ntri=100)


def _duroid():
    return Layer(name="Duroid 6035", epsr=3.6, tandel=0.0013, width=Length(20, mil))


def _vac(w=None, u=inch):
    return Layer(name="Vacuum") if w is None else Layer(name="Vacuum", width=Length(w, u))


def test_gblocks_golden():
    """test/GSMs_test.jl choose_gblocks1..4."""
    from pssfss_b200.elements import rectstrip

    def strip():
        return rectstrip(units=cm, Px=1, Py=1, Lx=0.5, Ly=0.5, Nx=10, Ny=10)

    cases = [
        ([Layer(), strip(), Layer(width=Length(1, mil), epsr=2.2), Layer(width=Length(1, mil)),
          Layer(width=Length(3, mm)), strip(), Layer(width=Length(1, mil), epsr=2.2), Layer()], 10e9),
        ([_vac(), _duroid(), _ring(0.5117), _duroid(), _vac(0.05), _duroid(), _ring(0.5117), _duroid(), _vac()], 2e9),
        ([_vac(), _duroid(), _ring(0.5117), _duroid(), _duroid(), _ring(0.5117), _duroid(), _vac()], 2e9),
        ([_vac(), _duroid(), _ring(0.5117), _duroid(), _vac(5, mil), _duroid(), _ring(0.5117), _duroid(),
          _vac(5, mil), _duroid(), _ring(0.5117), _duroid(), _vac()], 2e9),
    ]
    want = [c["gblocks"] for c in golden("gblocks")[1]["cases"]]
    for (strata, f), expect in zip(cases, want):
        layers, sheets, junc = S.junctions(strata, _is_layer)
        got = S.gblocks(layers, sheets, junc, 2 * math.pi * f / S.C0)
        assert [list(g) for g in got] == expect


def test_layer_mode_counts_golden():
    """test/Modes_test.jl: modes per layer for two ring screens on Duroid, 2-8 GHz, dbmin 25."""
    cases = [
        [_vac(), _duroid(), _ring(0.5117), _duroid(), _vac(0.2), _duroid(), _ring(0.5117), _duroid(), _vac()],
        [_vac(), _duroid(), _ring(0.5117), _duroid(), _vac(0.1), _vac(0.1), _duroid(), _ring(0.9005), _duroid(),
         _vac()],
        [_vac(), _duroid(), _ring(0.5117), _duroid(), _vac(0.1), _vac(0.1), _duroid(), _ring(0.5117), _duroid(),
         _vac()],
    ]
    want = [c["counts"] for c in golden("layer_mode_counts")[1]["cases"]]
    for strata, expect in zip(cases, want):
        layers, sheets, junc = S.junctions(strata, _is_layer)
        k0min, k0max = 2 * math.pi * 2e9 / S.C0, 2 * math.pi * 8e9 / S.C0
        gbls = S.gblocks(layers, sheets, junc, k0min)
        modes = S.layer_modes(layers, sheets, junc, gbls, k0max, 25.0)
        assert [0 if m is None else len(m["modes"]) for m in modes[1:]] == expect


def _stacks():
    from pssfss_b200.elements import meander, pecsheet, rectstrip
    strip = rectstrip(Lx=8, Ly=8, Px=10, Py=10, Nx=6, Ny=6, units=mm)
    small = rectstrip(Lx=3, Ly=3, Px=5, Py=5, Nx=4, Ny=4, units=mm)
    slot = rectstrip(Lx=6, Ly=2, Px=8, Py=8, Nx=6, Ny=3, units=mm, **{"class": "M"})
    mnd = meander(a=5, b=10, h=6, w1=0.3, w2=0.3, ntri=200, units=mm)
    sub = lambda w, e=2.2: Layer(epsr=e, width=Length(w, mm))  # noqa: E731
    return [
        ([Layer(), strip, Layer()], [10.0, 20.0]),
        ([Layer(), strip, sub(1.0), Layer()], [8.0, 18.0]),
        ([Layer(), mnd, sub(1.0), Layer()], [8.0, 18.0]),
        ([Layer(), strip, sub(0.5, 3.0), Layer(width=Length(2, mm)), slot, Layer()], [5.0, 25.0]),
        ([Layer(), sub(0.8, 2.5), slot, Layer(width=Length(2, mm)), Layer()], [11.0]),
        # the same sheet object four times between equal layers: the third Gblock repeats the second
        ([Layer(), strip, sub(0.1), Layer(width=Length(6, mm)), sub(0.1), strip, sub(0.1), Layer(width=Length(6, mm)),
          sub(0.1), strip, sub(0.1), Layer(width=Length(6, mm)), sub(0.1), strip, Layer()], [9.0, 12.0]),
        # sheets of different cells with a thick gap, then a thin one
        ([Layer(), strip, Layer(width=Length(5, mm)), small, Layer()], [10.0, 14.0]),
        ([Layer(), strip, sub(0.2), small, Layer()], [10.0, 14.0]),
        # a null sheet inside the stack and at its end
        ([Layer(), strip, sub(0.3), pecsheet(), sub(0.4), Layer()], [6.0, 9.0]),
        ([Layer(), sub(0.3), strip, Layer(width=Length(3, mm)), sub(0.2), pecsheet(), Layer()], [6.0, 9.0]),
        # several thin layers on both sides of one sheet, and a wide low-frequency band
        ([Layer(), sub(0.05, 4.0), sub(0.05), strip, sub(0.05), sub(0.05, 6.0), Layer()], [1.0, 30.0]),
        # layers between two sheets whose modes come from both neighbours
        ([Layer(), strip, Layer(width=Length(8, mm)), Layer(epsr=1.5, width=Length(8, mm)),
          Layer(width=Length(8, mm)), strip, Layer()], [12.0, 16.0]),
    ]


@pytest.mark.parametrize("k", range(12))
def test_selection_matches_the_planner(k):
    strata, freqs = _stacks()[k]
    plan = make_plan(strata, freqs, {"θ": 0.0, "ϕ": 0.0})
    junc, gbls, modes, dup = S.select(strata, freqs, _is_layer)
    assert junc[1:] == list(plan.junc)
    assert [tuple(g) for g in gbls] == [(g.first, g.last, g.j) for g in plan.gbls]
    for lay, L in enumerate(plan.layers, start=1):
        m = modes[lay]
        if m is None:
            assert len(L.P) == 0
            continue
        assert [(int(p), int(a), int(b)) for p, a, b in zip(L.P, L.M, L.N)] == m["modes"], lay
        assert np.array_equal(np.asarray(L.beta1, float), m["b1"]) and np.array_equal(np.asarray(L.beta2, float),
                                                                                       m["b2"]), lay
    assert list(plan.gbldup) == dup
    if k == 5:  # the repeated sheet: the middle Gblocks' GSMs are shared
        assert -1 in dup and any(d > 0 for d in dup)


def _parity_workloads():
    """The strata the GPU parity tests hand to ``oracle.analyze``: the strip gratings, the
    square patch, the two-sheet cascades (the Jerusalem cross also at its stated size), the
    ring patches and the meander of the gradient tests at its central-difference steps."""
    from pssfss_b200 import workloads
    from pssfss_b200.elements import jerusalemcross, polyring, rectstrip
    from pssfss_b200.gradient import meander_strata
    period = 299792458.0 * 100 / 2.54 * 1e-9
    out = []
    for cls in ("J", "M"):
        sh = rectstrip(Px=period / 20, Py=period, Lx=period / 20, Ly=period / 2, Nx=4, Ny=40, units=inch,
                       **{"class": cls})
        out.append(([Layer(), sh, Layer()], [0.8], {"θ": 0, "ϕ": 0}))
    out.append(([Layer(), rectstrip(Lx=8, Ly=8, Px=10, Py=10, Nx=16, Ny=16, units=mm), Layer()],
                list(np.linspace(10, 20, 11)), {"θ": 0, "ϕ": 0}))
    sub = Layer(epsr=3.0, tandel=0.002, width=Length(0.5, mm))
    jsheets = (rectstrip(Lx=6, Ly=0.5, Px=8, Py=8, Nx=12, Ny=2, units=mm),
               jerusalemcross(P=8, L1=6, L2=0.5, A=3, B=0.5, w=0.5, ntri=300, units=mm))
    for js in jsheets:
        ap = rectstrip(Lx=6, Ly=6, Px=8, Py=8, Nx=6, Ny=6, units=mm, **{"class": "M"})
        out.append(([Layer(), js, sub, Layer(width=Length(2, mm)), ap, Layer()], [5.0, 15.0, 25.0],
                    {"θ": 30, "ϕ": 45}))
    for period_mm, ro, ntri, theta in [(6.0, 0.40, 160, 0.0), (12.0, 0.44, 360, 45.0)]:
        r = ro * period_mm
        sh = polyring(s1=[period_mm, 0], s2=[0, period_mm], a=[r - 0.05 * period_mm], b=[r], sides=24, ntri=ntri,
                      units=mm)
        out.append(([Layer(), sh, Layer()], [10.0, 20.0], {"θ": theta, "ϕ": 0}))
    strata, flist, steer = workloads.jerusalem_aperture_cascade()
    out.append((strata, [float(flist[10]), float(flist[40])], steer))
    p0 = {"w": 0.3, "a": 5.0, "epsr": 2.2}
    for name in p0:
        for sgn in (1, -1):
            p = dict(p0, **{name: p0[name] * (1 + sgn * 1e-4)})
            out.append((meander_strata(p, ntri=400), [9.0, 13.0, 17.0], {"θ": 0.0, "ϕ": 0.0}))
    return out


def test_selection_matches_the_planner_on_parity_workloads():
    for strata, freqs, steer in _parity_workloads():
        plan = make_plan(strata, freqs, steer)
        junc, gbls, modes, dup = S.select(strata, freqs, _is_layer)
        assert junc[1:] == list(plan.junc)
        assert [tuple(g) for g in gbls] == [(g.first, g.last, g.j) for g in plan.gbls]
        for lay, L in enumerate(plan.layers, start=1):
            m = modes[lay]
            assert (len(L.P) == 0 if m is None else
                    [(int(p), int(a), int(b)) for p, a, b in zip(L.P, L.M, L.N)] == m["modes"])
        assert list(plan.gbldup) == dup


def test_rwg_topology_golden():
    """test/RWGData_test.jl: the 2 x 1 strip's basis functions and face-pair classes, through
    the oracle's own setup_rwg (oracle/rwg.py)."""
    from oracle import rwg as R
    from pssfss_b200.elements import rectstrip
    for fufp in (True, False):
        r = R.setup(rectstrip(Lx=1, Ly=1, Px=1, Py=1, Nx=2, Ny=1, units=mm, fufp=fufp))
        assert r.bfe.tolist() == [[8, 6, 9, 1, 2, 5], [8, 6, 9, 3, 4, 7]]
        assert r.bff.tolist() == [[1, 2, 3, 2, 4, 1], [2, 3, 4, 1, 3, 4]]
        assert r.ebf.tolist() == [4, 5, 4, 5, 6, 2, 6, 1, 3]
        assert r.eci.tolist() == [3, 3, 4, 4, 1, 0, 2, 0, 0]
        if fufp:
            assert r.ufpm.tolist() == [[1, 5, 9, 11], [2, 6, 10, 12], [3, 7, 1, 5], [4, 8, 2, 6]]
            assert r.ufp_rep.tolist() == [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 13, 14] and r.nufp == 12
        else:
            assert (r.ufpm.ravel(order="F") == np.arange(1, 17)).all() and r.nufp == 16


def test_rwg_topology_matches_the_package():
    """The oracle's setup_rwg against the package's on the sheets of the parity workloads and
    on the other structured meshes (diagonal strip, fine grating): identical basis functions,
    boundary codes and face-pair classes."""
    from oracle import rwg as R
    from pssfss_b200.elements import diagstrip, meander, rectstrip
    from pssfss_b200.rwg import setup_rwg
    from pssfss_b200.sheets import RWGSheet
    sheets = []
    for strata, _, _ in _parity_workloads():
        sheets += [s for s in strata if isinstance(s, RWGSheet) and s.style != "NULL"]
    sheets += [diagstrip(P=10, w=1, orient=45.0, Nl=20, Nw=4, units=mm),
               diagstrip(P=10, w=1, orient=-45.0, Nl=12, Nw=3, units=mm),
               meander(a=5, b=10, h=6, w1=0.3, w2=0.25, ntri=300, units=mm),
               rectstrip(Lx=8, Ly=8, Px=10, Py=10, Nx=6, Ny=6, units=mm, fufp=False)]
    seen = set()
    for sh in sheets:
        if id(sh) in seen:
            continue
        seen.add(id(sh))
        a, b = setup_rwg(sh), R.setup(sh)
        for f in ("bfe", "bff", "ebf", "eci", "ufpm", "ufp_rep"):
            assert np.array_equal(getattr(a, f), getattr(b, f)), (sh.style, f)
        assert a.nufp == b.nufp

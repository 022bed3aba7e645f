"""Host-side geometry, topology, modes and GSM algebra against the reference's tests.

test/RWGData_test.jl, test/RWGSheet_test.jl, test/Elements_test.jl, test/Rings_test.jl,
test/GSMs_test.jl (cascade identities, choose_gblocks), test/Modes_test.jl; the element
constructors the reference meshes with Triangle, checked by area, topology and physics.
"""
import math

import numpy as np
import pytest

import oracle
from conftest import golden
from pssfss_b200.elements import meander, meander_counts, rectstrip
from pssfss_b200.gsms import GSM, cascade, cascade_layer
from pssfss_b200.layers import Layer
from pssfss_b200.rings import Ring
from pssfss_b200.rwg import setup_rwg
from pssfss_b200.sheets import combine, recttri
from pssfss_b200.units import Length, inch, mm


def test_rings():
    assert list(Ring(0)) == [(0, 0)]
    assert list(Ring(1)) == [(1, -1), (1, 0), (1, 1), (-1, -1), (-1, 0), (-1, 1), (0, -1), (0, 1)]
    assert list(Ring(2)) == [(2, -2), (2, -1), (2, 0), (2, 1), (2, 2), (-2, -2), (-2, -1), (-2, 0),
                             (-2, 1), (-2, 2), (-1, -2), (0, -2), (1, -2), (-1, 2), (0, 2), (1, 2)]
    assert len(list(Ring(10))) == len(Ring(10)) == 80
    assert all(max(abs(m), abs(n)) == 100 for m, n in Ring(100))


def test_recttri_and_combine():
    sh1 = recttri([0., 0.], [1., 1.], 1, 1)
    assert sh1.rho.tolist() == [[0, 0], [1, 0], [0, 1], [1, 1]]
    assert sh1.e1.tolist() == [1, 3, 1, 2, 1] and sh1.e2.tolist() == [2, 4, 3, 4, 4]
    assert sh1.fe.ravel(order="F").tolist() == [2, 3, 5, 4, 5, 1]
    assert sh1.fv.ravel(order="F").tolist() == [1, 4, 3, 1, 2, 4]
    sh3 = combine(sh1, recttri([1., 0.], [2., 1.], 1, 1), "x", 1)
    assert sh3.rho.tolist() == [[0, 0], [1, 0], [0, 1], [1, 1], [2, 0], [2, 1]]
    assert sh3.e1.tolist() == [1, 3, 1, 2, 1, 2, 4, 5, 2]
    assert sh3.e2.tolist() == [2, 4, 3, 4, 4, 5, 6, 6, 6]
    assert sh3.fv.ravel(order="F").tolist() == [1, 4, 3, 1, 2, 4, 2, 6, 4, 2, 5, 6]
    assert sh3.fe.ravel(order="F").tolist() == [2, 3, 5, 4, 5, 1, 7, 4, 9, 8, 9, 6]
    sh3 = combine(sh1, recttri([0., 1.], [1., 2.], 1, 1), "y", 1.0)
    assert sh3.e1.tolist() == [1, 3, 1, 2, 1, 5, 3, 4, 3]
    assert sh3.fe.tolist() == [[2, 4, 6, 8], [3, 5, 7, 9], [5, 1, 9, 2]]
    assert sh3.fv.tolist() == [[1, 1, 3, 3], [4, 2, 6, 4], [3, 4, 5, 6]]
    sh3 = combine(sh1, recttri([1., 1.], [2., 2.], 1, 1), "y", 1.0)
    assert sh3.rho.tolist() == [[0, 0], [1, 0], [0, 1], [1, 1], [2, 1], [1, 2], [2, 2]]
    assert sh3.e1.tolist() == [1, 3, 1, 2, 1, 4, 6, 4, 5, 4]
    assert sh3.e2.tolist() == [2, 4, 3, 4, 4, 5, 7, 6, 7, 7]
    assert sh3.fe.tolist() == [[2, 4, 7, 9], [3, 5, 8, 10], [5, 1, 10, 6]]
    assert sh3.fv.tolist() == [[1, 1, 4, 4], [4, 2, 7, 5], [3, 4, 6, 7]]
    sh3 = combine(sh1, recttri([2., 0.], [3., 1.], 1, 1), " ", float("nan"))
    assert sh3.e1.tolist() == [1, 3, 1, 2, 1, 5, 7, 5, 6, 5]
    assert sh3.fv.tolist() == [[1, 1, 5, 5], [4, 2, 8, 6], [3, 4, 7, 8]]


def test_rectstrip_fields():
    sh = rectstrip(Lx=1, Ly=1.0, Nx=1, Ny=1, Px=1, Py=1, units=inch)
    assert (sh.rho[1] - sh.rho[0]).tolist() == [1, 0]
    assert sh.fufp and sh.cls == "J" and sh.units == inch
    assert np.allclose(sh.beta1, [2 * math.pi, 0]) and np.allclose(sh.beta2, [0, 2 * math.pi])


def test_rwgdata_fufp_true_false():
    for fufp in (True, False):
        r = setup_rwg(rectstrip(Lx=1, Ly=1, Px=1, Py=1, Nx=2, Ny=1, units=mm, fufp=fufp))
        assert r.bfe.tolist() == [[8, 6, 9, 1, 2, 5], [8, 6, 9, 3, 4, 7]]
        assert r.bff.tolist() == [[1, 2, 3, 2, 4, 1], [2, 3, 4, 1, 3, 4]]
        assert r.ebf.tolist() == [4, 5, 4, 5, 6, 2, 6, 1, 3]
        assert r.eci.tolist() == [3, 3, 4, 4, 1, 0, 2, 0, 0]
        if fufp:
            assert r.ufpm.tolist() == [[1, 5, 9, 11], [2, 6, 10, 12], [3, 7, 1, 5], [4, 8, 2, 6]]
            assert [list(x) for x in r.ufp2fp] == [[1, 11], [2, 12], [3], [4], [5, 15], [6, 16],
                                                    [7], [8], [9], [10], [13], [14]]
            assert r.nufp == 12
        else:
            assert (r.ufpm.ravel(order="F") == np.arange(1, 17)).all() and r.nufp == 16


def test_rwgbfft_golden():
    # test/RWGData_test.jl:46-48 and 56-58
    sh = rectstrip(Lx=1, Ly=1, Px=1, Py=1, Nx=2, Ny=1, units=mm, fufp=False)
    ft = oracle.rwgbfft(setup_rwg(sh), sh, [0., 0.], 0.0, 0.0)
    vals, _ = golden("rwgbfft_mm")
    assert np.allclose(ft[:3], np.reshape(vals, (3, 2)), rtol=1e-12, atol=0)
    sh = rectstrip(Lx=1, Ly=1, Px=1, Py=1, Nx=2, Ny=1, units=inch, fufp=False)
    ft = oracle.rwgbfft(setup_rwg(sh), sh, [20.0, -30.3], 0.8, -0.7)
    vals, _ = golden("rwgbfft_inch")
    assert np.allclose(ft[:3], np.reshape(vals, (3, 2)), rtol=1e-12, atol=0)


def test_meander_counts_and_topology():
    nx1, nx2, ny1, ny2, nt = meander_counts(5, 10, 6, 0.3, 0.3, 3000)
    sh = meander(a=5, b=10, h=6, w1=0.3, w2=0.3, ntri=3000, units=mm)
    assert sh.nface == nt == 2840
    r = setup_rwg(sh)
    assert r.nbf == 3976
    # every edge used by <= 2 faces, every face's edges distinct
    assert all(len(set(sh.fe[:, f])) == 3 for f in range(sh.nface))


def test_cascade_identities():
    # test/GSMs_test.jl:17-95
    c = cascade(GSM.identity(10, 20), GSM.identity(20, 15))
    assert np.linalg.norm(c.s11) == np.linalg.norm(c.s22) == 0
    off = ~np.eye(*c.s12.shape, dtype=bool)
    assert (np.diag(c.s12) == 1).all() and (c.s12[off] == 0).all()
    assert (np.diag(c.s21) == 1).all() and (c.s21[~np.eye(*c.s21.shape, dtype=bool)] == 0).all()
    al, be = 0.35, math.sqrt(1 - 0.35 ** 2)
    ga, de = 0.23, math.sqrt(1 - 0.23 ** 2)
    a = GSM.identity(1, 1)
    b = GSM.identity(1, 1)
    b.s11[:] = b.s22[:] = ga
    b.s12[:] = b.s21[:] = de
    c = cascade(a, b)
    D = 1 / (1 - a.s22[0, 0] * b.s11[0, 0])
    assert abs(c.s11[0, 0] - (a.s11 + a.s12 * a.s21 * b.s11 / D)[0, 0]) <= 1e-16
    assert abs(c.s12[0, 0] - (a.s12 * b.s12 / D)[0, 0]) <= 1e-16
    a = GSM.identity(1, 1)
    a.s11[:] = a.s22[:] = al
    a.s12[:] = a.s21[:] = be
    layer = Layer(width=Length(25, mm))
    layer.gamma = np.array([1.0j])
    prop = np.exp(-1.0j * 0.025)
    b = a.copy()
    cascade_layer(a, layer, 25)
    cascade_layer(b, layer)
    for x, y in ((a.s12, be * prop), (a.s22, al * prop ** 2), (b.s21, be * prop)):
        assert abs(x[0, 0] - y) <= 1e-16


def test_structured_ring_and_cross_meshes():
    """Own meshes for the shapes the reference meshes with Triangle: counter-clockwise
    faces, every interior edge shared by exactly two faces, total area equal to the shape's."""
    from pssfss_b200.elements import jerusalemcross, polyring
    from pssfss_b200.units import mm as MM
    import math as _m
    ring = polyring(s1=[10, 0], s2=[0, 10], a=[2.0], b=[3.0], sides=24, ntri=400, units=MM)
    patch = polyring(s1=[10, 0], s2=[0, 10], a=[0], b=[4.0], sides=4, ntri=300, units=MM, orient=45)
    cross = jerusalemcross(P=8, L1=6, L2=0.5, A=3, B=0.5, w=0.5, ntri=600, units=MM)
    af = 0.5 * 24 * _m.sin(2 * _m.pi / 24)
    for sh, area in ((ring, (9 - 4) * af), (patch, 16 * 0.5 * 4 * _m.sin(_m.pi / 2)),
                     (cross, 2 * 6 * 0.5 - 0.25 + 4 * (3 * 0.5 - 0.5 * 0.5))):
        rho = sh.rho
        fv = sh.fv - 1
        a = 0.5 * ((rho[fv[1], 0] - rho[fv[0], 0]) * (rho[fv[2], 1] - rho[fv[0], 1]) -
                   (rho[fv[2], 0] - rho[fv[0], 0]) * (rho[fv[1], 1] - rho[fv[0], 1]))
        assert (a > 0).all()
        assert abs(a.sum() - area) < 1e-9 * area
        counts = np.bincount(sh.fe.ravel(), minlength=sh.nedge + 1)[1:]
        assert counts.min() >= 1 and counts.max() <= 2
        rwg = setup_rwg(sh)
        assert rwg.nbf == int((counts == 2).sum())


def _split_strata(strata):
    """Layers, sheets and junc (sheet number at each interface, 0 = none) as in
    PSSFSS.jl:205-213."""
    from pssfss_b200.sheets import RWGSheet
    layers = [s for s in strata if isinstance(s, Layer)]
    sheets = [s for s in strata if isinstance(s, RWGSheet)]
    junc = [0] * (len(layers) - 1)
    nlay = ns = 0
    for s in strata:
        if isinstance(s, Layer):
            nlay += 1
        else:
            ns += 1
            junc[nlay - 1] = ns
    return layers, sheets, junc


def _ring(p):
    from pssfss_b200.elements import polyring
    return polyring(sides=4, orient=45, a=[0.1902], b=[0.2169], units=inch, s1=[p, 0], s2=[0, p], ntri=100)


def _duroid():
    from pssfss_b200.units import mil
    return Layer(name="Duroid 6035", epsr=3.6, tandel=0.0013, width=Length(20, mil))


def test_choose_layer_modes_counts():
    # test/Modes_test.jl: modes kept per layer by choose_layer_modes! for two ring screens on
    # Duroid with vacuum gaps, 2-8 GHz, dbmin = 25 (the count depends on the lattices and the
    # layers, not on the ring's triangulation).
    from pssfss_b200.constants import C0, TWOPI
    from pssfss_b200.gsms import choose_gblocks
    from pssfss_b200.modes import choose_layer_modes

    vac = lambda w=None: Layer(name="Vacuum") if w is None else Layer(name="Vacuum", width=Length(w, inch))
    cases = [
        [vac(), _duroid(), _ring(0.5117), _duroid(), vac(0.2), _duroid(), _ring(0.5117), _duroid(), vac()],
        [vac(), _duroid(), _ring(0.5117), _duroid(), vac(0.1), vac(0.1), _duroid(), _ring(0.9005), _duroid(), vac()],
        [vac(), _duroid(), _ring(0.5117), _duroid(), vac(0.1), vac(0.1), _duroid(), _ring(0.5117), _duroid(), vac()],
    ]
    want = [c["counts"] for c in golden("layer_mode_counts")[1]["cases"]]
    for strata, expect in zip(cases, want):
        layers, sheets, junc = _split_strata(strata)
        k0min, k0max = TWOPI * 2e9 / C0, TWOPI * 8e9 / C0
        gbl = choose_gblocks(layers, sheets, junc, k0min)
        choose_layer_modes(layers, sheets, junc, gbl, k0max, 25.0)
        assert [len(l.P) for l in layers] == expect


def test_choose_gblocks():
    # test/GSMs_test.jl choose_gblocks1..4: Gblock(first:last, j) for sheets on thin layers
    # and separated by gaps (a gap whose evanescent modes decay enough splits the Gblocks).
    from pssfss_b200.constants import C0, TWOPI
    from pssfss_b200.gsms import choose_gblocks
    from pssfss_b200.units import cm, mil

    def strip():
        return rectstrip(units=cm, Px=1, Py=1, Lx=0.5, Ly=0.5, Nx=10, Ny=10)

    vac = lambda w=None, u=inch: Layer(name="Vacuum") if w is None else Layer(name="Vacuum", width=Length(w, u))
    cases = [
        ([Layer(), strip(), Layer(width=Length(1, mil), epsr=2.2), Layer(width=Length(1, mil)),
          Layer(width=Length(3, mm)), strip(), Layer(width=Length(1, mil), epsr=2.2), Layer()], 10e9),
        ([vac(), _duroid(), _ring(0.5117), _duroid(), vac(0.05), _duroid(), _ring(0.5117), _duroid(), vac()], 2e9),
        ([vac(), _duroid(), _ring(0.5117), _duroid(), _duroid(), _ring(0.5117), _duroid(), vac()], 2e9),
        ([vac(), _duroid(), _ring(0.5117), _duroid(), vac(5, mil), _duroid(), _ring(0.5117), _duroid(),
          vac(5, mil), _duroid(), _ring(0.5117), _duroid(), vac()], 2e9),
    ]
    want = [c["gblocks"] for c in golden("gblocks")[1]["cases"]]
    for (strata, f), expect in zip(cases, want):
        layers, sheets, junc = _split_strata(strata)
        gbl = choose_gblocks(layers, sheets, junc, TWOPI * f / C0)
        assert [[g.first, g.last, g.j] for g in gbl] == expect


def test_diagstrip_mesh_and_mirror_symmetry():
    # diagstrip (Elements.jl:218-294): the strip along the cell diagonal tapers into the two
    # corners it runs to; the other two corners carry the matching pieces, so the sheet has
    # three pieces joined only through the periodic boundary.  Its area is √2·P·w, and the
    # -45° strip is the mirror image of the +45° one: the co-polarised transmissions swap
    # and the cross-polarised ones swap with a change of sign.
    from pssfss_b200.elements import _tritri, diagstrip
    from pssfss_b200.outputs import getsijmn

    def area(sh):
        r, f = sh.rho, sh.fv - 1
        return sum(abs((r[b][0] - r[a][0]) * (r[c][1] - r[a][1]) - (r[c][0] - r[a][0]) * (r[b][1] - r[a][1])) / 2
                   for a, b, c in f.T)

    for nw in range(1, 7):
        t = _tritri(2.0, nw)
        assert math.isclose(area(t), 1.0, rel_tol=1e-12) and t.nnode - t.nedge + t.nface == 1
    res = {}
    for o in (45, -45):
        d = diagstrip(P=10, w=1, orient=o, Nl=16, Nw=2, units=mm)
        assert math.isclose(area(d), math.sqrt(2) * 10, rel_tol=1e-12)
        assert d.nnode - d.nedge + d.nface == 3
        r = setup_rwg(d)
        assert np.bincount(r.eci, minlength=5)[1:].tolist() == [2, 2, 2, 2]  # one edge per corner leg
        res[o] = oracle.analyze([Layer(), d, Layer()], [12.0], {"θ": 0.0, "ϕ": 0.0})[0]
    s = lambda o, m, n: getsijmn(2, 1, m, n, res[o])
    # (to the modal tables' 1e-7 convergence; TE and TM of one orientation differ by ~3e-4)
    assert abs(s(45, 1, 1) - s(-45, 2, 2)) < 1e-7 and abs(s(45, 2, 2) - s(-45, 1, 1)) < 1e-7
    assert abs(s(45, 1, 2) + s(-45, 2, 1)) < 1e-7 and abs(s(45, 2, 1) + s(-45, 1, 2)) < 1e-7
    assert abs(s(45, 1, 2)) > 0.1


def test_loadedcross_mesh_and_lossless_balance():
    # loadedcross (Elements.jl:794-961): a cross loop of trace width w (an annulus, Euler
    # characteristic 0) or, for 2w >= L2, a solid cross (1), with the exact area.  Through the
    # oracle at normal incidence, below the first grating lobe and with no sheet resistance,
    # the power of each incident polarisation is conserved, and the four-fold symmetric
    # element transmits TE and TM alike with almost no cross-polarisation (the grid mesh
    # is symmetric only up to its diagonals).
    from pssfss_b200.elements import loadedcross
    from pssfss_b200.outputs import getsijmn

    def area(sh):
        r, f = sh.rho, sh.fv - 1
        return sum(abs((r[b][0] - r[a][0]) * (r[c][1] - r[a][1]) - (r[c][0] - r[a][0]) * (r[b][1] - r[a][1])) / 2
                   for a, b, c in f.T)

    for w, orient, euler in ((0.5, 0.0, 0), (0.5, 30.0, 0), (3.0, 0.0, 1)):
        sh = loadedcross(s1=[10, 0], s2=[0, 10], L1=8, L2=3, w=w, ntri=200, units=mm, orient=orient)
        a2 = 3 - 2 * w
        want = 2 * 8 * 3 - 9 - ((2 * (8 - 2 * w) * a2 - a2 * a2) if a2 > 0 else 0)
        assert math.isclose(area(sh), want, rel_tol=1e-12)
        assert sh.nnode - sh.nedge + sh.nface == euler
        r = oracle.analyze([Layer(), sh, Layer()], [12.0], {"θ": 0.0, "ϕ": 0.0})[0]
        S = lambda i, j, m, n: getsijmn(i, j, m, n, r)
        for n in (1, 2):
            assert abs(sum(abs(S(i, 1, m, n)) ** 2 for i in (1, 2) for m in (1, 2)) - 1) < 1e-5
        assert abs(S(2, 1, 1, 1) - S(2, 1, 2, 2)) < 2e-3 and abs(S(2, 1, 1, 2)) < 5e-3


def test_hollow_jerusalemcross_outlines():
    # jerusalemcross (Elements.jl:963): parts no wider than 2w are solid.  Hollow arms and
    # caps give one connected opening (Euler characteristic 0), hollow arms with solid caps
    # a cross-shaped slot (0), hollow caps on solid arms four openings (-3), all solid 1;
    # the meshed area is exact, and through the oracle a hollow cross keeps the power of
    # each polarisation and its TE/TM degeneracy at normal incidence.
    from pssfss_b200.elements import jerusalemcross
    from pssfss_b200.outputs import getsijmn

    def area(sh):
        r, f = sh.rho, sh.fv - 1
        return sum(abs((r[b][0] - r[a][0]) * (r[c][1] - r[a][1]) - (r[c][0] - r[a][0]) * (r[b][1] - r[a][1])) / 2
                   for a, b, c in f.T)

    L1, L2, A, B = 6.0, 1.0, 3.0, 0.8
    h1, h2, hA = L1 / 2, L2 / 2, A / 2
    solid = 2 * L1 * L2 - L2 * L2 + 4 * (A * B - L2 * B)
    for w, euler in ((0.1, 0), (0.3, 0), (0.45, 0), (0.6, 1)):
        sh = jerusalemcross(P=8, L1=L1, L2=L2, A=A, B=B, w=w, ntri=600, units=mm)
        g = 2 * (h2 - w)
        if 2 * w < B:      # slots through the arms into the caps' openings
            hole = 2 * (2 * (h1 - w) * g) - g * g + 4 * (B - 2 * w) * (2 * (hA - w) - g)
        elif 2 * w < L2:   # slot stopping a trace width short of the solid caps
            hole = 2 * (2 * (h1 - B - w) * g) - g * g
        else:
            hole = 0.0
        assert math.isclose(area(sh), solid - hole, rel_tol=1e-12)
        assert sh.nnode - sh.nedge + sh.nface == euler
    caps = jerusalemcross(P=8, L1=6, L2=0.5, A=3, B=1.2, w=0.3, ntri=300, units=mm)
    assert caps.nnode - caps.nedge + caps.nface == -3
    sh = jerusalemcross(P=8, L1=L1, L2=L2, A=A, B=B, w=0.1, ntri=300, units=mm)
    r = oracle.analyze([Layer(), sh, Layer()], [14.0], {"θ": 0.0, "ϕ": 0.0})[0]
    S = lambda i, j, m, n: getsijmn(i, j, m, n, r)
    for n in (1, 2):
        assert abs(sum(abs(S(i, 1, m, n)) ** 2 for i in (1, 2) for m in (1, 2)) - 1) < 1e-5
    assert abs(S(2, 1, 1, 1) - S(2, 1, 2, 2)) < 1e-6 and abs(S(2, 1, 1, 2)) < 1e-3


def test_cell_filling_polyring():
    # polyring with b[end] < 0 (Elements.jl:392-403, 440-482): the last ring fills the cell
    # out to its boundary with -b[end] edges along the shorter lattice vector, so the sheet
    # is a periodic screen with polygonal openings.  Exact area; matching edge counts on
    # opposite cell edges (periodic basis functions); through the oracle a square opening
    # in a square cell keeps the power of each polarisation and its TE/TM degeneracy.
    from pssfss_b200.elements import polyring
    from pssfss_b200.outputs import getsijmn

    def area(sh):
        r, f = sh.rho, sh.fv - 1
        return sum(abs((r[b][0] - r[a][0]) * (r[c][1] - r[a][1]) - (r[c][0] - r[a][0]) * (r[b][1] - r[a][1])) / 2
                   for a, b, c in f.T)

    cases = [(dict(s1=[10, 0], s2=[0, 10], a=[3.0], b=[-10], sides=4, orient=45, ntri=300), [10, 10, 10, 10]),
             (dict(s1=[10, 0], s2=[0, 10], a=[2.0, 3.5], b=[3.0, -12], sides=32, ntri=800), [12, 12, 12, 12]),
             (dict(s1=[1.1414, 0.0], s2=[0.5707, 0.9885], a=[0.3], b=[-8], sides=6, ntri=500), [8, 8, 8, 8]),
             (dict(s1=[10, 0], s2=[0, 14], a=[4.0], b=[-6], sides=24, ntri=300), [8, 8, 6, 6])]
    for kw, eci in cases:
        sh = polyring(units=mm, **kw)
        s1, s2 = np.array(kw["s1"], float), np.array(kw["s2"], float)
        af = 0.5 * kw["sides"] * math.sin(2 * math.pi / kw["sides"])
        want = (abs(s1[0] * s2[1] - s1[1] * s2[0]) - af * kw["a"][-1] ** 2 +
                sum((bb * bb - aa * aa) * af for aa, bb in zip(kw["a"][:-1], kw["b"][:-1])))
        assert math.isclose(area(sh), want, rel_tol=1e-12)
        assert sh.xi_eta_check and np.bincount(setup_rwg(sh).eci, minlength=5)[1:].tolist() == eci
    sh = polyring(units=mm, **cases[0][0])
    r = oracle.analyze([Layer(), sh, Layer()], [12.0], {"θ": 0.0, "ϕ": 0.0})[0]
    S = lambda i, j, m, n: getsijmn(i, j, m, n, r)
    for n in (1, 2):
        assert abs(sum(abs(S(i, 1, m, n)) ** 2 for i in (1, 2) for m in (1, 2)) - 1) < 1e-6
    assert abs(S(2, 1, 1, 1) - S(2, 1, 2, 2)) < 1e-3 and abs(S(2, 1, 1, 2)) < 1e-3
    assert 0.05 < abs(S(2, 1, 1, 1)) < 0.5   # an opening well below its cutoff passes little


def test_edge_current_unit_vector():
    # RWG.jl:339-363: a unit normal to the edge, pointing out of the plus face of its basis
    # function (from that face's free vertex across the edge)
    from pssfss_b200.rwg import edge_current_unit_vector
    sh = meander(a=5, b=10, h=6, w1=0.3, w2=0.3, ntri=200, units=mm)
    r = setup_rwg(sh)
    for ie in range(1, sh.nedge + 1):
        bf = int(r.ebf[ie - 1])
        if bf == 0:
            with pytest.raises(ValueError):
                edge_current_unit_vector(ie, r, sh)
            continue
        u = edge_current_unit_vector(ie, r, sh)
        n1, n2 = int(sh.e1[ie - 1]), int(sh.e2[ie - 1])
        f = int(r.bff[0, bf - 1])
        nfree = [int(v) for v in sh.fv[:, f - 1] if v not in (n1, n2)][0]
        assert abs(np.linalg.norm(u) - 1) < 1e-14 and abs(u @ (sh.rho[n2 - 1] - sh.rho[n1 - 1])) < 1e-12
        assert u @ (sh.rho[n1 - 1] - sh.rho[nfree - 1]) > 0


def test_gsm_file_round_trip(tmp_path):
    # test/GSMs_test.jl "GSM file": header (cells, units, mode lists) and one case group
    from pssfss_b200.gsms import append_gsm_data, initialize_gsm_file, read_gsm_file
    from pssfss_b200.layers import TE, TM
    alpha = 0.35
    beta = math.sqrt(1 - alpha ** 2)
    a = GSM.identity(1, 1)
    a.s11[:] = a.s22[:] = alpha
    a.s12[:] = a.s21[:] = beta
    l1 = Layer(epsr=2.0)
    l1.P, l1.M, l1.N = [TE, TM], [0, 0], [0, 0]
    l2 = Layer(epsr=2.0)
    l2.P, l2.M, l2.N = [TE, TM], [0, 0], [0, 0]
    l2.epsr = 1.0
    sh = rectstrip(Lx=1, Ly=1, Px=1, Py=1, Nx=2, Ny=1, units=mm, fufp=True)
    fname = str(tmp_path / "gsmfile.gsm")
    initialize_gsm_file(fname, l1, l2, sh, sh)
    case = {"θ": 0.0, "ϕ": 0.0, "FGHz": 2.0}
    append_gsm_data(fname, "1", a, l1, l2, case)
    dat = read_gsm_file(fname)
    assert dat["ModelistIn"] == ([TE, TM], [0, 0], [0, 0]) and dat["ModelistOut"] == ([TE, TM], [0, 0], [0, 0])
    assert dat["s1in"].tolist() == [1.0, 0.0] and dat["s2out"].tolist() == [0.0, 1.0]
    for k in ("s11", "s12", "s21", "s22"):
        assert np.array_equal(getattr(dat["1/gsm"], k), getattr(a, k))
    assert dat["1/epsmu1"] == (2.0 + 0j, 1.0 + 0j) and dat["1/epsmu2"] == (1.0 + 0j, 1.0 + 0j)
    assert dat["1/case"] == case and dat["unitsin"] == mm and dat["unitsout"] == mm
    import pickle
    other = tmp_path / "other.gsm"
    other.write_bytes(pickle.dumps({"FileType": "ResultFile"}))
    with pytest.raises(ValueError, match="not a GSM file"):
        read_gsm_file(str(other))


def test_sheet_file_round_trip(tmp_path):
    # test/RWGSheet_test.jl "read and write": a combined sheet written and read back
    from pssfss_b200.sheets import read_sheet_data, write_sheet_data
    sh = combine(recttri([0., 0.], [1., 1.], 2, 2), recttri([1., 0.], [2., 1.], 2, 2), "x", 1.0)
    fname = str(tmp_path / "sheet.dat")
    write_sheet_data(fname, sh)
    back = read_sheet_data(fname)
    for k in ("rho", "e1", "e2", "fv", "fe"):
        assert np.array_equal(getattr(back, k), getattr(sh, k))
    assert back.units == sh.units and back.style == sh.style


def test_benchmark_workloads_plan():
    # the workloads build and plan on the host with the sizes they are quoted at
    from pssfss_b200 import workloads
    from pssfss_b200.analyze import make_plan
    strata, f, st = workloads.square_patch_sweep()
    plan = make_plan(strata, f, st)
    assert plan.rwgdat[0].nbf == 736 and len(plan.points) == 11
    strata, f, st = workloads.meander_precision_sweep()
    assert setup_rwg(strata[1]).nbf == 3976 and len(f) == 101
    strata, f, st = workloads.jerusalem_aperture_cascade(ntri_cross=300, ntri_aperture=200)
    plan = make_plan(strata, f, st)
    assert len(plan.sheets) == 2 and len(plan.points) == 51 and plan.sheets[1].cls == "M"
    batch = workloads.ring_batch()
    assert len(batch) == 64
    sizes = [b[0][1].nface for b in batch]
    assert min(sizes) >= 250 and max(sizes) <= 3600 and len({b[2]["θ"] for b in batch}) == 4
    params, f, ntri = workloads.meander_gradient_workload()
    sh = workloads.meander_strata(ntri=ntri, **params)[1]
    assert sh.nface == 3960 and len(f) == 201


def test_unique_face_pair_paths_agree():
    # the packed one-key classing and the three-key sort give the same classes, numbered by
    # first member in column-major order (RWG.jl:287-319)
    from pssfss_b200 import rwg
    from pssfss_b200.elements import diagstrip
    for sh in (meander(a=5, b=10, h=6, w1=0.3, w2=0.3, ntri=300, units=mm),
               rectstrip(Lx=8, Ly=8, Px=10, Py=10, Nx=16, Ny=16, units=mm, fufp=True),
               diagstrip(P=10, w=1, orient=45, Nl=12, Nw=3, units=mm)):
        a = rwg.unique_face_pairs(sh)
        sid, dx, dy = rwg._ufp_keys(sh)
        b = rwg._unique_face_pairs_sorted(sh.nface, sid, dx, dy)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
        assert a[0][tuple(np.unravel_index(a[1] - 1, a[0].shape, order="F"))].tolist() == list(range(1, a[2] + 1))


def test_meshers_on_seeded_random_shapes():
    # the structured meshers over seeded random valid parameters: counter-clockwise,
    # non-degenerate triangles (checked when the sheet is built), exact areas, periodic
    # edges that pair up (setup_rwg)
    from pssfss_b200.elements import jerusalemcross, loadedcross, polyring

    def area(sh):
        r, f = sh.rho, sh.fv - 1
        return sum(abs((r[b][0] - r[a][0]) * (r[c][1] - r[a][1]) - (r[c][0] - r[a][0]) * (r[b][1] - r[a][1])) / 2
                   for a, b, c in f.T)

    rng = np.random.default_rng(7)
    for _ in range(20):
        p1, p2, skew = rng.uniform(5, 15), rng.uniform(5, 15), rng.uniform(-0.5, 0.5)
        s1, s2 = [p1, 0.0], [skew * p2, p2 * rng.uniform(0.7, 1.0)]
        cell = abs(s1[0] * s2[1] - s1[1] * s2[0])
        inr = 0.5 * min(cell / np.linalg.norm(s1), cell / np.linalg.norm(s2))
        sides, a = int(rng.integers(3, 40)), rng.uniform(0.1, 0.8) * inr
        sh = polyring(s1=s1, s2=s2, a=[a], b=[-int(rng.integers(2, 20))], sides=sides, orient=float(rng.uniform(0, 90)),
                      ntri=int(rng.integers(100, 1000)), units=mm)
        af = 0.5 * sides * math.sin(2 * math.pi / sides)
        assert math.isclose(area(sh), cell - af * a * a, rel_tol=1e-9)
        setup_rwg(sh)
        P = rng.uniform(6, 12)
        L1 = rng.uniform(0.4, 0.9) * P
        L2 = rng.uniform(0.1, 0.5) * L1
        w = rng.uniform(0.02, 0.6) * L2
        lc = loadedcross(s1=[P, 0], s2=[0, P], L1=L1, L2=L2, w=w, ntri=int(rng.integers(100, 600)), units=mm,
                         orient=float(rng.uniform(0, 90)))
        a2 = L2 - 2 * w
        assert math.isclose(area(lc), 2 * L1 * L2 - L2 * L2 - ((2 * (L1 - 2 * w) * a2 - a2 * a2) if a2 > 0 else 0),
                            rel_tol=1e-9)
        A, B = rng.uniform(1.05, 1.6) * L2, rng.uniform(0.1, 0.8) * (L1 - L2) / 2
        if A < P:
            setup_rwg(jerusalemcross(P=P, L1=L1, L2=L2, A=A, B=B, w=w, ntri=int(rng.integers(100, 600)), units=mm))


def _combine_loops(sh1, sh2, dup_coor, val):
    """Sheets.jl:234-389 written as its loops (first-match searches, sequential replacement and
    descending renumbering), the check on the array form of ``combine``.  Returns
    (rho, e1, e2, fv, fe)."""
    nv1, ne1, nf1 = sh1.nnode, sh1.nedge, sh1.nface
    vcen1, vcen2, ecen1, ecen2 = [], [], [], []
    if dup_coor != " ":
        d = sh1.rho[sh1.e1[0] - 1] - sh1.rho[sh1.e2[0] - 1]
        tol = 0.5e-4 * math.sqrt(d[0] * d[0] + d[1] * d[1])
        ax = 0 if dup_coor == "x" else 1
        for i in range(sh2.nnode):
            if abs(sh2.rho[i, ax] - val) < tol:
                for n1 in range(nv1):
                    dd = sh1.rho[n1] - sh2.rho[i]
                    if math.sqrt(dd[0] * dd[0] + dd[1] * dd[1]) < tol:
                        vcen2.append(i + 1)
                        vcen1.append(n1 + 1)
                        break
        for i in range(sh2.nedge):
            a, b = int(sh2.e1[i]), int(sh2.e2[i])
            if a in vcen2 and b in vcen2:
                va, vb = vcen1[vcen2.index(a)], vcen1[vcen2.index(b)]
                found = [j + 1 for j in range(ne1) if {int(sh1.e1[j]), int(sh1.e2[j])} == {va, vb}]
                if not found:
                    raise RuntimeError("no matching edge")
                ecen2.append(i + 1)
                ecen1.append(found[0])
    rho = np.vstack([sh1.rho, sh2.rho[[i for i in range(sh2.nnode) if i + 1 not in vcen2]]])
    e1, e2 = list(sh1.e1), list(sh1.e2)
    for i in range(sh2.nedge):
        if i + 1 in ecen2:
            continue
        for dst, src in ((e1, sh2.e1), (e2, sh2.e2)):
            v = int(src[i])
            dst.append(vcen1[vcen2.index(v)] if v in vcen2 else v + nv1)
    e1, e2 = np.array(e1, np.int64), np.array(e2, np.int64)
    fv = np.hstack([sh1.fv, sh2.fv + nv1]).astype(np.int64)
    fe = np.hstack([sh1.fe, sh2.fe + ne1]).astype(np.int64)
    for k in range(len(vcen2)):
        fv[fv == vcen2[k] + nv1] = vcen1[k]
    for k in range(len(ecen2)):
        fe[fe == ecen2[k] + ne1] = ecen1[k]
    for k in range(len(vcen2) - 1, -1, -1):
        for x in (e1, e2, fv):
            x[x > nv1 + vcen2[k]] -= 1
    for k in range(len(ecen2) - 1, -1, -1):
        fe[fe > ne1 + ecen2[k]] -= 1
    return rho, e1, e2, fv, fe


@pytest.mark.parametrize("seed", range(4))
def test_combine_matches_loop_form(seed):
    """Seeded strips merged along x, along y and without a shared line, then merged again with a
    third strip, as the element builders chain them: identical nodes, edges and faces; a shared
    line whose nodes do not match an edge of the first sheet raises in both forms."""
    rng = np.random.default_rng(seed)
    for _ in range(40):
        mode = ["x", "y", " "][int(rng.integers(3))]
        n1, n2, m = (int(v) for v in rng.integers(1, 7, 3))
        m2 = m if rng.random() < 0.8 else int(rng.integers(1, 7))
        h = float(rng.choice([1.0, 1.5]))
        if mode == "x":
            boxes = [([0., 0.], [1., h], n1, m), ([1., 0.], [2.5, h], n2, m2), ([2.5, 0.], [3., h], n1, m2)]
            vals = [1.0, 2.5]
        elif mode == "y":
            boxes = [([0., 0.], [h, 1.], m, n1), ([0., 1.], [h, 2.5], m2, n2), ([0., 2.5], [h, 3.], m2, n1)]
            vals = [1.0, 2.5]
        else:
            boxes = [([0., 0.], [1., 1.], n1, m), ([2., 0.], [3., 1.], n2, m2)]
            vals = [0.0]
        sh = recttri(*boxes[0])
        for box, val in zip(boxes[1:], vals):
            other = recttri(*box)
            try:
                want = _combine_loops(sh, other, mode, val)
            except RuntimeError:
                with pytest.raises(RuntimeError):
                    combine(sh, other, mode, val)
                break
            sh = combine(sh, other, mode, val)
            got = (sh.rho, sh.e1, sh.e2, sh.fv, sh.fe)
            for g, w in zip(got, want):
                assert g.shape == w.shape and np.array_equal(g, w)


def test_layer_copy_is_independent():
    """A point's layer copy takes its own mode lists and modal arrays: filling or editing them
    leaves the planned layer untouched."""
    lay = Layer(width=Length(1, mm), epsr=2.2, tandel=0.001)
    lay.P, lay.M, lay.N = [1, 2], [0, 0], [0, 0]
    lay.beta1 = np.array([1.0, 0.0])
    c = lay.copy()
    assert c.same_as(lay) and type(c) is Layer
    c.P.append(1)
    c.beta1[0] = 5.0
    c.gamma = np.ones(2, complex)
    assert lay.P == [1, 2] and lay.beta1[0] == 1.0 and len(lay.gamma) == 0

"""The quality mesher (pssfss_b200.meshsub) that stands in for Triangle behind ``meshsub``
(``src/Meshsub.jl:43-113``; switches ``pDa<area>q30Qe``).

Checked on the boundary graphs of the reference's unstructured elements (``polyring``,
``loadedcross``, ``jerusalemcross``, ``Elements.jl:368-558, 794-1100``):
  * exact predicates: collinear and co-circular inputs give 0, not a rounding-noise sign;
  * Delaunay: no node strictly inside any triangle's circumcircle (exact test);
  * quality: every angle >= 30 degrees, no triangle above the final area bound;
  * the graph is kept: the mesh's boundary edges lie on the input segments and add up to
    their length, the meshed area equals the region's, holes stay empty;
  * the triangle count lands within 10 % of ``ntri``, as the reference's area iteration;
  * a cell-filling ring gets no node added on the cell boundary, so opposite cell edges
    keep matching nodes (the periodic basis functions need them).
"""
import math

import numpy as np
import pytest

from pssfss_b200.elements import jerusalemcross, loadedcross, polyring
from pssfss_b200.meshsub import incircle, orient, triangulate
from pssfss_b200.units import mm


def _angles(r, f):
    out = []
    for k in range(3):
        p, q, s = r[f[k]], r[f[(k + 1) % 3]], r[f[(k + 2) % 3]]
        u, v = q - p, s - p
        c = (u * v).sum(1) / np.linalg.norm(u, axis=1) / np.linalg.norm(v, axis=1)
        out.append(np.degrees(np.arccos(np.clip(c, -1, 1))))
    return np.min(out, axis=0)


def _areas(r, f):
    return 0.5 * ((r[f[1], 0] - r[f[0], 0]) * (r[f[2], 1] - r[f[0], 1]) -
                  (r[f[2], 0] - r[f[0], 0]) * (r[f[1], 1] - r[f[0], 1]))


def _boundary_edges(f):
    cnt = {}
    for a, b, c in f.T:
        for p, q in ((a, b), (b, c), (c, a)):
            k = (min(p, q), max(p, q))
            cnt[k] = cnt.get(k, 0) + 1
    assert set(cnt.values()) <= {1, 2}
    return [k for k, n in cnt.items() if n == 1]


def test_predicates_are_exact_on_degenerate_inputs():
    # the sign of the exact determinant, whatever the rounding of its floating-point value:
    # nodes of a regular polygon (co-circular up to the rounding of their cosines), points
    # on y = x (exactly collinear), the corners of a square (exactly co-circular)
    from fractions import Fraction as F
    for n in (6, 24, 48):
        pts = [(5 + 4 * math.cos(2 * math.pi * i / n), 5 + 4 * math.sin(2 * math.pi * i / n)) for i in range(n)]
        a, b, c = pts[0], pts[n // 3], pts[2 * n // 3]
        for p in pts[1:6]:
            A, B, C, P = ([F(x) for x in q] for q in (a, b, c, p))
            d = sum(((X[0] - P[0]) ** 2 + (X[1] - P[1]) ** 2) * ((Y[0] - P[0]) * (Z[1] - P[1]) - (Z[0] - P[0]) * (Y[1] - P[1]))
                    for X, Y, Z in ((A, B, C), (B, C, A), (C, A, B)))
            assert incircle(*a, *b, *c, *p) == (d > 0) - (d < 0)
    assert orient(0.1, 0.1, 0.2, 0.2, 0.3, 0.3) == 0
    assert orient(0.0, 0.0, 1.0, 1.0, 3.0, 3.0) == 0
    assert orient(0.0, 0.0, 1.0, 0.0, 0.0, 1e-300) == 1
    assert incircle(0.0, 0.0, 1.0, 0.0, 1.0, 1.0, 0.0, 1.0) == 0


def _check_mesh(nodes, tri, max_area, holes=()):
    r, f = np.asarray(nodes), np.asarray(tri).T
    a = _areas(r, f)
    assert (a > 0).all()
    assert _angles(r, f).min() >= 30.0 - 1e-9
    assert a.max() <= max_area * (1 + 1e-12)
    # Delaunay: no node strictly inside a circumcircle
    for t in f.T:
        p = [tuple(r[v]) for v in t]
        for q in range(len(r)):
            if q in t:
                continue
            assert incircle(*p[0], *p[1], *p[2], *r[q]) <= 0
    return a.sum()


def test_annulus_graph_is_a_quality_delaunay_mesh():
    n, ro, ri = 24, 4.0, 3.0
    pts = [(5 + r * math.cos(2 * math.pi * i / n), 5 + r * math.sin(2 * math.pi * i / n)) for r in (ro, ri)
           for i in range(n)]
    segs = [(k * n + i, k * n + (i + 1) % n) for k in (0, 1) for i in range(n)]
    area_t = 0.5 * n * math.sin(2 * math.pi / n) * (ro * ro - ri * ri)
    nodes, tri = triangulate(pts, segs, [1] * n + [2] * n, [(5.0, 5.0)], area_t / 150)
    assert math.isclose(_check_mesh(nodes, tri, area_t / 150), area_t, rel_tol=1e-12)
    # boundary edges on the two polygons, lengths adding up to the perimeters
    rr = np.hypot(nodes[:, 0] - 5, nodes[:, 1] - 5)
    per = 0.0
    for a, b in _boundary_edges(np.asarray(tri).T):
        per += np.hypot(*(nodes[a] - nodes[b]))
        assert rr[a] > ri * math.cos(math.pi / n) - 1e-12 and rr[b] > ri * math.cos(math.pi / n) - 1e-12
    assert math.isclose(per, 2 * n * math.sin(math.pi / n) * (ro + ri), rel_tol=1e-12)
    # nothing meshed in the hole
    cen = nodes[np.asarray(tri)].mean(axis=1)
    assert (np.hypot(cen[:, 0] - 5, cen[:, 1] - 5) > ri * math.cos(math.pi / n)).all()


@pytest.mark.parametrize("make,ntri", [
    (lambda: polyring(s1=[10, 0], s2=[0, 10], a=[2.0], b=[3.0], sides=24, ntri=400, units=mm), 400),
    (lambda: polyring(s1=[10, 0], s2=[0, 10], a=[0], b=[4.0], sides=4, ntri=300, units=mm, orient=45), 300),
    (lambda: polyring(s1=[8, 0], s2=[0, 8], a=[0.0, 2.2], b=[1.5, 3.0], sides=16, ntri=500, units=mm), 500),
    (lambda: loadedcross(s1=[10, 0], s2=[0, 10], L1=8, L2=3, w=0.5, ntri=600, units=mm, orient=30), 600),
    (lambda: jerusalemcross(P=8, L1=6, L2=1.0, A=3, B=0.8, w=0.2, ntri=800, units=mm), 800),
])
def test_elements_hit_the_triangle_target_with_quality(make, ntri):
    sh = make()
    assert 0.9 * ntri <= sh.nface <= 1.1 * ntri
    r, f = sh.rho, sh.fv - 1
    assert (_areas(r, f) > 0).all()
    assert _angles(r, f).min() >= 30.0 - 1e-9
    # RWG topology: every edge on one or two faces, fe opposite fv
    _boundary_edges(f)
    for k in range(3):
        e = sh.fe[k] - 1
        a, b = f[(k + 1) % 3], f[(k + 2) % 3]
        assert (np.minimum(a, b) == np.minimum(sh.e1[e], sh.e2[e]) - 1).all()
        assert (np.maximum(a, b) == np.maximum(sh.e1[e], sh.e2[e]) - 1).all()


def test_cell_filling_ring_keeps_the_cell_boundary_nodes():
    ns = 10
    sh = polyring(s1=[10, 0], s2=[0, 10], a=[3.0], b=[-ns], sides=24, ntri=600, units=mm)
    r = sh.rho
    on = (np.isclose(r[:, 0], 0) | np.isclose(r[:, 0], 10) | np.isclose(r[:, 1], 0) | np.isclose(r[:, 1], 10))
    assert on.sum() == 4 * ns
    left = np.sort(r[np.isclose(r[:, 0], 0), 1])
    right = np.sort(r[np.isclose(r[:, 0], 10), 1])
    bottom = np.sort(r[np.isclose(r[:, 1], 0), 0])
    top = np.sort(r[np.isclose(r[:, 1], 10), 0])
    assert np.allclose(left, right) and np.allclose(bottom, top)
    assert math.isclose(_areas(r, sh.fv - 1).sum(), 100 - 12 * math.sin(2 * math.pi / 24) * 9, rel_tol=1e-12)

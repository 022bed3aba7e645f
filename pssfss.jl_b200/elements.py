"""Sheet constructors with structured meshes (PSSFSS.jl ``src/Elements.jl``).

``rectstrip`` (``:149-186``) and ``meander`` (``:617-729``) are built from ``recttri``
and ``combine`` exactly as in the reference, so node numbering, edge numbering and
coordinates are identical.  ``pecsheet``/``pmcsheet`` (``:108-126``) are the null
sheets.

``polyring`` (``:368-558``), ``loadedcross`` (``:794-961``) and ``jerusalemcross``
(``:963-1100``) build a boundary graph (points, segments, hole seeds) and mesh it with
``meshsub`` as the reference does; the reference's mesher is Shewchuk's Triangle, which is not
available, so ``meshsub.py`` meshes the graph by its own conforming Delaunay refinement under
the same switches: same shapes and mesh sizes, different triangulations, so results agree
with the reference only to discretisation accuracy.
"""
import math

import numpy as np

from .meshsub import meshsub
from .sheets import RWGSheet, combine, recttri, rotate, s1s2_to_b1b2, translate

_DEFAULTS = dict(cls="J", dx=0.0, dy=0.0, rot=0.0, Rsheet=0.0, save="", fufp=False)


def _check_kwargs(kwargs):
    """``check_optional_kw_arguments!`` (``Elements.jl:46-71``)."""
    if "class" in kwargs:
        kwargs["cls"] = kwargs.pop("class")
    bad = set(kwargs) - set(_DEFAULTS)
    if bad:
        raise ValueError("Illegal keywords: " + ", ".join(sorted(bad)))
    for k, v in _DEFAULTS.items():
        kwargs.setdefault(k, v)
    if kwargs["cls"] not in ("J", "M"):
        raise ValueError(f"Illegal value {kwargs['cls']} for class")
    for k in ("dx", "dy", "rot", "Rsheet"):
        if not isinstance(kwargs[k], (int, float)):
            raise ValueError(f"{k} must be a Real")
    if kwargs["Rsheet"] < 0:
        raise ValueError("Rsheet must be nonnegative")
    if not isinstance(kwargs["save"], str):
        raise ValueError("save must be an AbstractString")
    return kwargs


def _testpos(**kw):
    for k, v in kw.items():
        if not v > 0:
            raise ValueError(f"{k} must be positive!")


def pecsheet():
    """Perfect electric conducting sheet (``Elements.jl:108``)."""
    sh = RWGSheet()
    sh.style = "NULL"
    sh.cls = "E"
    return sh


def pmcsheet():
    """Perfect magnetic conducting sheet (``Elements.jl:121``)."""
    sh = RWGSheet()
    sh.style = "NULL"
    sh.cls = "H"
    return sh


def rectstrip(*, Lx, Ly, Nx, Ny, Px, Py, units, **kwarg):
    """Rectangular strip in a rectangular cell (``Elements.jl:149-186``)."""
    kwargs = dict(kwarg)
    kwargs.setdefault("fufp", True)
    _check_kwargs(kwargs)
    _testpos(Lx=Lx, Ly=Ly, Nx=Nx, Ny=Ny, Px=Px, Py=Py)
    x0 = 0.5 * (Px - Lx)
    y0 = 0.5 * (Py - Ly)
    sheet = recttri([x0, y0], [x0 + Lx, y0 + Ly], Nx, Ny)
    sheet.style = "rectstrip"
    sheet.units = units
    sheet.s1 = np.array([float(Px), 0.0])
    sheet.s2 = np.array([0.0, float(Py)])
    sheet.beta1, sheet.beta2 = s1s2_to_b1b2(sheet.s1, sheet.s2)
    sheet.fr = np.full(sheet.nface, float(kwargs["Rsheet"]))
    sheet.fufp = kwargs["fufp"]
    sheet.cls = kwargs["cls"]
    rotate(sheet, kwargs["rot"])
    if kwargs["dx"] != 0 or kwargs["dy"] != 0:
        sheet.rho = np.array([[kwargs["dx"] + x, kwargs["dy"] + y] for x, y in sheet.rho])
    sheet.xi_eta_check = (Lx == Px or Ly == Py)
    return sheet


def meander_counts(a, b, h, w1, w2, ntri):
    """Segment counts ``(nx1, nx2, ny1, ny2)`` and triangle total (``Elements.jl:635-646``)."""
    hm = h - 2 * w2
    t1 = w2 * (a + 2 * w1) / (2 * (hm * hm))
    t2 = w1 / hm
    fny2 = math.sqrt(ntri / (4 * (t1 + t2)))
    ny2 = round(fny2)
    ny2 = 1 if ny2 <= 0 else ny2
    ny1 = round(fny2 * w2 / (h - 2 * w2))
    ny1 = 1 if ny1 <= 0 else ny1
    nx1 = round(fny2 * (a - 2 * w1) / (4 * (h - 2 * w2)))
    nx1 = 1 if nx1 <= 0 else nx1
    nx2 = round(fny2 * w1 / (h - 2 * w2))
    nx2 = 1 if nx2 <= 0 else nx2
    ntotal = 4 * (2 * ny1 * (nx1 + nx2) + nx2 * ny2)
    return nx1, nx2, ny1, ny2, ntotal


def meander(*, a, b, h, w1, w2, ntri, units, orient=0.0, **kwarg):
    """Meanderline strip (``Elements.jl:617-729``)."""
    kwargs = dict(kwarg)
    kwargs.setdefault("fufp", True)
    _check_kwargs(kwargs)
    _testpos(a=a, b=b, h=h, w1=w1, w2=w2, ntri=ntri)
    if orient != 0 and a != b:
        raise ValueError("Nonzero orient only allowed for square unit cell")
    morient = orient % 360
    if morient not in (0, 90, 180, 270):
        raise ValueError("orient must be a multiple of 90")
    nx1, nx2, ny1, ny2, _ = meander_counts(a, b, h, w1, w2, ntri)
    yoffset = (b - h) / 2
    Lx = (a / 2 - w1) / 2
    Ly = h - 2 * w2

    def rt(bl, d):
        return [bl[0] + d[0], bl[1] + d[1]]

    bl = [0.0, yoffset]
    sh1 = recttri(bl, rt(bl, [Lx, w2]), nx1, ny1)
    bl = [Lx, yoffset]
    sh2 = recttri(bl, rt(bl, [w1, w2]), nx2, ny1)
    sh3 = combine(sh1, sh2, "x", Lx)
    bl = [Lx, yoffset + w2]
    sh1 = recttri(bl, rt(bl, [w1, Ly]), nx2, ny2)
    sh2 = combine(sh3, sh1, "y", bl[1])
    bl = [Lx, yoffset + w2 + Ly]
    sh1 = recttri(bl, rt(bl, [w1, w2]), nx2, ny1)
    sh3 = combine(sh2, sh1, "y", bl[1])
    bl = [Lx + w1, yoffset + w2 + Ly]
    tr = rt(bl, [2 * Lx, w2])
    sh1 = recttri(bl, tr, 2 * nx1, ny1)
    sh2 = combine(sh3, sh1, "x", bl[0])
    bl = [tr[0], bl[1]]
    tr = rt(bl, [w1, w2])
    sh1 = recttri(bl, tr, nx2, ny1)
    sh3 = combine(sh2, sh1, "x", bl[0])
    bl = [bl[0], yoffset + w2]
    tr = rt(bl, [w1, Ly])
    sh1 = recttri(bl, tr, nx2, ny2)
    sh2 = combine(sh3, sh1, "y", tr[1])
    bl = [bl[0], yoffset]
    tr = rt(bl, [w1, w2])
    sh1 = recttri(bl, tr, nx2, ny1)
    sh3 = combine(sh2, sh1, "y", tr[1])
    bl = [tr[0], yoffset]
    tr = rt(bl, [Lx, w2])
    sh1 = recttri(bl, tr, nx1, ny1)
    sheet = combine(sh3, sh1, "x", bl[0])
    if morient != 0:
        if morient == 90:
            xf = lambda x, y: (b - y, x)
        elif morient == 180:
            xf = lambda x, y: (a - x, b - y)
        else:
            xf = lambda x, y: (y, a - x)
        sheet.rho = np.array([xf(x, y) for x, y in sheet.rho], float)
    sheet.fr = np.full(sheet.nface, float(kwargs["Rsheet"]))
    sheet.fufp = kwargs["fufp"]
    sheet.cls = kwargs["cls"]
    sheet.style = "meander"
    sheet.units = units
    sheet.s1 = np.array([float(a), 0.0])
    sheet.s2 = np.array([0.0, float(b)])
    sheet.beta1, sheet.beta2 = s1s2_to_b1b2(sheet.s1, sheet.s2)
    rotate(sheet, kwargs["rot"])
    if kwargs["dx"] != 0 or kwargs["dy"] != 0:
        sheet.rho = np.array([[kwargs["dx"] + x, kwargs["dy"] + y] for x, y in sheet.rho])
    sheet.xi_eta_check = True
    return sheet


def _tritri(w, nw):
    """Isosceles right triangle, apex at the origin, base of length ``w`` on x = w/2
    bisected by the x-axis (``Elements.jl:296``).  Nodes on the grid of the reference's
    layout (spacing w/nw; for odd nw the columns sit at half steps and the apex is alone);
    the columns are joined by squares split on a diagonal and one half-square at each end,
    a structured triangulation of the region the reference hands to Triangle."""
    dxy = w / nw
    cols = []
    if nw % 2 == 0:
        k = nw // 2
        for i in range(k + 1):
            cols.append([(i * dxy, j * dxy) for j in range(-i, i + 1)])
    else:
        k = (nw + 1) // 2
        cols.append([(0.0, 0.0)])
        for mx in range(1, k + 1):
            x = (2 * mx - 1) / 2 * dxy
            cols.append([(x, -x + t * dxy) for t in range(2 * mx)])
    rho, ids = [], []
    for col in cols:
        ids.append(list(range(len(rho), len(rho) + len(col))))
        rho.extend(col)
    tris = []
    for a, b in zip(ids[:-1], ids[1:]):
        if len(b) == 2:  # odd nw: the lone apex and the first half-step column
            tris.append((a[0], b[0], b[1]))
            continue
        # column b has two more nodes than a, one beyond each end; node a[t] aligns with b[t+1]
        tris.append((a[0], b[0], b[1]))                  # lower end
        for t in range(len(a) - 1):                       # squares
            tris.append((a[t], b[t + 1], b[t + 2]))
            tris.append((a[t], b[t + 2], a[t + 1]))
        tris.append((a[-1], b[-2], b[-1]))               # upper end
    rho = np.array(rho, float)
    out = []
    for t in tris:
        p0, p1, p2 = (rho[i] for i in t)
        cross = (p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1])
        out.append(t if cross > 0 else (t[0], t[2], t[1]))
    return _sheet_from_triangles(rho, out)


def diagstrip(*, P, w, orient, Nl, Nw, units, **kwarg):
    """Strip along a diagonal of a square cell of side ``P`` (``Elements.jl:218-294``):
    width ``w``, ``orient`` 45 (lower left to upper right) or -45, ``Nl`` x ``Nw`` cells on
    the rectangular middle part; the ends taper to the cell corners as right isosceles
    triangles (``_tritri``), and the two opposite corners carry the matching pieces so the
    strip is continuous from cell to cell."""
    kwargs = dict(kwarg)
    kwargs.setdefault("fufp", True)
    _check_kwargs(kwargs)
    _testpos(P=P, w=w, Nl=Nl, Nw=Nw)
    if kwargs["dx"] != 0 or kwargs["dy"] != 0:
        raise ValueError("Translation not allowed for this style of sheet")
    if abs(orient) != 45:
        raise ValueError("orient must be 45 or -45")
    r2 = math.sqrt(2.0)
    xbl = w / 2 - (r2 * P if orient < 0 else 0.0)
    rhobl = np.array([xbl, -w / 2])
    rhotr = rhobl + np.array([r2 * P - w, w])
    sh1 = recttri(rhobl, rhotr, Nl, Nw)
    sh2 = translate(rotate(_tritri(w, Nw), 180.0), rhotr[0] + w / 2, 0.0)
    sh3 = combine(sh1, sh2, "x", rhotr[0])
    sh2 = translate(_tritri(w, Nw), xbl - w / 2, 0.0)
    sh1 = combine(sh3, sh2, "x", xbl)
    rotate(sh1, orient)
    if orient < 0:
        translate(sh1, P, 0.0)
    if orient > 0:
        sh2 = translate(rotate(_tritri(w, Nw), -45.0), 0.0, P)      # top left corner
        sh3 = combine(sh1, sh2, " ", 0.0)
        sh1 = translate(rotate(_tritri(w, Nw), 135.0), P, 0.0)     # bottom right corner
    else:
        sh2 = translate(rotate(_tritri(w, Nw), -135.0), P, P)      # top right corner
        sh3 = combine(sh1, sh2, " ", 0.0)
        sh1 = translate(rotate(_tritri(w, Nw), 45.0), 0.0, 0.0)    # bottom left corner
    sheet = combine(sh3, sh1, " ", 0.0)
    sheet.rot = 0.0
    _finish_sheet(sheet, "diagstrip", units, [P, 0.0], [0.0, P], kwargs)
    sheet.xi_eta_check = True
    return sheet


def _sheet_from_triangles(rho, tris):
    """RWGSheet topology from node coordinates (nnode, 2) and counter-clockwise triangles
    (nface, 3) of 0-based node indices: 1-based ``fv``, ``fe`` with ``fe[k]`` the edge
    opposite ``fv[k]``, and edges ``e1``/``e2`` numbered in order of first appearance."""
    from .sheets import RWGSheet
    rho = np.asarray(rho, float)
    tris = np.asarray(tris, np.int64)
    area = ((rho[tris[:, 1], 0] - rho[tris[:, 0], 0]) * (rho[tris[:, 2], 1] - rho[tris[:, 0], 1]) -
            (rho[tris[:, 2], 0] - rho[tris[:, 0], 0]) * (rho[tris[:, 1], 1] - rho[tris[:, 0], 1]))
    if np.any(area <= 0):
        raise ValueError("triangles must be counter-clockwise and non-degenerate")
    edges = {}
    e1, e2 = [], []
    fe = np.zeros((3, len(tris)), np.int64)
    for f, (a, b, c) in enumerate(tris):
        for k, (p, q) in enumerate(((b, c), (c, a), (a, b))):  # edge opposite vertex k
            key = (min(p, q), max(p, q))
            if key not in edges:
                edges[key] = len(e1) + 1
                e1.append(key[0] + 1)
                e2.append(key[1] + 1)
            fe[k, f] = edges[key]
    sh = RWGSheet()
    sh.rho = rho
    sh.fv = (tris.T + 1).astype(np.int64)
    sh.fe = fe
    sh.e1 = np.array(e1, np.int64)
    sh.e2 = np.array(e2, np.int64)
    return sh


def _finish_sheet(sheet, style, units, s1, s2, kwargs):
    sheet.style = style
    sheet.units = units
    sheet.s1 = np.asarray(s1, float)
    sheet.s2 = np.asarray(s2, float)
    sheet.beta1, sheet.beta2 = s1s2_to_b1b2(sheet.s1, sheet.s2)
    sheet.fr = np.full(sheet.nface, float(kwargs["Rsheet"]))
    sheet.fufp = kwargs["fufp"]
    sheet.cls = kwargs["cls"]
    rotate(sheet, kwargs["rot"])
    if kwargs["dx"] != 0 or kwargs["dy"] != 0:
        sheet.rho = np.array([[kwargs["dx"] + x, kwargs["dy"] + y] for x, y in sheet.rho])
    sheet.xi_eta_check = False
    return sheet


def polyring(*, s1, s2, a, b, sides, ntri, units, orient=0.0, **kwarg):
    """Concentric regular-polygon rings (``Elements.jl:368-558``): ring i spans radii
    a[i]..b[i] (a[i] = 0: a solid polygon), centred in the cell, first vertex at angle
    ``orient`` (degrees), about ``ntri`` triangles in total.  ``b[-1] < 0`` makes the last
    ring fill the cell out to its boundary, with ``-b[-1]`` edges along the shorter lattice
    vector (the longer one in proportion), and the sheet is periodic across the cell edges.
    The boundary graph, its hole seeds and the area target are the reference's; the graph is
    meshed by ``meshsub`` (conforming Delaunay, 30-degree angle bound), the cell boundary of
    a cell-filling ring without added nodes so opposite edges keep matching nodes."""
    kwargs = dict(kwarg)
    kwargs.setdefault("fufp", False)
    _check_kwargs(kwargs)
    _testpos(sides=sides, ntri=ntri)
    a = [float(x) for x in a]
    b = [float(x) for x in b]
    if len(a) != len(b):
        raise ValueError("length(a) !== length(b)")
    nring = len(a)
    fillcell = b[-1] < 0
    for i in range(nring):
        if a[i] >= b[i] and not (fillcell and i == nring - 1):
            raise ValueError(f"a[{i + 1}] >= b[{i + 1}]")
        if i + 1 < nring and b[i] >= a[i + 1]:
            raise ValueError(f"b[{i + 1}] >= a[{i + 2}]")
    s1 = np.asarray(s1, float)
    s2 = np.asarray(s2, float)
    if s1.shape != (2,) or s2.shape != (2,):
        raise ValueError("s1 and s2 must have length 2")
    rho0 = 0.5 * (s1 + s2)
    alpha = 2 * math.pi / sides
    area_factor = 0.5 * sides * math.sin(alpha)
    areas = [(bb * bb - aa * aa) * area_factor for aa, bb in zip(a, b)]
    if fillcell:
        if a[-1] <= 0:
            raise ValueError("a cell-filling ring needs a[end] > 0")
        nshort = int(round(-b[-1]))
        if nshort < 1:
            raise ValueError("-b[end] must be a positive number of edges")
        n1, n2 = np.linalg.norm(s1), np.linalg.norm(s2)
        ns1, ns2 = (nshort, round(nshort * n2 / n1)) if n1 <= n2 else (round(nshort * n1 / n2), nshort)
        areas[-1] = abs(s1[0] * s2[1] - s1[1] * s2[0]) - area_factor * a[-1] * a[-1]
    pts, segs, marks = [], [], []

    def loop(points, marker):
        base = len(pts)
        pts.extend(points)
        k = len(points)
        segs.extend((base + i, base + (i + 1) % k) for i in range(k))
        marks.extend([marker] * k)

    def polygon(r):
        o = math.radians(orient)
        return [rho0 + r * np.array([math.cos(o + i * alpha), math.sin(o + i * alpha)]) for i in range(sides)]
    boundary = 0
    for iring in range(nring):
        if a[iring] == 0:
            boundary += 1
            loop(polygon(b[iring]), boundary)
        elif fillcell and iring == nring - 1:
            boundary += 1
            cell = ([i / ns1 * s1 for i in range(ns1)] + [s1 + i / ns2 * s2 for i in range(ns2)] +
                    [s1 + s2 - i / ns1 * s1 for i in range(ns1)] + [s2 - i / ns2 * s2 for i in range(ns2)])
            loop(cell, boundary)
            cell_marker = boundary
            boundary += 1
            loop(polygon(a[iring]), boundary)
        else:
            for r in (b[iring], a[iring]):
                boundary += 1
                loop(polygon(r), boundary)
    holes = []
    if a[0] > 0:
        holes.append(rho0)
    u = np.array([math.cos(math.radians(orient)), math.sin(math.radians(orient))])
    for i in range(nring - 1):
        holes.append(rho0 + 0.5 * (b[i] + a[i + 1]) * u)
    sheet = meshsub(points=np.array(pts).T, seglist=np.array(segs).T + 1, segmarkers=marks,
                    holes=np.array(holes).T if holes else None, area=sum(areas) / ntri, ntri=ntri,
                    fixed_markers=(cell_marker,) if fillcell else ())
    _finish_sheet(sheet, "polyring", units, s1, s2, kwargs)
    sheet.xi_eta_check = fillcell
    return sheet


def _rect_union_outline(rects, holes=()):
    """Boundary graph of a union of axis-aligned rectangles (x0, y0, x1, y1) less the union
    of the ``holes`` rectangles: the boundary loops of the region (corners only, the region
    on the left of each segment), one marker per loop, and a seed point just outside the
    region beside every loop (hole seeds for ``meshsub``)."""
    allr = list(rects) + list(holes)
    xs = np.array(sorted(set(round(v, 12) for r in allr for v in (r[0], r[2]))))
    ys = np.array(sorted(set(round(v, 12) for r in allr for v in (r[1], r[3]))))
    xc, yc = 0.5 * (xs[:-1] + xs[1:]), 0.5 * (ys[:-1] + ys[1:])
    inside = np.zeros((len(xc), len(yc)), bool)
    for x0, y0, x1, y1 in rects:
        inside |= ((xc > x0) & (xc < x1))[:, None] & ((yc > y0) & (yc < y1))[None, :]
    for x0, y0, x1, y1 in holes:
        inside &= ~(((xc > x0) & (xc < x1))[:, None] & ((yc > y0) & (yc < y1))[None, :])

    def ins(i, j):
        return 0 <= i < len(xc) and 0 <= j < len(yc) and inside[i, j]
    nxt = {}  # directed boundary edges, region on the left: start grid node -> end grid node
    for i in range(len(xc)):
        for j in range(len(yc)):
            if not inside[i, j]:
                continue
            if not ins(i, j - 1):
                nxt.setdefault((i, j), []).append((i + 1, j))
            if not ins(i + 1, j):
                nxt.setdefault((i + 1, j), []).append((i + 1, j + 1))
            if not ins(i, j + 1):
                nxt.setdefault((i + 1, j + 1), []).append((i, j + 1))
            if not ins(i - 1, j):
                nxt.setdefault((i, j + 1), []).append((i, j))
    pts, segs, marks, seeds = [], [], [], []
    dmin = min(np.diff(xs).min(), np.diff(ys).min())
    while nxt:
        start = min(nxt)
        loop = [start]
        cur, prev_dir = start, None
        while True:
            outs = nxt[cur]
            if len(outs) > 1 and prev_dir is not None:  # a pinch: turn left first
                outs.sort(key=lambda q: -((prev_dir[0] * (q[1] - cur[1]) - prev_dir[1] * (q[0] - cur[0]))))
            q = outs.pop(0)
            if not outs:
                del nxt[cur]
            prev_dir = (q[0] - cur[0], q[1] - cur[1])
            cur = q
            if cur == start:
                break
            loop.append(cur)
        # corners only
        k = len(loop)
        corner = []
        for m in range(k):
            p0, p1, p2 = loop[m - 1], loop[m], loop[(m + 1) % k]
            if (p1[0] - p0[0]) * (p2[1] - p1[1]) - (p1[1] - p0[1]) * (p2[0] - p1[0]) != 0:
                corner.append(p1)
        base = len(pts)
        pts.extend((xs[i], ys[j]) for i, j in corner)
        marker = len(seeds) + 1
        segs.extend((base + m, base + (m + 1) % len(corner)) for m in range(len(corner)))
        marks.extend([marker] * len(corner))
        (i0, j0), (i1, j1) = loop[0], loop[1]
        mx, my = 0.5 * (xs[i0] + xs[i1]), 0.5 * (ys[j0] + ys[j1])
        dx, dy = np.sign(i1 - i0), np.sign(j1 - j0)
        seeds.append((mx + 0.25 * dmin * dy, my - 0.25 * dmin * dx))  # right of the edge: outside
    return np.array(pts), np.array(segs), marks, np.array(seeds)


def _outline_area(pts, segs):
    """Area enclosed by the boundary loops (region on the left of every segment)."""
    p, q = pts[segs[:, 0]], pts[segs[:, 1]]
    return 0.5 * float(np.sum(p[:, 0] * q[:, 1] - q[:, 0] * p[:, 1]))


def _mesh_outline(rects, holes, ntri, rot=None, shift=(0.0, 0.0)):
    """``meshsub`` of a rectangle union's outline (about ``ntri`` triangles, maximum area
    the region's over ``ntri`` as the reference's ``areat / ntri``), optionally rotated by
    the matrix ``rot`` (row vectors) and shifted."""
    pts, segs, marks, seeds = _rect_union_outline(rects, holes)
    if rot is not None:
        pts, seeds = pts @ rot, seeds @ rot
    pts, seeds = pts + np.asarray(shift), seeds + np.asarray(shift)
    return meshsub(points=pts.T, seglist=segs.T + 1, segmarkers=marks, holes=seeds.T,
                   area=_outline_area(pts, segs) / ntri, ntri=ntri)


def loadedcross(*, s1, s2, L1, L2, w, ntri, units, orient=0.0, **kwarg):
    """Loaded cross (``Elements.jl:794-961``): a cross of arm length ``L1`` (tip to tip) and
    arm width ``L2`` centred in the cell, hollowed to a loop of trace width ``w`` when
    2w < L2 (solid otherwise), rotated by ``orient`` degrees about its centre.  The outline
    (axis-aligned before the rotation) is meshed by ``meshsub`` to about ``ntri`` triangles."""
    kwargs = dict(kwarg)
    kwargs.setdefault("fufp", False)
    _check_kwargs(kwargs)
    _testpos(L1=L1, L2=L2, w=w, ntri=ntri)
    s1 = np.asarray(s1, float)
    s2 = np.asarray(s2, float)
    if s1.shape != (2,) or s2.shape != (2,):
        raise ValueError("s1 and s2 must be 2-vectors")
    if not L2 < L1:
        raise ValueError("L2 must be smaller than L1")
    h1, h2 = L1 / 2, L2 / 2
    rects = [(-h1, -h2, h1, h2), (-h2, -h1, h2, h1)]
    holes = []
    if 2 * w < L2:
        holes = [(-h1 + w, -h2 + w, h1 - w, h2 - w), (-h2 + w, -h1 + w, h2 - w, h1 - w)]
    rot = None
    if orient != 0:
        sn, cs = math.sin(math.radians(orient)), math.cos(math.radians(orient))
        rot = np.array([[cs, sn], [-sn, cs]])
    sheet = _mesh_outline(rects, holes, ntri, rot, 0.5 * (s1 + s2))
    return _finish_sheet(sheet, "loadedcross", units, s1, s2, kwargs)


def jerusalemcross(*, P, L1, L2, A, B, w, ntri, units, **kwarg):
    """Jerusalem cross in a square cell of period P (``Elements.jl:963``): arms of length L1
    (tip to tip) and width L2, end caps of length A and width B, drawn as an outline of
    trace width w.  As in the reference, a part whose width is at most 2w is solid: w >= L2/2
    fills the arms, w >= B/2 the caps, both fill the whole cross.  With hollow arms and
    solid caps the arm slot stops a trace width short of the caps; with both hollow the
    slot runs into the caps' openings.  The outline is meshed by ``meshsub`` to about
    ``ntri`` triangles."""
    kwargs = dict(kwarg)
    kwargs.setdefault("fufp", False)
    _check_kwargs(kwargs)
    _testpos(P=P, L1=L1, L2=L2, A=A, B=B, w=w, ntri=ntri)
    if not (L1 < P and A < P and L2 < A and (L1 - L2) / 2 > B):
        raise ValueError("inconsistent Jerusalem-cross dimensions")
    c = P / 2
    h1, h2, hA = L1 / 2, L2 / 2, A / 2
    rects = [(c - h1, c - h2, c + h1, c + h2), (c - h2, c - h1, c + h2, c + h1),   # arms
             (c - h1, c - hA, c - h1 + B, c + hA), (c + h1 - B, c - hA, c + h1, c + hA),  # caps
             (c - hA, c - h1, c + hA, c - h1 + B), (c - hA, c + h1 - B, c + hA, c + h1)]
    hollow_arms, hollow_caps = 2 * w < L2, 2 * w < B
    holes = []
    if hollow_arms:
        reach = h1 - w if hollow_caps else h1 - B - w   # the slot's half length
        g = h2 - w
        holes += [(c - reach, c - g, c + reach, c + g), (c - g, c - reach, c + g, c + reach)]
    if hollow_caps:
        a_, b_ = hA - w, h1 - w
        holes += [(c - b_, c - a_, c - h1 + B - w, c + a_), (c + h1 - B + w, c - a_, c + b_, c + a_),
                  (c - a_, c - b_, c + a_, c - h1 + B - w), (c - a_, c + h1 - B + w, c + a_, c + b_)]
    sheet = _mesh_outline(rects, holes, ntri)
    return _finish_sheet(sheet, "jerusalemcross", units, [float(P), 0.0], [0.0, float(P)], kwargs)

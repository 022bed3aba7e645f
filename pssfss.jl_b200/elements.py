"""Sheet constructors with structured meshes (PSSFSS.jl ``src/Elements.jl``).

``rectstrip`` (``:149-186``) and ``meander`` (``:617-729``) are built from ``recttri``
and ``combine`` exactly as in the reference, so node numbering, edge numbering and
coordinates are identical.  ``pecsheet``/``pmcsheet`` (``:108-126``) are the null
sheets.

``polyring`` (``:368-558``) and ``jerusalemcross`` (``:963-...``) take the reference's
geometry arguments but are meshed here with structured meshes of their own (a polar grid
per ring; a rectilinear grid over the union of rectangles), because the reference meshes
them with Shewchuk's Triangle, which is not available: same shapes, different
triangulations, so results agree with the reference only to discretisation accuracy.
"""
import math

import numpy as np

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
    ``orient`` (degrees).  Structured polar mesh of about ``ntri`` triangles in total,
    shared among the rings by area.  ``b[-1] < 0`` makes the last ring fill the cell out to
    its boundary, with ``-b[-1]`` edges along the shorter lattice vector (the longer one in
    proportion): its polygonal inner edge is joined to the cell boundary by layers blended
    along rays from the centre, the last of them zipped to the boundary nodes by angle, and
    the sheet is periodic across the cell edges."""
    kwargs = dict(kwarg)
    kwargs.setdefault("fufp", False)
    _check_kwargs(kwargs)
    _testpos(sides=sides, ntri=ntri)
    a = [float(x) for x in a]
    b = [float(x) for x in b]
    if len(a) != len(b):
        raise ValueError("length(a) !== length(b)")
    fillcell = b[-1] < 0
    for i in range(len(a)):
        if a[i] >= b[i] and not (fillcell and i == len(a) - 1):
            raise ValueError(f"a[{i + 1}] >= b[{i + 1}]")
        if i + 1 < len(a) and b[i] >= a[i + 1]:
            raise ValueError(f"b[{i + 1}] >= a[{i + 2}]")
    s1 = np.asarray(s1, float)
    s2 = np.asarray(s2, float)
    rho0 = 0.5 * (s1 + s2)
    alpha = 2 * math.pi / sides
    area_factor = 0.5 * sides * math.sin(alpha)
    areas = [(bb * bb - aa * aa) * area_factor for aa, bb in zip(a, b)]
    if fillcell:
        if a[-1] <= 0:
            raise ValueError("a cell-filling ring needs a[end] > 0")
        areas[-1] = abs(s1[0] * s2[1] - s1[1] * s2[0]) - area_factor * a[-1] * a[-1]
    rho, tris = [], []
    for iring, (aa, bb, ar) in enumerate(zip(a, b, areas)):
        nt = max(2 * sides, round(ntri * ar / sum(areas)))
        if fillcell and iring == len(a) - 1:
            _cell_ring(rho, tris, rho0, s1, s2, int(round(-bb)), aa, sides, orient, nt)
            continue
        # ns segments per polygon side, nr radial layers, cells as close to square as the
        # triangle budget allows: 2 * sides * ns * nr ~ nt with (bb - aa) / nr ~ side(rmid) / ns
        rmid = 0.5 * (aa + bb)
        side = 2 * rmid * math.sin(alpha / 2)
        ratio = (bb - aa) / side  # nr / ns
        ns = max(1, round(math.sqrt(nt / (2 * sides * ratio))))
        nr = max(1, round(nt / (2 * sides * ns)))
        m = sides * ns  # nodes per layer
        verts = [np.array([math.cos(math.radians(orient) + i * alpha), math.sin(math.radians(orient) + i * alpha)])
                 for i in range(sides)]
        dirs = [verts[i] + (verts[(i + 1) % sides] - verts[i]) * (t / ns) for i in range(sides) for t in range(ns)]
        layers = []
        r_in = aa if aa > 0 else bb / (nr + 1)
        nl = nr + 1 if aa > 0 else nr
        for k in range(nl + (0 if aa > 0 else 1)):
            r = (aa + (bb - aa) * k / nr) if aa > 0 else bb * (k + 1) / (nr + 1)
            base = len(rho)
            rho.extend(rho0 + r * d for d in dirs)
            layers.append(base)
        if aa == 0:  # centre node and its fan to the first layer
            c = len(rho)
            rho.append(rho0.copy())
            for i in range(m):
                tris.append((c, layers[0] + i, layers[0] + (i + 1) % m))
        for k in range(len(layers) - 1):
            lo, hi = layers[k], layers[k + 1]
            for i in range(m):
                i1 = (i + 1) % m
                tris.append((lo + i, hi + i, hi + i1))
                tris.append((lo + i, hi + i1, lo + i1))
    sheet = _sheet_from_triangles(rho, tris)
    _finish_sheet(sheet, "polyring", units, s1, s2, kwargs)
    sheet.xi_eta_check = fillcell
    return sheet


def _cell_ring(rho, tris, rho0, s1, s2, nshort, a, sides, orient, nt):
    """Append the mesh of the region between the regular polygon of radius ``a`` (centred at
    ``rho0``, first vertex at ``orient`` degrees) and the boundary of the cell spanned by
    ``s1``, ``s2`` from the origin.  Boundary nodes are uniform, ``nshort`` edges along the
    shorter lattice vector and the longer one in proportion (``Elements.jl:393-403``), so
    opposite edges match for the periodic basis functions.  The polygon, with about as many
    nodes as the boundary, is carried outward in layers along the rays through its nodes
    (quad strips split on a diagonal); the last layer is joined to the boundary nodes by a
    merge in angle about the centre."""
    if nshort < 1:
        raise ValueError("-b[end] must be a positive number of edges")
    n1, n2 = np.linalg.norm(s1), np.linalg.norm(s2)
    ns1, ns2 = (nshort, round(nshort * n2 / n1)) if n1 <= n2 else (round(nshort * n1 / n2), nshort)
    outer = ([i / ns1 * s1 for i in range(ns1)] + [s1 + i / ns2 * s2 for i in range(ns2)] +
             [s1 + s2 - i / ns1 * s1 for i in range(ns1)] + [s2 - i / ns2 * s2 for i in range(ns2)])
    M = len(outer)
    ns = max(1, round(M / sides))
    m = sides * ns
    alpha = 2 * math.pi / sides
    verts = [rho0 + a * np.array([math.cos(math.radians(orient) + i * alpha), math.sin(math.radians(orient) + i * alpha)])
             for i in range(sides)]
    poly = [verts[i] + (verts[(i + 1) % sides] - verts[i]) * (t / ns) for i in range(sides) for t in range(ns)]
    Binv = np.linalg.inv(np.column_stack([s1, s2]))

    def reach(d):  # distance from the centre to the cell boundary along direction d
        q = Binv @ d
        return 0.5 / max(abs(q[0]), abs(q[1]))
    rays = []
    for p in poly:
        v = p - rho0
        r0 = np.linalg.norm(v)
        rays.append((r0, v / r0, reach(v / r0)))
    nlayer = max(1, 1 + round((nt - m - M) / (2 * m)))
    layers = []
    for k in range(nlayer):
        base = len(rho)
        rho.extend(rho0 + (r0 + (R - r0) * k / nlayer) * d for r0, d, R in rays)
        layers.append(base)
    for k in range(nlayer - 1):
        lo, hi = layers[k], layers[k + 1]
        for i in range(m):
            i1 = (i + 1) % m
            tris.append((lo + i, hi + i, hi + i1))
            tris.append((lo + i, hi + i1, lo + i1))
    obase = len(rho)
    rho.extend(outer)

    def ang(p):
        return math.atan2(p[1] - rho0[1], p[0] - rho0[0])
    ref = ang(outer[0])
    inner = [layers[-1] + i for i in range(m)]
    ai = [(ang(rho[q]) - ref) % (2 * math.pi) for q in inner]
    s0 = int(np.argmin(ai))
    inner, ai = inner[s0:] + inner[:s0], ai[s0:] + ai[:s0]
    ao = [(ang(p) - ref) % (2 * math.pi) for p in outer]
    ao[0] = 0.0
    i = j = 0
    while i < m or j < M:
        nxt_i = ai[(i + 1) % m] + (2 * math.pi if i + 1 >= m else 0.0)
        nxt_o = ao[(j + 1) % M] + (2 * math.pi if j + 1 >= M else 0.0)
        I, O = inner[i % m], obase + j % M
        if j < M and (i >= m or nxt_o <= nxt_i):
            tris.append((I, O, obase + (j + 1) % M))
            j += 1
        else:
            tris.append((I, O, inner[(i + 1) % m]))
            i += 1


def _rect_union_mesh(rects, h, holes=()):
    """Conforming triangulation of a union of axis-aligned rectangles (x0, y0, x1, y1) less
    the union of the ``holes`` rectangles: grid lines at every rectangle edge, refined to
    steps <= h, cells inside the region split along the lower-left/upper-right diagonal."""
    def lines(vals):
        vals = sorted(set(round(v, 12) for v in vals))
        out = [vals[0]]
        for lo, hi in zip(vals, vals[1:]):
            k = max(1, math.ceil((hi - lo) / h - 1e-9))
            out.extend(lo + (hi - lo) * (i + 1) / k for i in range(k))
        return np.array(out)
    allr = list(rects) + list(holes)
    xs = lines([r[0] for r in allr] + [r[2] for r in allr])
    ys = lines([r[1] for r in allr] + [r[3] for r in allr])
    inside = np.zeros((len(xs) - 1, len(ys) - 1), bool)
    xc = 0.5 * (xs[:-1] + xs[1:])
    yc = 0.5 * (ys[:-1] + ys[1:])
    for x0, y0, x1, y1 in rects:
        inside |= ((xc > x0) & (xc < x1))[:, None] & ((yc > y0) & (yc < y1))[None, :]
    for x0, y0, x1, y1 in holes:
        inside &= ~(((xc > x0) & (xc < x1))[:, None] & ((yc > y0) & (yc < y1))[None, :])
    nid = -np.ones((len(xs), len(ys)), np.int64)
    rho, tris = [], []

    def node(i, j):
        if nid[i, j] < 0:
            nid[i, j] = len(rho)
            rho.append((xs[i], ys[j]))
        return nid[i, j]
    for j in range(len(ys) - 1):
        for i in range(len(xs) - 1):
            if inside[i, j]:
                ll, lr, ur, ul = node(i, j), node(i + 1, j), node(i + 1, j + 1), node(i, j + 1)
                tris.append((ll, ur, ul))
                tris.append((ll, lr, ur))
    return np.array(rho), np.array(tris)


def loadedcross(*, s1, s2, L1, L2, w, ntri, units, orient=0.0, **kwarg):
    """Loaded cross (``Elements.jl:794-961``): a cross of arm length ``L1`` (tip to tip) and
    arm width ``L2`` centred in the cell, hollowed to a loop of trace width ``w`` when
    2w < L2 (solid otherwise), rotated by ``orient`` degrees about its centre.  The outline
    is axis-aligned before the rotation, so it is meshed by a conforming grid (cells of
    about equal area, ~``ntri`` triangles) instead of the reference's Triangle mesh."""
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
    area = 2 * L1 * L2 - L2 * L2
    holes = []
    if 2 * w < L2:
        holes = [(-h1 + w, -h2 + w, h1 - w, h2 - w), (-h2 + w, -h1 + w, h2 - w, h1 - w)]
        a1, a2 = L1 - 2 * w, L2 - 2 * w
        area -= 2 * a1 * a2 - a2 * a2
    h = math.sqrt(2 * area / ntri)
    rho, tris = _rect_union_mesh(rects, min(h, w if holes else h), holes)
    if orient != 0:
        sn, cs = math.sin(math.radians(orient)), math.cos(math.radians(orient))
        rho = rho @ np.array([[cs, sn], [-sn, cs]])
    rho = rho + 0.5 * (s1 + s2)
    sheet = _sheet_from_triangles(rho, tris)
    return _finish_sheet(sheet, "loadedcross", units, s1, s2, kwargs)


def jerusalemcross(*, P, L1, L2, A, B, w, ntri, units, **kwarg):
    """Jerusalem cross in a square cell of period P (``Elements.jl:963``): arms of length L1
    (tip to tip) and width L2, end caps of length A and width B, drawn as an outline of
    trace width w.  As in the reference, a part whose width is at most 2w is solid: w >= L2/2
    fills the arms, w >= B/2 the caps, both fill the whole cross.  With hollow arms and
    solid caps the arm slot stops a trace width short of the caps; with both hollow the
    slot runs into the caps' openings.  The outline is axis-aligned, so it is meshed by a
    conforming grid (about ``ntri`` triangles) instead of the reference's Triangle mesh."""
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
    area = 2 * L1 * L2 - L2 * L2 + 4 * (A * B - L2 * B)
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
    h = math.sqrt(2 * area / ntri)  # two triangles per h x h cell
    rho, tris = _rect_union_mesh(rects, min(h, w) if holes else h, holes)
    sheet = _sheet_from_triangles(rho, tris)
    return _finish_sheet(sheet, "jerusalemcross", units, [float(P), 0.0], [0.0, float(P)], kwargs)

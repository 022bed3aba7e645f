"""Quality triangulation of polygonal regions: ``meshsub`` (``src/Meshsub.jl:12-113``).

The reference hands a planar straight-line graph (boundary points, segments, segment
markers, hole seeds) to Shewchuk's Triangle with the switches ``pDa<area>q30Qe`` and
repeats the call, scaling the maximum triangle area by ``(ntri_got / ntri) ** (1/3)``, until
the triangle count is within 10 % of ``ntri`` (at most 14 calls, ``Meshsub.jl:64-80``).
Triangle is not available here, so this module meshes the same graph with its own
conforming Delaunay refinement (Ruppert's algorithm, with the switches' meaning):

* ``p``: the input segments are kept - a segment whose diametral circle holds a vertex
  (it is "encroached", or missing from the triangulation) is split at its midpoint;
* ``D``: every triangle is Delaunay (no vertex inside any circumcircle): the mesh is a
  Delaunay triangulation of its vertices, built by Bowyer-Watson insertion with exact
  orientation and in-circle predicates (floating-point filter, exact integer fallback);
* ``a``: triangles larger than the area bound are split at their circumcentre;
* ``q``: triangles with an angle below the bound (circumradius over shortest edge above
  1 / (2 sin q)) are split at their circumcentre; a circumcentre that would encroach a
  segment is not inserted, the segment is split instead;
* holes: triangles reachable from a hole seed (or from outside the graph) without
  crossing a segment are removed.

Same input graph, same rules and the same area iteration; the triangulations differ from
Triangle's in the order of insertions, so meshes are alike in size and quality, not equal.
Segments whose marker is in ``fixed_markers`` are never split (no points are added on
them, as Triangle's ``Y`` switch): the periodic cell boundary of a cell-filling ring keeps
its matching nodes on opposite sides.
"""
import math

import numpy as np

__all__ = ["meshsub", "triangulate"]

_EPS = 2.0 ** -53
_ORIENT_BOUND = (3.0 + 16.0 * _EPS) * _EPS
_INCIRCLE_BOUND = (10.0 + 96.0 * _EPS) * _EPS


def _ints(*vals):
    """The floats as integers over one common power-of-two denominator (exact)."""
    rat = [v.as_integer_ratio() for v in vals]
    den = max(d for _, d in rat)
    return [n * (den // d) for n, d in rat]


def _orient_exact(ax, ay, bx, by, cx, cy):
    ax, ay, bx, by, cx, cy = _ints(ax, ay, bx, by, cx, cy)
    d = (bx - ax) * (cy - ay) - (by - ay) * (cx - ax)
    return (d > 0) - (d < 0)


def orient(ax, ay, bx, by, cx, cy):
    """Sign of the signed area of (a, b, c): +1 counter-clockwise, -1 clockwise, 0 collinear."""
    l = (bx - ax) * (cy - ay)
    r = (by - ay) * (cx - ax)
    d = l - r
    if abs(d) > _ORIENT_BOUND * (abs(l) + abs(r)):
        return 1 if d > 0 else -1
    return _orient_exact(ax, ay, bx, by, cx, cy)


def _incircle_exact(ax, ay, bx, by, cx, cy, dx, dy):
    ax, ay, bx, by, cx, cy, dx, dy = _ints(ax, ay, bx, by, cx, cy, dx, dy)
    adx, ady, bdx, bdy, cdx, cdy = ax - dx, ay - dy, bx - dx, by - dy, cx - dx, cy - dy
    d = ((adx * adx + ady * ady) * (bdx * cdy - cdx * bdy) + (bdx * bdx + bdy * bdy) * (cdx * ady - adx * cdy) +
         (cdx * cdx + cdy * cdy) * (adx * bdy - bdx * ady))
    return (d > 0) - (d < 0)


def incircle(ax, ay, bx, by, cx, cy, dx, dy):
    """+1 if d is strictly inside the circle through the counter-clockwise a, b, c; 0 on it."""
    adx, ady, bdx, bdy, cdx, cdy = ax - dx, ay - dy, bx - dx, by - dy, cx - dx, cy - dy
    alift, blift, clift = adx * adx + ady * ady, bdx * bdx + bdy * bdy, cdx * cdx + cdy * cdy
    bc, ca, ab = bdx * cdy - cdx * bdy, cdx * ady - adx * cdy, adx * bdy - bdx * ady
    d = alift * bc + blift * ca + clift * ab
    perm = (alift * (abs(bdx * cdy) + abs(cdx * bdy)) + blift * (abs(cdx * ady) + abs(adx * cdy)) +
            clift * (abs(adx * bdy) + abs(bdx * ady)))
    if abs(d) > _INCIRCLE_BOUND * perm:
        return 1 if d > 0 else -1
    return _incircle_exact(ax, ay, bx, by, cx, cy, dx, dy)


class _Mesher:
    """Delaunay triangulation under refinement.  Triangle t has counter-clockwise vertices
    V[t] and neighbours N[t], N[t][k] across the edge opposite V[t][k] (-1: none)."""

    def __init__(self, pts, nsuper_scale=50.0):
        pts = np.asarray(pts, float)
        lo, hi = pts.min(axis=0), pts.max(axis=0)
        c = 0.5 * (lo + hi)
        m = max(hi[0] - lo[0], hi[1] - lo[1], 1e-300) * nsuper_scale
        self.X = [c[0] - 3 * m, c[0] + 3 * m, c[0]]
        self.Y = [c[1] - 2 * m, c[1] - 2 * m, c[1] + 3 * m]
        self.V = [[0, 1, 2]]
        self.N = [[-1, -1, -1]]
        self.alive = [True]
        self.inside = [False]
        self.vt = [0, 0, 0]  # an alive triangle at each vertex
        self.seg = {}        # subsegments (low, high) -> marker
        self.last = 0

    # ---- geometry -------------------------------------------------------------------------
    def _incircle_t(self, t, px, py):
        a, b, c = self.V[t]
        X, Y = self.X, self.Y
        return incircle(X[a], Y[a], X[b], Y[b], X[c], Y[c], px, py)

    def locate(self, px, py, start=None):
        """A triangle containing (px, py) (on its boundary allowed), by a visibility walk."""
        t = self.last if start is None or not self.alive[start] else start
        if not self.alive[t]:
            t = next(i for i in range(len(self.V) - 1, -1, -1) if self.alive[i])
        X, Y, V, N = self.X, self.Y, self.V, self.N
        k0 = 0
        for _ in range(4 * len(V) + 16):
            v = V[t]
            moved = False
            for j in range(3):
                k = (k0 + j) % 3
                a, b = v[(k + 1) % 3], v[(k + 2) % 3]
                if orient(X[a], Y[a], X[b], Y[b], px, py) < 0:
                    t = N[t][k]
                    if t < 0:
                        raise RuntimeError("point outside the triangulation")
                    moved = True
                    break
            if not moved:
                return t
            k0 = (k0 + 1) % 3
        raise RuntimeError("point location did not terminate")

    def edge_tris(self, a, b):
        """(t, k) with V[t][k] == a and V[t][(k+1)%3] == b if the directed edge a->b exists."""
        t0 = self.vt[a]
        t = t0
        V, N = self.V, self.N
        for _ in range(1000):
            v = V[t]
            i = v.index(a)
            if v[(i + 1) % 3] == b:
                return t, i
            t = N[t][(i + 1) % 3]  # across edge (a, v[i+2]): the next triangle around a
            if t < 0 or t == t0:
                return None
        return None

    def has_edge(self, a, b):
        return self.edge_tris(a, b) is not None or self.edge_tris(b, a) is not None

    def encroached(self, a, b):
        """Subsegment (a, b) is missing, or a vertex lies strictly inside its diametral circle."""
        X, Y = self.X, self.Y
        found = False
        for p, q in ((a, b), (b, a)):
            r = self.edge_tris(p, q)
            if r is None:
                continue
            found = True
            t, i = r
            c = self.V[t][(i + 2) % 3]
            if c > 2 and (X[c] - X[a]) * (X[c] - X[b]) + (Y[c] - Y[a]) * (Y[c] - Y[b]) < 0:
                return True
        return not found

    # ---- insertion ---------------------------------------------------------------------------
    def cavity(self, px, py, t0):
        """Triangles whose circumcircle strictly contains p, grown from t0."""
        cav = [t0]
        seen = {t0}
        i = 0
        N = self.N
        while i < len(cav):
            t = cav[i]
            i += 1
            for n in N[t]:
                if n >= 0 and n not in seen:
                    seen.add(n)
                    if self._incircle_t(n, px, py) > 0:
                        cav.append(n)
        return cav, set(cav)

    def cavity_segments(self, px, py, cav, cset):
        """Subsegments p would destroy or encroach: (internal to the cavity, on its boundary
        with p inside their diametral circle)."""
        X, Y, V, N, seg = self.X, self.Y, self.V, self.N, self.seg
        hit = []
        for t in cav:
            v = V[t]
            for k in range(3):
                a, b = v[(k + 1) % 3], v[(k + 2) % 3]
                key = (a, b) if a < b else (b, a)
                if key not in seg:
                    continue
                n = N[t][k]
                if n in cset:
                    hit.append(key)
                elif (px - X[a]) * (px - X[b]) + (py - Y[a]) * (py - Y[b]) < 0:
                    hit.append(key)
        return list(dict.fromkeys(hit))

    def insert(self, px, py, cav, cset, inherit=True):
        """Bowyer-Watson: replace the cavity by the fan of p.  Returns (vertex, new triangles,
        whether a subsegment was swallowed)."""
        X, Y, V, N = self.X, self.Y, self.V, self.N
        p = len(X)
        X.append(px)
        Y.append(py)
        self.vt.append(-1)
        by_u, by_v, new = {}, {}, []
        swallowed = False
        for t in cav:
            v = V[t]
            for k in range(3):
                n = N[t][k]
                a, b = v[(k + 1) % 3], v[(k + 2) % 3]
                if n in cset:
                    if ((a, b) if a < b else (b, a)) in self.seg:
                        swallowed = True
                    continue
                nt = len(V)
                V.append([p, a, b])
                N.append([n, -1, -1])
                self.alive.append(True)
                self.inside.append(self.inside[t] if inherit else False)
                if n >= 0:
                    N[n][N[n].index(t)] = nt
                by_u[a] = nt
                by_v[b] = nt
                new.append(nt)
        for t in cav:
            self.alive[t] = False
        for nt in new:
            _, a, b = V[nt]
            N[nt][1] = by_u[b]   # across (b, p)
            N[nt][2] = by_v[a]   # across (p, a)
            self.vt[a] = nt
            self.vt[b] = nt
        self.vt[p] = new[0]
        self.last = new[0]
        return p, new, swallowed

    def insert_point(self, px, py, start=None):
        t0 = self.locate(px, py, start)
        v = self.V[t0]
        for q in v:
            if self.X[q] == px and self.Y[q] == py:
                return q, [], False
        cav, cset = self.cavity(px, py, t0)
        return self.insert(px, py, cav, cset)

    # ---- regions ---------------------------------------------------------------------------
    def label(self, holes):
        """Inside = not reachable from the super triangle's corners or a hole seed without
        crossing a subsegment."""
        V, N, alive, seg = self.V, self.N, self.alive, self.seg
        ext = [False] * len(V)
        stack = [t for t in range(len(V)) if alive[t] and (V[t][0] < 3 or V[t][1] < 3 or V[t][2] < 3)]
        for hx, hy in holes:
            stack.append(self.locate(hx, hy))
        for t in stack:
            ext[t] = True
        while stack:
            t = stack.pop()
            v = V[t]
            for k in range(3):
                n = N[t][k]
                if n < 0 or ext[n]:
                    continue
                a, b = v[(k + 1) % 3], v[(k + 2) % 3]
                if ((a, b) if a < b else (b, a)) in seg:
                    continue
                ext[n] = True
                stack.append(n)
        self.inside = [alive[t] and not ext[t] for t in range(len(V))]


def _split_segment(M, key, enc, fixed):
    a, b = key
    mark = M.seg.pop(key)
    mx, my = 0.5 * (M.X[a] + M.X[b]), 0.5 * (M.Y[a] + M.Y[b])
    r = M.edge_tris(a, b) or M.edge_tris(b, a)
    start = r[0] if r else None
    t0 = M.locate(mx, my, start)
    cav, cset = M.cavity(mx, my, t0)
    hit = M.cavity_segments(mx, my, cav, cset)
    p, new, swallowed = M.insert(mx, my, cav, cset)
    for s in ((a, p), (p, b)):
        M.seg[(min(s), max(s))] = mark
    # the halves, and any subsegment the midpoint encroaches or swallowed, are checked again
    for s in [(min(a, p), max(a, p)), (min(p, b), max(p, b))] + hit:
        if s in M.seg and M.seg[s] not in fixed:
            enc.append(s)
    return new, swallowed


def triangulate(points, segments, markers, holes, max_area, min_angle=30.0, fixed_markers=(), max_vertices=None):
    """Conforming Delaunay quality triangulation of the graph (0-based ``segments`` (ns, 2)).
    Returns (nodes (n, 2), counter-clockwise triangles (m, 3), 0-based)."""
    pts = np.asarray(points, float).reshape(-1, 2)
    segs = np.asarray(segments, np.int64).reshape(-1, 2)
    markers = list(markers) if len(markers) else [1] * len(segs)
    fixed = set(fixed_markers)
    M = _Mesher(pts)
    ids = []
    for x, y in pts:
        q, _, _ = M.insert_point(float(x), float(y))
        ids.append(q)
    for (i, j), mk in zip(segs, markers):
        a, b = ids[i], ids[j]
        if a != b:
            M.seg[(min(a, b), max(a, b))] = mk
    # recover and unencroach the segments
    enc = [s for s in M.seg if M.seg[s] not in fixed]
    cap = max_vertices or (200000 + 50 * len(pts))
    while enc:
        s = enc.pop()
        if s in M.seg and M.encroached(*s):
            _split_segment(M, s, enc, fixed)
            if len(M.X) > cap:
                raise RuntimeError("meshsub: segment recovery did not terminate")
    for (a, b) in M.seg:
        if not M.has_edge(a, b):
            raise RuntimeError("meshsub: a segment that may not be split is missing from the triangulation")
    hole_pts = [tuple(map(float, h)) for h in np.asarray(holes, float).reshape(-1, 2)]
    M.label(hole_pts)
    # quality refinement
    bound = 1.0 / (2.0 * math.sin(math.radians(min_angle)))
    X, Y, V = M.X, M.Y, M.V

    def bad(t):
        a, b, c = V[t]
        ax, ay, bx, by, cx, cy = X[a], Y[a], X[b], Y[b], X[c], Y[c]
        ar = 0.5 * ((bx - ax) * (cy - ay) - (by - ay) * (cx - ax))
        if ar > max_area:
            return True
        la = (bx - cx) ** 2 + (by - cy) ** 2
        lb = (ax - cx) ** 2 + (ay - cy) ** 2
        lc = (ax - bx) ** 2 + (ay - by) ** 2
        # circumradius^2 = la lb lc / (16 ar^2); ratio to the shortest edge
        return la * lb * lc / (16.0 * ar * ar * min(la, lb, lc)) > bound * bound

    queue = [t for t in range(len(V)) if M.inside[t]]
    forced, done_force = [], set()
    dirty = False
    gave_up = set()
    qi = 0
    while True:
        if enc or forced:
            # segments a rejected circumcentre would encroach are split unconditionally; a
            # split that swallowed another subsegment leaves the regions to be labelled again
            # once every subsegment is back in the triangulation
            s = forced.pop() if forced else enc.pop()
            if s in M.seg and (s in done_force or M.encroached(*s)):
                new, swallowed = _split_segment(M, s, enc, fixed)
                queue.extend(new)
                dirty = dirty or swallowed
            done_force.discard(s)
            continue
        if dirty:
            if any(not M.has_edge(a, b) for (a, b) in M.seg):
                raise RuntimeError("meshsub: a segment that may not be split left the triangulation")
            M.label(hole_pts)
            dirty = False
        if qi >= len(queue):
            break
        t = queue[qi]
        qi += 1
        if not M.alive[t] or not M.inside[t] or t in gave_up or not bad(t):
            continue
        a, b, c = V[t]
        ax, ay, bx, by, cx, cy = X[a], Y[a], X[b], Y[b], X[c], Y[c]
        d = 2.0 * ((bx - ax) * (cy - ay) - (by - ay) * (cx - ax))
        b2, c2 = (bx - ax) ** 2 + (by - ay) ** 2, (cx - ax) ** 2 + (cy - ay) ** 2
        ux = ax + ((cy - ay) * b2 - (by - ay) * c2) / d
        uy = ay + ((bx - ax) * c2 - (cx - ax) * b2) / d
        try:
            t0 = M.locate(ux, uy, t)
        except RuntimeError:
            gave_up.add(t)
            continue
        if any(X[q] == ux and Y[q] == uy for q in V[t0]):
            gave_up.add(t)
            continue
        cav, cset = M.cavity(ux, uy, t0)
        hit = M.cavity_segments(ux, uy, cav, cset)
        if hit:
            split = [s for s in hit if M.seg[s] not in fixed]
            if split:
                forced.extend(split)
                done_force.update(split)
                queue.append(t)  # looked at again once the segments are split
            else:
                gave_up.add(t)
            continue
        if not all(M.inside[x] for x in cav):
            gave_up.add(t)
            continue
        _, new, _ = M.insert(ux, uy, cav, cset)
        queue.extend(new)
        if len(X) > cap:
            raise RuntimeError("meshsub: refinement did not terminate")
    tris = [V[t] for t in range(len(V)) if M.alive[t] and M.inside[t]]
    used = sorted({v for t in tris for v in t})
    if any(v < 3 for v in used):
        raise RuntimeError("meshsub: the graph does not enclose its region")
    renum = {v: i for i, v in enumerate(used)}
    nodes = np.array([[X[v], Y[v]] for v in used], float)
    tri = np.array([[renum[v] for v in t] for t in tris], np.int64)
    return nodes, tri


def meshsub(*, points, seglist, area, ntri, segmarkers=(), holes=None, min_angle=30.0, fixed_markers=()):
    """``meshsub`` (``Meshsub.jl:43-113``): ``points`` (2, np), 1-based ``seglist`` (2, ns),
    ``holes`` (2, nh) seed points, maximum triangle ``area``.  The area bound is rescaled by
    (ntri_got / ntri)^(1/3) until the count is within 10 % of ``ntri`` (at most 14 meshes).
    Returns the sheet (``RWGSheet``) with nodes, edges, faces and zero face resistance."""
    from .elements import _sheet_from_triangles
    pts = np.asarray(points, float)
    if pts.ndim != 2 or pts.shape[0] != 2:
        raise ValueError("points first dimension must be 2")
    seg = np.asarray(seglist, np.int64)
    if seg.ndim != 2 or seg.shape[0] != 2:
        raise ValueError("seglist first dimension must be 2")
    if len(segmarkers) and len(segmarkers) != seg.shape[1]:
        raise ValueError("wrong length(segmarkers)")
    hl = np.zeros((0, 2)) if holes is None or np.size(holes) == 0 else np.asarray(holes, float).reshape(2, -1).T
    a = float(area)
    nodes = tri = None
    for _ in range(14):
        for q in (min_angle, 25.0, 20.7):  # a weaker angle bound if the refinement runs away
            try:
                nodes, tri = triangulate(pts.T, seg.T - 1, list(segmarkers), hl, a, min(q, min_angle), fixed_markers)
                break
            except RuntimeError:
                if q == 20.7:
                    raise
        got = len(tri)
        if 0.9 * ntri <= got <= 1.1 * ntri:
            break
        a *= (got / ntri) ** (1.0 / 3.0)
    sh = _sheet_from_triangles(nodes, tri)
    sh.fr = np.zeros(sh.nface)
    return sh

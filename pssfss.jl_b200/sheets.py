"""Triangulated sheet type and structured-mesh builders.

Mirrors PSSFSS.jl ``src/Sheets.jl``: ``RWGSheet`` (``:19-58``), ``rotate!`` (``:177``),
``translate!`` (``:198``), ``combine`` (``:234-389``) and ``recttri`` (``:398-480``).
Index arrays keep the reference's conventions so that golden topology values from its
tests compare directly: ``e1``/``e2`` are length-``nedge`` int64 arrays of 1-based node
numbers, ``fv``/``fe`` are ``(3, nface)`` int64 arrays of 1-based node/edge numbers
(column ``i`` is face ``i``; ``fe[k, i]`` is the edge opposite vertex ``fv[k, i]``), and
``rho`` is an ``(nnode, 2)`` float64 array of node coordinates in sheet units.
"""
import math

import numpy as np

from .units import mm


def s1s2_to_b1b2(s1, s2):
    """Reciprocal lattice vectors from direct ones (``Elements.jl:27-36``)."""
    z = s1[0] * s2[1] - s1[1] * s2[0]
    fact = (2 * math.pi) / math.sqrt(0.0 + 0.0 + z * z)
    b1 = np.array([fact * s2[1], fact * (0.0 * 0.0 - s2[0] * 1.0)])
    b2 = np.array([fact * (0.0 * 0.0 - 1.0 * s1[1]), fact * (1.0 * s1[0] - 0.0 * 0.0)])
    return b1, b2


class RWGSheet:
    """A periodic triangulated sheet (``Sheets.jl:19-58``).

    The J/K face-pair integral cache of the reference lives on the device inside the
    CUDA library; only its key ``(psi1, psi2, u)`` semantics are kept.
    """

    def __init__(self):
        self.style = ""
        self.units = mm
        self.s1 = np.zeros(2)
        self.s2 = np.zeros(2)
        self.beta1 = np.zeros(2)
        self.beta2 = np.zeros(2)
        self.dx = 0.0
        self.dy = 0.0
        self.rot = 0.0
        self.rho = np.zeros((0, 2))
        self.e1 = np.zeros(0, np.int64)
        self.e2 = np.zeros(0, np.int64)
        self.fv = np.zeros((3, 0), np.int64)
        self.fe = np.zeros((3, 0), np.int64)
        self.fr = np.zeros(0)
        self.psi1 = 0.0
        self.psi2 = 0.0
        self.u = 0.0
        self.cls = " "
        self.info = ""
        self.xi_eta_check = True
        self.fufp = False

    @property
    def nface(self):
        return self.fv.shape[1]

    @property
    def nedge(self):
        return len(self.e1)

    @property
    def nnode(self):
        return self.rho.shape[0]

    def __repr__(self):
        return (f"RWGSheet: style={self.style}, class={self.cls}, {self.nnode} nodes, "
                f"{self.nedge} edges, {self.nface} faces")


def rotate(sh, rot):
    """Rotate a sheet counter-clockwise by ``rot`` degrees (``Sheets.jl:177-190``)."""
    if rot == 0:
        return sh
    s, c = _sincosd(rot)
    R = np.array([[c, -s], [s, c]])

    def rm(v):
        return np.array([R[0, 0] * v[0] + R[0, 1] * v[1], R[1, 0] * v[0] + R[1, 1] * v[1]])

    sh.s1 = rm(sh.s1)
    sh.s2 = rm(sh.s2)
    sh.beta1 = rm(sh.beta1)
    sh.beta2 = rm(sh.beta2)
    sh.rho = np.array([rm(p) for p in sh.rho]).reshape(-1, 2)
    sh.rot = rot
    return sh


def _sincosd(deg):
    """Degree sine/cosine with exact values at multiples of 90 (Julia ``sincosd``)."""
    r = math.fmod(deg, 360.0)
    for k, (s, c) in ((0, (0.0, 1.0)), (90, (1.0, 0.0)), (180, (0.0, -1.0)), (270, (-1.0, 0.0))):
        if r == k or r == k - 360:
            return s, c
    x = math.radians(deg)
    return math.sin(x), math.cos(x)


def translate(sh, dx, dy):
    """Translate a sheet by (dx, dy) (``Sheets.jl:198-205``)."""
    if dx == 0 and dy == 0:
        return sh
    sh.rho = sh.rho + np.array([dx, dy])[None, :]
    return sh


def recttri(rhobl, rhotr, nx, ny):
    """Structured triangulation of a rectangle (``Sheets.jl:398-480``)."""
    nodecount = (nx + 1) * (ny + 1)
    edgecount = 3 * nx * ny + nx + ny
    facecount = 2 * nx * ny
    sh = RWGSheet()
    rhobl = np.asarray(rhobl, float)
    rhotr = np.asarray(rhotr, float)
    drho = (rhotr - rhobl) / np.array([nx, ny], float)
    rho = np.zeros((nodecount, 2))
    n = 0
    for j in range(ny + 1):
        yj = j * drho[1]
        for i in range(nx + 1):
            rho[n, 0] = rhobl[0] + i * drho[0]
            rho[n, 1] = rhobl[1] + yj
            n += 1
    sh.rho = rho
    e1 = np.zeros(edgecount, np.int64)
    e2 = np.zeros(edgecount, np.int64)
    e = 0
    for j in range(ny + 1):                       # horizontal edges
        kadd = j * (nx + 1)
        for i in range(1, nx + 1):
            e1[e] = i + kadd
            e2[e] = e1[e] + 1
            e += 1
    for j in range(1, ny + 1):                    # vertical edges
        kadd = (j - 1) * (nx + 1) + 1
        for i in range(0, nx + 1):
            e1[e] = i + kadd
            e2[e] = e1[e] + (nx + 1)
            e += 1
    for j in range(1, ny + 1):                    # diagonal edges
        kadd1 = (j - 1) * (nx + 1)
        kadd2 = 1 + j * (nx + 1)
        for i in range(1, nx + 1):
            e1[e] = i + kadd1
            e2[e] = i + kadd2
            e += 1
    sh.e1, sh.e2 = e1, e2
    fv = np.zeros((3, facecount), np.int64)
    fe = np.zeros((3, facecount), np.int64)
    nhe = nx * ny + nx
    nve = nx * ny + ny
    f = 0
    for j in range(1, ny + 1):
        nadd1 = (j - 1) * (nx + 1)
        nadd2 = 1 + j * (nx + 1)
        for i in range(1, nx + 1):
            fv[0, f] = i + nadd1            # lower left
            fv[1, f] = i + nadd2            # upper right
            fv[2, f] = i + nadd2 - 1        # upper left
            fe[0, f] = i + j * nx           # upper edge
            fe[1, f] = i + nhe + nadd1      # left edge
            fe[2, f] = i + nhe + nve + (j - 1) * nx  # diagonal edge
            f += 1
            fv[0, f] = fv[0, f - 1]
            fv[1, f] = 1 + fv[0, f - 1]
            fv[2, f] = fv[1, f - 1]
            fe[0, f] = 1 + fe[1, f - 1]
            fe[1, f] = fe[2, f - 1]
            fe[2, f] = fe[0, f - 1] - nx
            f += 1
    sh.fv, sh.fe = fv, fe
    return sh


def _renumber_after_removal(vals, removed):
    """Decrement every value by the number of ``removed`` thresholds (sorted, distinct) below
    it: the effect of the reference's descending ``x[x .> r] .-= 1`` loops on values that are
    none of the thresholds."""
    return vals - np.searchsorted(removed, vals, side="left")


def combine(sh1, sh2, dup_coor, dup_coor_value):
    """Merge two triangulations that may share a line of nodes and edges
    (``Sheets.jl:234-389``).

    The reference's rules are kept: a node of ``sh2`` within ``tol`` of the line pairs with
    the first node of ``sh1`` within ``tol`` of it, a shared edge with the first ``sh1`` edge
    joining the paired nodes, and the shared nodes and edges of ``sh2`` are dropped with the
    later indices closed up.  The searches and renumberings are array operations."""
    if sh1.units != sh2.units:
        raise ValueError("Inconsistent units for sh1 and sh2")
    nv1, ne1, nf1 = sh1.nnode, sh1.nedge, sh1.nface
    vcen1 = vcen2 = ecen1 = ecen2 = np.zeros(0, np.int64)
    if dup_coor != " ":
        d = sh1.rho[sh1.e1[0] - 1] - sh1.rho[sh1.e2[0] - 1]
        tol = 0.5e-4 * math.sqrt(d[0] * d[0] + d[1] * d[1])
        ax = 0 if dup_coor == "x" else 1
        cand2 = np.flatnonzero(np.abs(sh2.rho[:, ax] - dup_coor_value) < tol)
        # a matching sh1 node lies within 2 tol of the line; a wider band keeps rounding out
        near1 = np.flatnonzero(np.abs(sh1.rho[:, ax] - dup_coor_value) < 3 * tol)
        v1, v2 = [], []
        if len(cand2) and len(near1):
            dx = sh1.rho[near1, 0][None, :] - sh2.rho[cand2, 0][:, None]
            dy = sh1.rho[near1, 1][None, :] - sh2.rho[cand2, 1][:, None]
            hit = np.sqrt(dx * dx + dy * dy) < tol
            has = hit.any(axis=1)
            first = near1[np.argmax(hit, axis=1)]  # near1 ascending: the first sh1 match
            v2 = cand2[has] + 1
            v1 = first[has] + 1
        vcen2 = np.asarray(v2, np.int64)
        vcen1 = np.asarray(v1, np.int64)
        if len(vcen2):
            # sh2 edges with both ends shared, in sh2 order, and the first sh1 edge on the
            # same (unordered) node pair
            vpair = np.zeros(sh2.nnode + 1, np.int64)
            vpair[vcen2] = vcen1
            a2, b2 = np.asarray(sh2.e1, np.int64), np.asarray(sh2.e2, np.int64)
            both = (vpair[a2] > 0) & (vpair[b2] > 0)
            ecen2 = np.flatnonzero(both) + 1
            va, vb = vpair[a2[both]], vpair[b2[both]]
            big = np.int64(nv1 + 1)
            a1, b1 = np.asarray(sh1.e1, np.int64), np.asarray(sh1.e2, np.int64)
            key1 = np.minimum(a1, b1) * big + np.maximum(a1, b1)
            ukey, ufirst = np.unique(key1, return_index=True)
            want = np.minimum(va, vb) * big + np.maximum(va, vb)
            pos = np.searchsorted(ukey, want)
            ok = (pos < len(ukey)) & (ukey[np.minimum(pos, len(ukey) - 1)] == want)
            if not ok.all():
                raise RuntimeError("Unable to find matching duplicate edge in combine_sheet")
            ecen1 = ufirst[pos].astype(np.int64) + 1
    Nvcen, Necen = len(vcen2), len(ecen2)
    sh3 = RWGSheet()
    sh3.units = sh1.units
    voffset = nv1
    # sh2 node index (1-based) -> merged index before the shared nodes are closed up
    vmap2 = np.arange(sh2.nnode + 1, dtype=np.int64) + voffset
    vmap2[vcen2] = vcen1
    # vertices
    keepv = np.ones(sh2.nnode, bool)
    keepv[vcen2 - 1] = False
    sh3.rho = np.vstack([sh1.rho, sh2.rho[keepv]])
    # edges
    removed_v = voffset + vcen2  # ascending
    keepe = np.ones(sh2.nedge, bool)
    keepe[ecen2 - 1] = False
    e1 = np.concatenate([np.asarray(sh1.e1, np.int64),
                         _renumber_after_removal(vmap2[np.asarray(sh2.e1, np.int64)[keepe]], removed_v)])
    e2 = np.concatenate([np.asarray(sh1.e2, np.int64),
                         _renumber_after_removal(vmap2[np.asarray(sh2.e2, np.int64)[keepe]], removed_v)])
    sh3.e1, sh3.e2 = e1, e2
    # faces / vertices
    fv = np.zeros((3, nf1 + sh2.nface), np.int64)
    fv[:, :nf1] = sh1.fv
    fv[:, nf1:] = _renumber_after_removal(vmap2[np.asarray(sh2.fv, np.int64)], removed_v)
    sh3.fv = fv
    # faces / edges
    eoffset = ne1
    emap2 = np.arange(sh2.nedge + 1, dtype=np.int64) + eoffset
    emap2[ecen2] = ecen1
    fe = np.zeros((3, nf1 + sh2.nface), np.int64)
    fe[:, :nf1] = sh1.fe
    fe[:, nf1:] = _renumber_after_removal(emap2[np.asarray(sh2.fe, np.int64)], eoffset + ecen2)
    sh3.fe = fe
    assert Necen == len(ecen1) and Nvcen == len(vcen1)
    return sh3


def write_sheet_data(filename, sheet):
    """Save a sheet's geometry for ``read_sheet_data`` (``Sheets.jl:113-117``; the reference
    writes JLD2, here a pickled ``{"sheet": sheet}``)."""
    import pickle
    with open(filename, "wb") as f:
        pickle.dump({"sheet": sheet}, f)


def read_sheet_data(filename):
    """The sheet saved by ``write_sheet_data`` (``Sheets.jl:98-106``)."""
    import pickle
    with open(filename, "rb") as f:
        dat = pickle.load(f)
    if not isinstance(dat, dict) or "sheet" not in dat:
        raise ValueError(f"{filename} does not contain sheet data")
    return dat["sheet"]

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


def combine(sh1, sh2, dup_coor, dup_coor_value):
    """Merge two triangulations that may share a line of nodes and edges
    (``Sheets.jl:234-389``)."""
    if sh1.units != sh2.units:
        raise ValueError("Inconsistent units for sh1 and sh2")
    nv1, ne1, nf1 = sh1.nnode, sh1.nedge, sh1.nface
    vcen1, vcen2 = [], []
    ecen1, ecen2 = [], []
    if dup_coor != " ":
        d = sh1.rho[sh1.e1[0] - 1] - sh1.rho[sh1.e2[0] - 1]
        tol = 0.5e-4 * math.sqrt(d[0] * d[0] + d[1] * d[1])
        for i in range(sh2.nnode):
            test = sh2.rho[i, 0] if dup_coor == "x" else sh2.rho[i, 1]
            if abs(test - dup_coor_value) < tol:
                n1match = 0
                for n1 in range(nv1):
                    dd = sh1.rho[n1] - sh2.rho[i]
                    if math.sqrt(dd[0] * dd[0] + dd[1] * dd[1]) < tol:
                        n1match = n1 + 1
                        break
                if n1match != 0:
                    vcen2.append(i + 1)
                    vcen1.append(n1match)
        vset2 = {v: k for k, v in enumerate(vcen2)}
        for i in range(sh2.nedge):
            a, b = int(sh2.e1[i]), int(sh2.e2[i])
            if a in vset2 and b in vset2:
                ecen2.append(i + 1)
                va, vb = vcen1[vset2[a]], vcen1[vset2[b]]
                found = 0
                for j1 in range(ne1):
                    if (sh1.e1[j1] == va and sh1.e2[j1] == vb) or (sh1.e2[j1] == va and sh1.e1[j1] == vb):
                        found = j1 + 1
                        break
                if found == 0:
                    raise RuntimeError("Unable to find matching duplicate edge in combine_sheet")
                ecen1.append(found)
    Nvcen, Necen = len(vcen2), len(ecen2)
    sh3 = RWGSheet()
    sh3.units = sh1.units
    # vertices
    if dup_coor == " ":
        sh3.rho = np.vstack([sh1.rho, sh2.rho])
    else:
        keep = [i for i in range(sh2.nnode) if (i + 1) not in vcen2]
        sh3.rho = np.vstack([sh1.rho, sh2.rho[keep]])
    # edges
    e1 = np.zeros(ne1 + sh2.nedge - Necen, np.int64)
    e2 = np.zeros_like(e1)
    e1[:ne1] = sh1.e1
    e2[:ne1] = sh1.e2
    voffset = nv1
    if dup_coor == " ":
        e1[ne1:] = sh2.e1 + voffset
        e2[ne1:] = sh2.e2 + voffset
    else:
        eoffset = ne1
        ecen2_set = set(ecen2)
        vmap = {v: vcen1[k] for k, v in enumerate(vcen2)}
        for i in range(sh2.nedge):
            if (i + 1) in ecen2_set:
                eoffset -= 1
                continue
            a, b = int(sh2.e1[i]), int(sh2.e2[i])
            e1[i + eoffset] = vmap[a] if a in vmap else a + voffset
            e2[i + eoffset] = vmap[b] if b in vmap else b + voffset
        for i in range(Nvcen - 1, -1, -1):
            thr = nv1 + vcen2[i]
            e1[e1 > thr] -= 1
            e2[e2 > thr] -= 1
    sh3.e1, sh3.e2 = e1, e2
    # faces / vertices
    fv = np.zeros((3, nf1 + sh2.nface), np.int64)
    fv[:, :nf1] = sh1.fv
    fv[:, nf1:] = sh2.fv + voffset
    for n2 in range(Nvcen):
        fv[fv == vcen2[n2] + voffset] = vcen1[n2]
    for i in range(Nvcen - 1, -1, -1):
        fv[fv > voffset + vcen2[i]] -= 1
    sh3.fv = fv
    # faces / edges
    eoffset = ne1
    fe = np.zeros((3, nf1 + sh2.nface), np.int64)
    fe[:, :nf1] = sh1.fe
    fe[:, nf1:] = sh2.fe + eoffset
    if dup_coor != " ":
        for n2 in range(len(ecen2)):
            fe[fe == ecen2[n2] + eoffset] = ecen1[n2]
        for i in range(len(ecen2) - 1, -1, -1):
            fe[fe > eoffset + ecen2[i]] -= 1
    sh3.fe = fe
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

"""TEST INFRASTRUCTURE ONLY -- independent restatement of ``setup_rwg`` (PSSFSS.jl v0.1.4,
src/RWG.jl:90-324): the RWG basis functions of a triangulated sheet and its unique face-pair
classes.

Nothing here imports the package under test; a sheet is read as plain data (``rho``
nnode x 2, ``fv``/``fe`` 3 x nface and ``e1``/``e2`` with 1-based values, ``beta1``,
``beta2``, ``xi_eta_check``, ``fufp``).  The result carries the fields the oracle's fill
reads: ``bfe``, ``bff`` (2 x nbf), ``ebf``, ``eci`` (nedge), ``ufpm`` (nface x nface, match
face fastest), ``ufp_rep`` (1-based column-major index of each class's first pair), ``nufp``.

* interior basis functions: every pair of faces fp < fm sharing an edge, ordered as the
  reference's loops meet them (fp, then fm, then the edge's slot in fp, then in fm);
* boundary basis functions (xi_eta_check): edges on eta = 0 paired with the eta = 1 edge of
  the same xi extent, then xi = 0 with xi = 1 by eta extent (tolerance 1e-5), each joining the
  first face holding either edge;
* unique face pairs (fufp): the pairs (match m, source n) whose 6-vectors (centroid of m minus
  each vertex of n) lie within r = 1e-6 |c1 - c2| of the first member, numbered in
  column-major order of first appearance (the KD-tree range search of RWG.jl:287-319, here by
  exact grouping of the vectors rounded to a grid of r, every member then checked against its
  class's first vector at radius r).
"""
import math

import numpy as np


class Topology:
    def __init__(self, bfe, bff, ebf, eci, ufpm, ufp_rep, nufp):
        self.bfe, self.bff, self.ebf, self.eci = bfe, bff, ebf, eci
        self.ufpm, self.ufp_rep, self.nufp = ufpm, ufp_rep, nufp

    @property
    def nbf(self):
        return self.bfe.shape[1]


def _xi_eta(sheet):
    """Per edge (xi, eta) of its initial and terminal node (get_ie_ξη, RWG.jl:388-398)."""
    rho = np.asarray(sheet.rho, float)
    b1, b2 = np.asarray(sheet.beta1, float), np.asarray(sheet.beta2, float)
    p0 = rho[np.asarray(sheet.e1, np.int64) - 1]
    p1 = rho[np.asarray(sheet.e2, np.int64) - 1]
    tp = 2 * math.pi
    return ((b1[0] * p0[:, 0] + b1[1] * p0[:, 1]) / tp, (b1[0] * p1[:, 0] + b1[1] * p1[:, 1]) / tp,
            (b2[0] * p0[:, 0] + b2[1] * p0[:, 1]) / tp, (b2[0] * p1[:, 0] + b2[1] * p1[:, 1]) / tp)


def setup(sheet):
    tol = 1e-5
    fe = np.asarray(sheet.fe, np.int64)
    nface, nedge = fe.shape[1], len(sheet.e1)
    # interior basis functions
    face = np.repeat(np.arange(1, nface + 1), 3)
    slot = np.tile(np.arange(3), nface)
    edge = fe.T.ravel()
    order = np.lexsort((slot, face, edge))
    e_s, f_s, k_s = edge[order], face[order], slot[order]
    starts = np.flatnonzero(np.r_[True, e_s[1:] != e_s[:-1]])
    ends = np.r_[starts[1:], len(e_s)]
    rows = []
    for a, b in zip(starts, ends):
        for i in range(a, b):
            for j in range(i + 1, b):
                if f_s[i] < f_s[j]:
                    rows.append((int(f_s[i]), int(f_s[j]), int(k_s[i]), int(k_s[j]), int(e_s[i])))
    rows.sort()
    interior = np.array(rows, np.int64).reshape(-1, 5)
    # unit-cell boundary edges
    eci = np.zeros(nedge, np.int64)
    lists = {1: [], 2: [], 3: [], 4: []}
    if sheet.xi_eta_check:
        xi0, xi1, et0, et1 = _xi_eta(sheet)
        for g in range(nedge):
            if abs(xi0[g]) < tol and abs(xi1[g]) < tol:
                code = 1
            elif abs(xi0[g] - 1) < tol and abs(xi1[g] - 1) < tol:
                code = 2
            elif abs(et0[g]) < tol and abs(et1[g]) < tol:
                code = 3
            elif abs(et0[g] - 1) < tol and abs(et1[g] - 1) < tol:
                code = 4
            else:
                continue
            eci[g] = code
            lists[code].append(g + 1)
    if len(lists[1]) != len(lists[2]) or len(lists[3]) != len(lists[4]):
        raise ValueError("inconsistent numbers of opposite unit-cell boundary edges")
    first_face = np.zeros(nedge + 1, np.int64)
    for f in range(nface, 0, -1):  # lowest face index wins
        first_face[fe[:, f - 1]] = f
    nbf = len(interior) + len(lists[1]) + len(lists[3])
    bfe = np.zeros((2, nbf), np.int64)
    bff = np.zeros((2, nbf), np.int64)
    ebf = np.zeros(nedge, np.int64)
    for i, (fa, fb, _, _, e) in enumerate(interior):
        bfe[:, i] = e
        bff[:, i] = (fa, fb)
        ebf[e - 1] = i + 1
    i = len(interior)
    if sheet.xi_eta_check:
        xi0, xi1, et0, et1 = _xi_eta(sheet)
        for low, high, lo_v, hi_v in ((3, 4, xi0, xi1), (1, 2, et0, et1)):
            for g0 in lists[low]:
                a0, b0 = sorted((lo_v[g0 - 1], hi_v[g0 - 1]))
                match = [g for g in lists[high]
                         if abs(min(lo_v[g - 1], hi_v[g - 1]) - a0) < tol and abs(max(lo_v[g - 1], hi_v[g - 1]) - b0) < tol]
                if not match or first_face[g0] == 0 or first_face[match[0]] == 0:
                    raise ValueError(f"no partner or face for unit-cell boundary edge {g0}")
                g1 = match[0]
                bfe[:, i] = (g0, g1)
                bff[:, i] = (first_face[g0], first_face[g1])
                ebf[g0 - 1] = ebf[g1 - 1] = i + 1
                i += 1
    # unique face pairs
    npair = nface * nface
    if not sheet.fufp:
        ufpm = np.arange(1, npair + 1, dtype=np.int64).reshape((nface, nface), order="F")
        return Topology(bfe, bff, ebf, eci, ufpm, np.arange(1, npair + 1, dtype=np.int64), npair)
    rho = np.asarray(sheet.rho, float)
    fv = np.asarray(sheet.fv, np.int64)
    r = [rho[fv[k] - 1] for k in range(3)]
    cen = (r[0] + r[1] + r[2]) / 3
    rad = 1e-6 * float(np.linalg.norm(cen[0] - cen[1]))
    # column-major pair index p = m + n * nface (m: match, n: source)
    vec = np.concatenate([(cen[:, None, :] - r[k][None, :, :]) for k in range(3)], axis=2)  # [m, n, 6]
    vec = vec.transpose(1, 0, 2).reshape(npair, 6)  # row p = (n, m) with m fastest
    keys = np.round(vec / rad).astype(np.int64)
    _, first, inv = np.unique(keys, axis=0, return_index=True, return_inverse=True)
    inv = inv.ravel()
    rank = np.empty(len(first), np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(first))
    cls = rank[inv]
    rep = np.sort(first)
    if np.any(np.linalg.norm(vec - vec[rep[cls]], axis=1) >= rad):
        raise ValueError("a face pair lies outside the radius of its class's first member")
    ufpm = (cls + 1).reshape((nface, nface), order="F")
    return Topology(bfe, bff, ebf, eci, ufpm, rep.astype(np.int64) + 1, len(first))

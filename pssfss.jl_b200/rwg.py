"""RWG basis-function topology (PSSFSS.jl ``src/RWG.jl:27-324``).

``setup_rwg(sheet)`` returns the same ``bfe``, ``bff``, ``ebf``, ``eci``, ``ufpm``,
``ufp2fp`` and ``nufp`` as the reference (1-based values, Julia column-major meaning).

Unique face pairs (``RWG.jl:287-319``): the reference puts face pairs (m, n) (match m,
source n) whose 6-vectors ``(c_m - r1_n, c_m - r2_n, c_m - r3_n)`` lie within
``1e-6*|c_1 - c_2|`` of each other into one class, numbered in column-major order of
their first member.  Here the same classes are formed by exact grouping of the
quantised key ``(source-triangle shape, c_m - r1_n)`` on a grid of that radius: the
three vectors are determined by ``c_m - r1_n`` and the source triangle's edge vectors,
and translation-equivalent pairs agree to rounding error, far inside the radius.  A
pair whose key straddles a grid line would form its own class; its integrals then
equal the class's to rounding error, so results are unchanged.
"""
import math

import numpy as np


class RWGData:
    def __init__(self, bfe, bff, ebf, eci, ufpm, ufp_rep, nufp):
        self.bfe = bfe            # (2, nbf) int64, 1-based edge numbers
        self.bff = bff            # (2, nbf) int64, 1-based face numbers (plus, minus)
        self.ebf = ebf            # (nedge,) int64, basis function of each edge or 0
        self.eci = eci            # (nedge,) int64 in 0..4, unit-cell boundary code
        self.ufpm = ufpm          # (nface, nface) int64, ufpm[m, n] = class of (match m, source n)
        self.ufp_rep = ufp_rep    # (nufp,) int64, 1-based column-major index of each class's first pair
        self.nufp = nufp

    @property
    def nbf(self):
        return self.bfe.shape[1]

    @property
    def ufp2fp(self):
        """List of 1-based column-major face-pair indices per class (``RWG.jl:69``)."""
        flat = self.ufpm.ravel(order="F")
        order = np.argsort(flat, kind="stable")
        counts = np.bincount(flat, minlength=self.nufp + 1)[1:]
        ptr = np.concatenate([[0], np.cumsum(counts)])
        return [order[ptr[i]:ptr[i + 1]] + 1 for i in range(self.nufp)]


def _xieta(sheet, node):
    p = sheet.rho[node - 1]
    b1, b2 = sheet.beta1, sheet.beta2
    return (b1[0] * p[0] + b1[1] * p[1]) / (2 * math.pi), (b2[0] * p[0] + b2[1] * p[1]) / (2 * math.pi)


def get_ie_xieta(ie, sheet):
    """``get_ie_ξη`` (``RWG.jl:388-398``) for 1-based edge ``ie``."""
    xi0, eta0 = _xieta(sheet, int(sheet.e1[ie - 1]))
    xi1, eta1 = _xieta(sheet, int(sheet.e2[ie - 1]))
    return xi0, xi1, eta0, eta1


def _edge_xieta(sheet):
    """(xi, eta) of every edge's initial and terminal node (``get_ie_ξη``, ``RWG.jl:388-398``),
    as four arrays over the edges, computed as ``_xieta`` does node by node."""
    rho = np.asarray(sheet.rho, float)
    b1, b2 = sheet.beta1, sheet.beta2
    p0 = rho[np.asarray(sheet.e1, np.int64) - 1]
    p1 = rho[np.asarray(sheet.e2, np.int64) - 1]
    tp = 2 * math.pi
    return ((b1[0] * p0[:, 0] + b1[1] * p0[:, 1]) / tp, (b1[0] * p1[:, 0] + b1[1] * p1[:, 1]) / tp,
            (b2[0] * p0[:, 0] + b2[1] * p0[:, 1]) / tp, (b2[0] * p1[:, 0] + b2[1] * p1[:, 1]) / tp)


def setup_rwg(sheet):
    """Basis functions, boundary codes and unique face pairs of ``sheet`` (``RWG.jl:90``)."""
    tol = 1.0e-5
    nface = sheet.nface
    nedge = sheet.nedge
    fe = np.asarray(sheet.fe, np.int64)

    # Interior basis functions: each pair of faces (fp < fm) sharing an edge, ordered by
    # (fp, fm, local edge slot in fp, local edge slot in fm) like the reference's loops.
    # The 3 nface (face, slot, edge) incidences sorted by edge, face, slot: an edge of two
    # faces gives one pair; an edge of more faces gives every pair of distinct faces.
    face = np.repeat(np.arange(1, nface + 1, dtype=np.int64), 3)
    slot = np.tile(np.arange(3, dtype=np.int64), nface)
    edge = fe.T.ravel()
    order = np.lexsort((slot, face, edge))
    e_s, f_s, k_s = edge[order], face[order], slot[order]
    start = np.flatnonzero(np.r_[True, e_s[1:] != e_s[:-1]])
    size = np.diff(np.r_[start, len(e_s)])
    two = start[size == 2]
    rows = [np.stack([f_s[two], f_s[two + 1], k_s[two], k_s[two + 1], e_s[two]], axis=1)]
    for s0, n in zip(start[size > 2], size[size > 2]):  # an edge of three or more faces
        rows.append(np.array([(f_s[a], f_s[b], k_s[a], k_s[b], e_s[a]) for a in range(s0, s0 + n)
                              for b in range(a + 1, s0 + n)], np.int64).reshape(-1, 5))
    rows = np.concatenate(rows)
    rows = rows[rows[:, 0] < rows[:, 1]]
    rows = rows[np.lexsort((rows[:, 3], rows[:, 2], rows[:, 1], rows[:, 0]))]
    pf, mf, pe = rows[:, 0], rows[:, 1], rows[:, 4]
    nbf_int = len(rows)

    # Unit-cell boundary edges (codes 1: xi = 0, 2: xi = 1, 3: eta = 0, 4: eta = 1, tested in
    # that order); the xi = 0 and eta = 0 edges each add a basis function.
    eci = np.zeros(nedge, np.int64)
    if sheet.xi_eta_check:
        xi0, xi1, eta0, eta1 = _edge_xieta(sheet)
        conds = [(np.abs(xi0) < tol) & (np.abs(xi1) < tol), (np.abs(xi0 - 1) < tol) & (np.abs(xi1 - 1) < tol),
                 (np.abs(eta0) < tol) & (np.abs(eta1) < tol), (np.abs(eta0 - 1) < tol) & (np.abs(eta1 - 1) < tol)]
        eci = np.select(conds, [1, 2, 3, 4], 0).astype(np.int64)
    ie_xi0, ie_xi1 = np.flatnonzero(eci == 1) + 1, np.flatnonzero(eci == 2) + 1
    ie_eta0, ie_eta1 = np.flatnonzero(eci == 3) + 1, np.flatnonzero(eci == 4) + 1
    if len(ie_xi0) != len(ie_xi1):
        raise ValueError("Inconsistent # edges at ξ=0 and ξ=1")
    if len(ie_eta0) != len(ie_eta1):
        raise ValueError("Inconsistent # edges at η=0 and η=1")
    nbf = nbf_int + len(ie_xi0) + len(ie_eta0)

    bfe = np.zeros((2, nbf), np.int64)
    bff = np.zeros((2, nbf), np.int64)
    ebf = np.zeros(nedge, np.int64)
    bfe[0, :nbf_int] = pe
    bfe[1, :nbf_int] = pe
    bff[0, :nbf_int] = pf
    bff[1, :nbf_int] = mf
    if np.all(size <= 2):
        ebf[pe - 1] = np.arange(1, nbf_int + 1)
    else:
        for k, e in enumerate(pe):  # an edge in several pairs keeps its last one
            ebf[e - 1] = k + 1
    i = nbf_int

    # first (lowest-numbered) face holding each edge, 0 for none: the head of its sorted run
    first = np.zeros(nedge + 1, np.int64)
    first[e_s[start]] = f_s[start]

    def pair_boundary(list0, list1, use_xi):
        nonlocal i
        if len(list0) == 0:
            return
        xi0, xi1, eta0, eta1 = _edge_xieta(sheet)
        a, b = (xi0, xi1) if use_xi else (eta0, eta1)
        lo1, hi1 = np.minimum(a[list1 - 1], b[list1 - 1]), np.maximum(a[list1 - 1], b[list1 - 1])
        for ge0 in list0:
            face0 = first[ge0]
            if face0 == 0:
                raise ValueError(f"Unable to locate face containing boundary edge {ge0}")
            mn0, mx0 = min(a[ge0 - 1], b[ge0 - 1]), max(a[ge0 - 1], b[ge0 - 1])
            hit = np.flatnonzero((np.abs(lo1 - mn0) < tol) & (np.abs(hi1 - mx0) < tol))
            if len(hit) == 0:
                raise ValueError(f"Unable to locate edge corresponding to edge {ge0}")
            ge1 = int(list1[hit[0]])
            face1 = first[ge1]
            if face1 == 0:
                raise ValueError(f"Unable to locate face containing boundary edge {ge1}")
            bfe[:, i] = (ge0, ge1)
            bff[:, i] = (face0, face1)
            ebf[ge0 - 1] = i + 1
            ebf[ge1 - 1] = i + 1
            i += 1

    pair_boundary(ie_eta0, ie_eta1, use_xi=True)   # η=0 ↔ η=1 edges matched on ξ extent
    pair_boundary(ie_xi0, ie_xi1, use_xi=False)    # ξ=0 ↔ ξ=1 edges matched on η extent
    if i != nbf:
        raise ValueError("Inconsistent number of basis functions")

    if not sheet.fufp:
        nufp = nface * nface
        ufpm = np.arange(1, nufp + 1, dtype=np.int64).reshape((nface, nface), order="F")
        return RWGData(bfe, bff, ebf, eci, ufpm, np.arange(1, nufp + 1, dtype=np.int64), nufp)
    ufpm, rep, nufp = unique_face_pairs(sheet)
    return RWGData(bfe, bff, ebf, eci, ufpm, rep, nufp)


def _ufp_keys(sheet):
    """Per face pair (match m, source n): the source triangle's shape class and the offset of
    the match centroid from the source's first vertex, quantised on a grid of 1e-6 of the
    first two centroids' distance (the KD-tree radius of ``RWG.jl:305-315``)."""
    cen, r1, shape_id, g = _ufp_geometry(sheet)
    dx = np.round((cen[:, None, 0] - r1[None, :, 0]) / g).astype(np.int64)  # [m, n]
    dy = np.round((cen[:, None, 1] - r1[None, :, 1]) / g).astype(np.int64)
    return shape_id, dx, dy


def _ufp_geometry(sheet):
    """Centroids, first vertices, source-shape ids and the quantisation grid of the classing."""
    rho = sheet.rho
    r1 = rho[sheet.fv[0] - 1]
    r2 = rho[sheet.fv[1] - 1]
    r3 = rho[sheet.fv[2] - 1]
    cen = (r1 + r2 + r3) / 3
    d = cen[0] - cen[1]
    g = 1e-6 * math.sqrt(d[0] * d[0] + d[1] * d[1])
    shape_key = np.round(np.hstack([r2 - r1, r3 - r1]) / g).astype(np.int64)
    _, shape_id = np.unique(shape_key, axis=0, return_inverse=True)
    return cen, r1, shape_id.ravel().astype(np.int64), g


def unique_face_pairs(sheet, where="auto"):
    """Translation-equivalence classes of face pairs (``RWG.jl:287-319``), numbered in the
    order of their first member in column-major (match fastest) order.

    ``where="auto"`` classes on the GPU when one is present (``pss_face_pair_classes``: a hash
    table keyed on the same quantised keys, one thread per pair) and the sheet fits its limits;
    else on the host, where the three keys are packed into one integer when they fit in 62 bits
    (one sort) or sorted together."""
    nface = sheet.nface
    if where != "host":
        from . import engine
        if where == "device" or (nface <= engine.CLASSING_MAX_FACES and engine.device_available()):
            cen, r1, shape_id, g = _ufp_geometry(sheet)
            span = float(np.ptp(np.vstack([cen, r1]), axis=0).max())  # bounds every |offset|
            if span / g < 2.0 ** 30:
                try:
                    return engine.face_pair_classes(cen, r1, shape_id, g)
                except RuntimeError:
                    if where == "device":
                        raise  # asked for the device explicitly; "auto" classes on the host
            if where == "device":
                raise ValueError("face-pair offsets exceed the device classing's key range")
    shape_id, dx, dy = _ufp_keys(sheet)
    dx -= dx.min()
    dy -= dy.min()
    bx, by, bs = int(dx.max()).bit_length(), int(dy.max()).bit_length(), int(shape_id.max()).bit_length()
    if bx + by + bs > 62:
        return _unique_face_pairs_sorted(nface, shape_id, dx, dy)
    key = ((shape_id[None, :] << (bx + by)) | (dx << by) | dy).ravel(order="F")
    del dx, dy
    _, first, inv = np.unique(key, return_index=True, return_inverse=True)
    rank = np.empty(len(first), np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(first))
    cls = rank[inv.ravel()]
    # classes numbered by first appearance: a new class shows where cls passes its running max
    rep = np.flatnonzero(np.r_[True, cls[1:] > np.maximum.accumulate(cls)[:-1]])
    return (cls + 1).reshape((nface, nface), order="F"), (rep + 1).astype(np.int64), len(first)


def _unique_face_pairs_sorted(nface, shape_id, dx, dy):
    """``unique_face_pairs`` by a three-key sort (keys wider than one 62-bit integer)."""
    k0 = np.broadcast_to(shape_id[None, :], (nface, nface)).ravel(order="F")
    k1 = dx.ravel(order="F")
    k2 = dy.ravel(order="F")
    order = np.lexsort((k2, k1, k0))
    ks0, ks1, ks2 = k0[order], k1[order], k2[order]
    newgrp = np.ones(len(order), bool)
    newgrp[1:] = (ks0[1:] != ks0[:-1]) | (ks1[1:] != ks1[:-1]) | (ks2[1:] != ks2[:-1])
    starts = np.flatnonzero(newgrp)
    grp_sorted = np.cumsum(newgrp) - 1
    rep = np.minimum.reduceat(order, starts)      # smallest column-major index per group
    rank = np.empty(len(rep), np.int64)
    rank[np.argsort(rep, kind="stable")] = np.arange(len(rep))
    cls = np.empty(len(order), np.int64)
    cls[order] = rank[grp_sorted] + 1
    ufpm = cls.reshape((nface, nface), order="F")
    rep_sorted = np.sort(rep) + 1
    return ufpm, rep_sorted.astype(np.int64), len(rep)


def edge_current_unit_vector(ie, rwgdat, sheet):
    """Unit vector of the positive reference direction of the basis function on edge ``ie``
    (1-based; ``RWG.jl:339-363``): normal to the edge, pointing out of the basis function's
    plus face (away from that face's free vertex)."""
    bf = int(rwgdat.ebf[ie - 1])
    if bf == 0:
        raise ValueError(f"No basis function for edge {ie}")
    n1, n2 = int(sheet.e1[ie - 1]), int(sheet.e2[ie - 1])
    r21 = sheet.rho[n2 - 1] - sheet.rho[n1 - 1]
    t = r21 / math.hypot(r21[0], r21[1])
    u = np.array([-t[1], t[0]])  # ẑ × edge direction
    f = int(rwgdat.bff[0, bf - 1])
    nfree = next(int(v) for v in sheet.fv[:, f - 1] if v != n1 and v != n2)
    return -u if (sheet.rho[n1 - 1] - sheet.rho[nfree - 1]) @ u < 0 else u

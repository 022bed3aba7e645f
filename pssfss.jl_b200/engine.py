"""ctypes binding of ``libpssfss_b200.so`` (the CUDA hot path; C ABI in include/pssfss_b200.h).

There is no CPU fallback: if the library cannot be loaded or no CUDA device is present,
every call raises ``RuntimeError``.
"""
import collections
import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libpssfss_b200.so")

PSS_FP64 = 0
PSS_FP32_REFINE = 1
PRECISIONS = {"fp64": PSS_FP64, "fp32r": PSS_FP32_REFINE}

STATUS_BITS = {1: "table_noconv", 2: "jk_noconv", 4: "singular", 8: "refine_noconv", 16: "nonfinite",
               32: "fp64_fallback", 64: "device_timeout"}
FATAL_STATUS = 4 | 16 | 64

_lib = None
_lock = threading.RLock()  # context() reports a failed create through lib() while holding it
_ctx = {}
# uploaded sheets, most recently used last; a sheet's device arrays (its face-pair integral
# cache grows as nface^2 for unstructured sheets) are freed when it falls out
_sheets = collections.OrderedDict()
SHEET_CACHE = max(1, int(os.environ.get("PSS_SHEET_CACHE", "8")))

_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_L = ctypes.c_int64
_C = ctypes.c_char

# name -> (restype, argtypes); every function declared in include/pssfss_b200.h
SIGNATURES = {
    "pss_last_error": (ctypes.c_char_p, []),
    "pss_version": (_I, []),
    "pss_kernel_launches": (_L, []),
    "pss_ctx_create": (_I, [_I, _I, _P]),
    "pss_ctx_destroy": (_I, [_P]),
    "pss_ctx_device": (_I, [_P, _P]),
    "pss_cascade": (_I, [_P, _I, _I, _P, _P, _P, _P, _P]),
    "pss_face_pair_classes": (_I, [_P, _L, _P, _P, _P, _D, _P, _P, _L, _P]),
    "pss_sheet_create": (_I, [_P, _C, _D, _P, _P, _P, _P, _L, _P, _L, _P, _P, _P, _L, _L, _P, _P, _P, _L,
                              _P, _P, _P]),
    "pss_sheet_destroy": (_I, [_P]),
    "pss_sheet_clear_cache": (_I, [_P]),
    "pss_partial_gsms": (_I, [_P, _I, _P, _P, _P, _I, _D, _I, _P, _P, _I, _P, _P, _P, _P, _I, _P, _P]),
    "pss_partial_gsms_multi": (_I, [_I, _P, _I]),
    "pss_partial_gsms_lin": (_I, [_P, _I, _P, _P, _P, _I, _D, _I, _P, _P, _I, _P, _P, _P, _P, _I, _P, _P, _P,
                                  _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P]),
    "pss_partial_gsms_adj": (_I, [_P, _I, _P, _P, _P, _I, _D, _I, _P, _P, _I, _P, _P, _P, _P, _I, _P, _P, _P,
                                  _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P]),
    "pss_fill_matrix": (_I, [_P, _I, _P, _P, _P, _I, _D, _D, _D, _D, _P, _P]),
    "pss_modal_tables": (_I, [_P, _I, _I, _P, _P, _P, _I, _D, _D, _D, _D, _P, _P, _D, _L, _P, _P, _P, _P]),
    "pss_face_integrals": (_I, [_P, _D, _D, _D, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "pss_basis_transforms": (_I, [_P, _I, _P, _D, _D, _P]),
    "pss_lu_solve": (_I, [_P, _I, _P, _I, _P, _I, _P, _P]),
    "pss_last_timings": (_I, [_P, _P]),
    "pss_profile": (_I, [_P, _I]),
    "pss_profile_result": (_I, [_P, _P]),
    "pss_schur_update": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P]),
    "pss_lu_factor_noalloc": (_I, [_I, _P, _L, _P, _P, _P]),
    "pss_set_wait_limit": (_I, [_L]),
    "pss_lu32_factor": (_I, [_P, _I, _P, _P, _P, _P]),
}


def set_profiling(on, device=0, nworkers=None):
    _check(lib().pss_profile(context(device, nworkers), int(on)), "pss_profile")


PROFILE_KINDS = ("tc_update", "panel", "simt_update")  # PSS_PROF_* order


def profile_result(device=0, nworkers=None):
    """Per kernel kind: launches, summed device ms and algorithmic work (flops, or bytes for
    the panel) of the last ``partial_gsms`` call made while profiling was enabled."""
    out = np.zeros(3 * len(PROFILE_KINDS))
    _check(lib().pss_profile_result(context(device, nworkers), _p(out)), "pss_profile_result")
    return {k: {"launches": int(out[3 * i]), "ms": float(out[3 * i + 1]), "work": float(out[3 * i + 2])}
            for i, k in enumerate(PROFILE_KINDS)}


def device_available():
    """True when the library loads and a CUDA device is present (no context is created)."""
    try:
        L = lib()
    except RuntimeError:
        return False
    try:
        import torch
        return bool(torch.cuda.is_available())
    except Exception:
        return False


def lib():
    """Load the library (raises if it is missing: the CUDA path is the only path)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIBPATH):
                raise RuntimeError(f"{LIBPATH} not built; run __graft_entry__.build() (nvcc, sm_100a)")
            L = ctypes.CDLL(LIBPATH)
            for name, (res, args) in SIGNATURES.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def _check(rc, what):
    if rc != 0:
        msg = lib().pss_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed ({rc}): {msg}")


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f64(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def _c2d(x):
    """complex array -> contiguous interleaved float64 view."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128))
    return a


def _i64(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.int64))


def context(device=0, nworkers=None):
    """Per-device ``pss_ctx`` (created once)."""
    if nworkers is None:
        # one stream per worker, each factoring a batch of points at a time (PSS_BATCH,
        # default 12, read by the library); more streams than the process's hardware work
        # queues (CUDA_DEVICE_MAX_CONNECTIONS, default 8) would share queues
        queues = int(os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS", "8"))
        nworkers = int(os.environ.get("PSS_WORKERS", str(max(1, min(3, queues)))))
    key = (device, nworkers)
    L = lib()
    with _lock:
        c = _ctx.get(key)
        if c is None:
            h = ctypes.c_void_p()
            _check(L.pss_ctx_create(device, nworkers, ctypes.byref(h)), "pss_ctx_create")
            c = _ctx[key] = h
    return c


def region_arrays(layers):
    eps = _c2d([l.epsr for l in layers])
    mu = _c2d([l.mur for l in layers])
    w = _f64([l.width for l in layers])
    return eps, mu, w


class DeviceSheet:
    """A sheet uploaded to one device context (``pss_sheet``)."""

    def __init__(self, ctx, sheet, rwg):
        self.sheet, self.rwg = sheet, rwg
        h = ctypes.c_void_p()
        rho = _f64(sheet.rho)
        fv = _i64(sheet.fv.ravel(order="F"))
        fe = _i64(sheet.fe.ravel(order="F"))
        fr = _f64(sheet.fr)
        bff = _i64(rwg.bff.ravel(order="F"))
        ebf = _i64(rwg.ebf)
        eci = _i64(rwg.eci)
        ufpm = _i64(rwg.ufpm.ravel(order="F"))
        rep = _i64(rwg.ufp_rep)
        _check(lib().pss_sheet_create(ctx, sheet.cls.encode(), sheet.units.units_per_meter, _p(_f64(sheet.s1)),
                                      _p(_f64(sheet.s2)), _p(_f64(sheet.beta1)), _p(_f64(sheet.beta2)),
                                      sheet.nnode, _p(rho), sheet.nface, _p(fv), _p(fe), _p(fr), sheet.nedge,
                                      rwg.nbf, _p(bff), _p(ebf), _p(eci), rwg.nufp, _p(ufpm), _p(rep),
                                      ctypes.byref(h)), "pss_sheet_create")
        self.h = h

    def __del__(self):
        try:
            if self.h:
                lib().pss_sheet_destroy(self.h)
        except Exception:
            pass


def device_sheet(sheet, rwg, device=0, nworkers=None):
    ctx = context(device, nworkers)
    key = (id(sheet), id(rwg), ctx.value)
    evicted = []
    with _lock:
        ds = _sheets.get(key)
        if ds is not None and ds.sheet is sheet and ds.rwg is rwg:
            _sheets.move_to_end(key)
            return ds
    ds = DeviceSheet(ctx, sheet, rwg)
    with _lock:
        _sheets[key] = ds
        while len(_sheets) > SHEET_CACHE:
            evicted.append(_sheets.popitem(last=False)[1])
    del evicted  # pss_sheet_destroy runs here, outside the lock
    return ds


def clear_face_integrals(sheet, rwg, device=0, nworkers=None):
    """Drop the uploaded sheet's cached face-pair integrals (``pss_sheet_clear_cache``)."""
    _check(lib().pss_sheet_clear_cache(device_sheet(sheet, rwg, device, nworkers).h), "pss_sheet_clear_cache")


def partial_gsms(sheet, rwg, points, region_rng, s, u, ios, precision="fp64", device=0, stats=None,
                 nworkers=None):
    """Scattered partial GSMs of one sheet at every point (``pss_partial_gsms``)."""
    i1, i2 = region_rng
    region = points[0].layers[i1 - 1:i2]
    eps, mu, w = region_arrays(region)
    npts = len(points)
    nm = len(ios[0].wobs)
    k0 = _f64([pt.k0 for pt in points])
    psi = _f64([[io.psi1, io.psi2] for io in ios])
    kvec = _f64(np.stack([io.kvec for io in ios]))
    src = _c2d(np.stack([io.src for io in ios]))
    tobs = _f64(np.stack([io.tobs for io in ios]))
    wobs = _c2d(np.stack([io.wobs for io in ios]))
    dS = np.zeros((npts, nm, nm), complex)       # per point column-major -> transpose below
    status = np.zeros(npts, np.int32)
    ds = device_sheet(sheet, rwg, device, nworkers)
    _check(lib().pss_partial_gsms(ds.h, len(region), _p(eps), _p(mu), _p(w), s, float(u), npts, _p(k0),
                                  _p(psi), nm, _p(kvec), _p(src), _p(tobs), _p(wobs), PRECISIONS[precision],
                                  _p(dS), _p(status)), "pss_partial_gsms")
    if stats is not None:
        t = np.zeros(8)
        lib().pss_last_timings(context(device, nworkers), _p(t))
        stats.setdefault("status", []).extend(status.tolist())
        stats["timings_ms"] = dict(zip(["tables", "face_integrals", "fill", "transforms", "unused",
                                        "factor_solve", "project", "total"], t.tolist()))
        stats["timings_ms"].pop("unused")
    bad = status & FATAL_STATUS
    if bad.any():
        raise RuntimeError(f"solver status {status.tolist()} (singular, non-finite or device timeout)")
    return [d.T.copy() for d in dS]


class Problem(ctypes.Structure):
    """``pss_problem`` of include/pssfss_b200.h."""
    _fields_ = [("sheet", _P), ("nl", _I), ("eps", _P), ("mu", _P), ("width", _P), ("s", _I), ("u", _D),
                ("npts", _I), ("k0", _P), ("psi", _P), ("nmodes", _I), ("kvec", _P), ("src", _P), ("tobs", _P),
                ("wobs", _P), ("batch", _I), ("panel_w", _I), ("outer_nb", _I), ("dS", _P), ("status", _P)]


def partial_gsms_multi(problems, precision="fp64", device=0, nworkers=None, stats=None):
    """Scattered partial GSMs of many sheet sweeps in one ``pss_partial_gsms_multi`` call.

    ``problems``: list of dicts with the arguments of ``partial_gsms`` (``sheet``, ``rwg``,
    ``points``, ``region_rng``, ``s``, ``u``, ``ios``) and optionally ``batch``, ``panel_w``,
    ``outer_nb`` (0: defaults).  Returns one list of per-point dS matrices per problem."""
    keep, arr, outs = [], (Problem * len(problems))(), []
    for k, pr in enumerate(problems):
        i1, i2 = pr["region_rng"]
        pts, ios = pr["points"], pr["ios"]
        region = pts[0].layers[i1 - 1:i2]
        eps, mu, w = region_arrays(region)
        npts, nm = len(pts), len(ios[0].wobs)
        bufs = dict(eps=eps, mu=mu, w=w, k0=_f64([pt.k0 for pt in pts]),
                    psi=_f64([[io.psi1, io.psi2] for io in ios]), kvec=_f64(np.stack([io.kvec for io in ios])),
                    src=_c2d(np.stack([io.src for io in ios])), tobs=_f64(np.stack([io.tobs for io in ios])),
                    wobs=_c2d(np.stack([io.wobs for io in ios])), dS=np.zeros((npts, nm, nm), complex),
                    status=np.zeros(npts, np.int32),
                    ds=device_sheet(pr["sheet"], pr["rwg"], device, nworkers))
        keep.append(bufs)
        arr[k] = Problem(bufs["ds"].h, len(region), _p(eps), _p(mu), _p(w), int(pr["s"]), float(pr["u"]), npts,
                         _p(bufs["k0"]), _p(bufs["psi"]), nm, _p(bufs["kvec"]), _p(bufs["src"]), _p(bufs["tobs"]),
                         _p(bufs["wobs"]), int(pr.get("batch", 0)), int(pr.get("panel_w", 0)),
                         int(pr.get("outer_nb", 0)), _p(bufs["dS"]), _p(bufs["status"]))
    _check(lib().pss_partial_gsms_multi(len(problems), ctypes.cast(arr, ctypes.c_void_p), PRECISIONS[precision]),
           "pss_partial_gsms_multi")
    if stats is not None:
        t = np.zeros(8)
        lib().pss_last_timings(context(device, nworkers), _p(t))
        stats["status"] = [b["status"].tolist() for b in keep]
        stats["timings_ms"] = dict(zip(["tables", "face_integrals", "fill", "transforms", "unused",
                                        "factor_solve", "project", "total"], t.tolist()))
        stats["timings_ms"].pop("unused")
    for b in keep:
        if (b["status"] & FATAL_STATUS).any():
            raise RuntimeError(f"solver status {b['status'].tolist()} (singular, non-finite or device timeout)")
        outs.append([d.T.copy() for d in b["dS"]])
    return outs


def partial_gsms_adjoint(sheet, rwg, points, region_rng, s, u, ios, perturbed, precision="fp64", device=0):
    """``partial_gsms_linearized`` in its adjoint form (``pss_partial_gsms_adj``): one
    factorisation, forward and transposed solves on it, and per perturbed set a fused
    assemble-and-contract pass instead of a stored matrix and further solves."""
    return partial_gsms_linearized(sheet, rwg, points, region_rng, s, u, ios, perturbed, precision, device,
                                   entry="pss_partial_gsms_adj")


def partial_gsms_linearized(sheet, rwg, points, region_rng, s, u, ios, perturbed, precision="fp64", device=0,
                            entry="pss_partial_gsms_lin"):
    """Scattered partial GSMs of one sheet Gblock and their first-order values at each
    perturbed input set (``pss_partial_gsms_lin``, or ``entry``), the ``partial_lin`` form
    that ``gradient.linearized_gradient`` takes.  ``perturbed``: (sheet_k, rwg_k, points_k,
    u_k, ios_k) per set, with the topology of ``sheet``."""
    i1, i2 = region_rng
    region = points[0].layers[i1 - 1:i2]
    eps, mu, w = region_arrays(region)
    npts, nm, K = len(points), len(ios[0].wobs), len(perturbed)

    def modes(ios_):
        return (_f64(np.stack([io.kvec for io in ios_])), _c2d(np.stack([io.src for io in ios_])),
                _f64(np.stack([io.tobs for io in ios_])), _c2d(np.stack([io.wobs for io in ios_])))
    k0 = _f64([pt.k0 for pt in points])
    psi = _f64([[io.psi1, io.psi2] for io in ios])
    kvec, src, tobs, wobs = modes(ios)
    ds = device_sheet(sheet, rwg, device)
    held = [device_sheet(sh_k, rw_k, device) for sh_k, rw_k, _, _, _ in perturbed]
    psh = (ctypes.c_void_p * max(K, 1))(*[d.h.value for d in held])
    pe, pm, pw, pu, pp, pk, ps, pt, pwo = [], [], [], [], [], [], [], [], []
    for (_, _, pts_k, u_k, ios_k) in perturbed:
        e_, m_, w_ = region_arrays(pts_k[0].layers[i1 - 1:i2])
        pe.append(e_)
        pm.append(m_)
        pw.append(w_)
        pu.append(float(u_k))
        pp.append([[io.psi1, io.psi2] for io in ios_k])
        a, b, c, d = modes(ios_k)
        pk.append(a)
        ps.append(b)
        pt.append(c)
        pwo.append(d)
    z = np.zeros(1)
    arr = (lambda xs, f: f(np.stack(xs)) if xs else z)
    peps, pmu, pwidth = arr(pe, _c2d), arr(pm, _c2d), arr(pw, _f64)
    pu_, ppsi, pkvec = arr(pu, _f64), arr(pp, _f64), arr(pk, _f64)
    psrc, ptobs, pwobs = arr(ps, _c2d), arr(pt, _f64), arr(pwo, _c2d)
    dS = np.zeros((npts, nm, nm), complex)
    dSp = np.zeros((max(K, 1), npts, nm, nm), complex)
    status = np.zeros(npts, np.int32)
    _check(getattr(lib(), entry)(ds.h, len(region), _p(eps), _p(mu), _p(w), s, float(u), npts, _p(k0), _p(psi),
                                 nm, _p(kvec), _p(src), _p(tobs), _p(wobs), K, psh, _p(peps), _p(pmu),
                                 _p(pwidth), _p(pu_), _p(ppsi), _p(pkvec), _p(psrc), _p(ptobs), _p(pwobs),
                                 PRECISIONS[precision], _p(dS), _p(dSp), _p(status)), entry)
    if (status & FATAL_STATUS).any():
        raise RuntimeError(f"solver status {status.tolist()} (singular, non-finite or device timeout)")
    del held
    return [d.T.copy() for d in dS], [[d.T.copy() for d in dSp[k]] for k in range(K)]


CLASSING_MAX_FACES = 16384


def face_pair_classes(cen, r1, shape_id, g, device=0):
    """Unique face-pair classes on the device (``pss_face_pair_classes``): returns (ufpm
    (nface x nface int64, 1-based, column-major), rep (1-based pair indices), nufp)."""
    nface = len(shape_id)
    cen = _f64(cen)
    r1 = _f64(r1)
    shape = _i64(shape_id)
    ufpm = np.zeros((nface, nface), np.int32, order="F")
    cap = max(1024, nface * nface // 8)
    nufp = ctypes.c_int64()
    for _ in range(2):
        rep = np.zeros(cap, np.int64)
        rc = lib().pss_face_pair_classes(context(device), nface, _p(cen), _p(r1), _p(shape), float(g),
                                         ufpm.ctypes.data_as(ctypes.c_void_p), _p(rep), cap, ctypes.byref(nufp))
        if rc == -5:
            cap = int(nufp.value)
            continue
        _check(rc, "pss_face_pair_classes")
        break
    n = int(nufp.value)
    return ufpm.astype(np.int64), rep[:n].copy(), n


CASCADE_MAX_MODES = 64


def cascade_points(chains, device=0):
    """GSM cascade of many points on the device (``pss_cascade``).  ``chains``: per point a
    list ``[p0, (B_0, p_1), (B_1, p_2), ...]`` - p0 the propagation factors of layer 0, then
    per Gblock its GSM (``.s11 .. .s22``) and the factors of the layer behind it.  Every point
    must have the same mode counts.  Returns per point (s11, s12, s21, s22)."""
    npts = len(chains)
    p0 = np.asarray(chains[0][0])
    blocks = chains[0][1:]
    dims = [len(p0)] + [len(p) for _, p in blocks]
    nblk = len(blocks)
    recs, props = [], []
    for ch in chains:
        pr = [np.asarray(ch[0], complex)]
        rec = []
        for B, p in ch[1:]:
            rec += [np.asarray(B.s11, complex).ravel(order="F"), np.asarray(B.s12, complex).ravel(order="F"),
                    np.asarray(B.s21, complex).ravel(order="F"), np.asarray(B.s22, complex).ravel(order="F")]
            pr.append(np.asarray(p, complex))
        recs.append(np.concatenate(rec))
        props.append(np.concatenate(pr))
    gsm = _c2d(np.concatenate(recs))
    prop = _c2d(np.concatenate(props))
    n0, nK = dims[0], dims[-1]
    per = n0 * n0 + 2 * n0 * nK + nK * nK
    out = np.zeros(npts * per, complex)
    status = np.zeros(npts, np.int32)
    d = np.ascontiguousarray(np.asarray(dims, np.int32))
    _check(lib().pss_cascade(context(device), npts, nblk, _p(d), _p(gsm), _p(prop), _p(out), _p(status)),
           "pss_cascade")
    if (status & 4).any():
        raise RuntimeError(f"pss_cascade: singular star-product system at points {np.flatnonzero(status).tolist()}")
    res = []
    for i in range(npts):
        o = out[i * per:(i + 1) * per]
        a, b, c = n0 * n0, n0 * n0 + n0 * nK, n0 * n0 + 2 * n0 * nK
        res.append((o[:a].reshape((n0, n0), order="F"), o[a:b].reshape((n0, nK), order="F"),
                    o[b:c].reshape((nK, n0), order="F"), o[c:].reshape((nK, nK), order="F")))
    return res


def fill_matrix(sheet, rwg, layers, s, u, k0, psi1, psi2, device=0):
    ds = device_sheet(sheet, rwg, device)
    eps, mu, w = region_arrays(layers)
    n = rwg.nbf
    Z = np.zeros((n, n), complex, order="F")
    mm = ctypes.c_int()
    _check(lib().pss_fill_matrix(ds.h, len(layers), _p(eps), _p(mu), _p(w), s, float(u), float(k0), float(psi1),
                                 float(psi2), Z.ctypes.data_as(ctypes.c_void_p), ctypes.byref(mm)),
           "pss_fill_matrix")
    return Z, mm.value


def modal_tables(magnetic, k0, u, psi1, psi2, layers, s, b1, b2, convtest=1e-7, device=0):
    ctx = context(device)
    eps, mu, w = region_arrays(layers)
    cap = (2048 + 2) ** 2
    t1 = np.zeros(cap, complex)
    t2 = np.zeros(cap, complex)
    mm = ctypes.c_int()
    st = ctypes.c_int()
    _check(lib().pss_modal_tables(ctx, int(magnetic), len(layers), _p(eps), _p(mu), _p(w), s, float(k0), float(u),
                                  float(psi1), float(psi2), _p(_f64(b1)), _p(_f64(b2)), float(convtest), cap,
                                  _p(t1), _p(t2), ctypes.byref(mm), ctypes.byref(st)), "pss_modal_tables")
    L = (mm.value + 2) ** 2
    return mm.value, t1[:L].copy(), t2[:L].copy(), st.value


def face_integrals(sheet, rwg, ulocal, psi1, psi2, device=0):
    ds = device_sheet(sheet, rwg, device)
    n = rwg.nufp
    out = {k: np.zeros(n, complex) for k in ("J", "Jxi", "Jeta", "K", "Kxi", "Keta")}
    rho_r = np.zeros(2 * n)
    rinv = np.zeros(n)
    nc = ctypes.c_int()
    _check(lib().pss_face_integrals(ds.h, float(ulocal), float(psi1), float(psi2), _p(out["J"]), _p(out["Jxi"]),
                                    _p(out["Jeta"]), _p(out["K"]), _p(out["Kxi"]), _p(out["Keta"]), _p(rho_r),
                                    _p(rinv), ctypes.byref(nc)), "pss_face_integrals")
    out["rho_r"], out["rinv"], out["nonconv"] = rho_r, rinv, nc.value
    return out


def basis_transforms(sheet, rwg, kvecs, psi1, psi2, device=0):
    ds = device_sheet(sheet, rwg, device)
    kv = _f64(np.atleast_2d(kvecs))
    nm = kv.shape[0]
    F = np.zeros((nm, rwg.nbf, 2), complex)
    _check(lib().pss_basis_transforms(ds.h, nm, _p(kv), float(psi1), float(psi2), _p(F)), "pss_basis_transforms")
    return F


def lu_solve(Z, B, precision="fp64", device=0):
    ctx = context(device)
    Z = np.asfortranarray(np.asarray(Z, complex))
    B = np.asfortranarray(np.asarray(B, complex).reshape(Z.shape[0], -1))
    n, nrhs = B.shape
    X = np.zeros((n, nrhs), complex, order="F")
    st = ctypes.c_int()
    _check(lib().pss_lu_solve(ctx, n, Z.ctypes.data_as(ctypes.c_void_p), nrhs, B.ctypes.data_as(ctypes.c_void_p),
                              PRECISIONS[precision], X.ctypes.data_as(ctypes.c_void_p), ctypes.byref(st)),
           "pss_lu_solve")
    return X, st.value


def lu32_factor(Z, device=0):
    """FP32 LU of the FP32 + refinement form (``pss_lu32_factor``): returns (LU packed
    complex64, 1-based ipiv, info)."""
    ctx = context(device)
    Z = np.asfortranarray(np.asarray(Z, complex))
    n = Z.shape[0]
    LU = np.zeros((n, n), np.complex64, order="F")
    ipiv = np.zeros(n, np.int32)
    info = ctypes.c_int()
    _check(lib().pss_lu32_factor(ctx, n, Z.ctypes.data_as(ctypes.c_void_p), LU.ctypes.data_as(ctypes.c_void_p),
                                 ipiv.ctypes.data_as(ctypes.c_void_p), ctypes.byref(info)), "pss_lu32_factor")
    return LU, ipiv, info.value


def schur_update(L, U, C, device=0):
    """C - L @ U in complex FP32 on the tensor cores (``pss_schur_update``); returns (C', status)."""
    L = np.asarray(L, np.complex64)
    U = np.asarray(U, np.complex64)
    C = np.asarray(C, np.complex64)
    m, k = L.shape
    k2, n = U.shape
    if k2 != k or C.shape != (m, n):
        raise ValueError("shape mismatch")
    parts = [np.ascontiguousarray(x, np.float32) for x in (L.real, L.imag, U.real, U.imag, C.real, C.imag)]
    st = ctypes.c_int()
    _check(lib().pss_schur_update(context(device), m, n, k, *[_p(x) for x in parts], ctypes.byref(st)),
           "pss_schur_update")
    return parts[4] + 1j * parts[5], st.value

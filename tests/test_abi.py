"""The C-ABI library loads and exports every symbol the public header declares (no GPU
calls), and the Python binding declares a signature for each of them."""
import os
import re

import pytest

from pssfss_b200 import _build, engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "pssfss_b200.h")).read()
    return sorted(set(re.findall(r"\b(pss_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    _build.build()
    L = engine.lib()
    syms = header_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(engine.SIGNATURES)
    assert L.pss_version() >= 100


def test_no_device_error_is_reported_not_raised_in_c():
    # Without a GPU the context creation must fail cleanly with a message.
    import ctypes
    if os.environ.get("CUDA_VISIBLE_DEVICES") is None:
        try:
            import torch
            if torch.cuda.is_available():
                pytest.skip("a GPU is present")
        except Exception:
            pass
    h = ctypes.c_void_p()
    rc = engine.lib().pss_ctx_create(0, 1, ctypes.byref(h))
    assert rc != 0
    assert b"device" in engine.lib().pss_last_error().lower() or b"cuda" in engine.lib().pss_last_error().lower()
    # and the binding raises it (from inside its context cache, without deadlocking on its lock)
    import threading
    out = {}

    def make():
        try:
            engine.context(0, 1)
        except RuntimeError as e:
            out["err"] = str(e)
    t = threading.Thread(target=make, daemon=True)
    t.start()
    t.join(60)
    assert not t.is_alive(), "engine.context() hung on a failed pss_ctx_create"
    assert "pss_ctx_create" in out.get("err", "")


def test_entry_points_reject_bad_arguments_before_any_device_use():
    # Every export returns 0 or a negative code with a message and never aborts; these checks
    # run before a device is touched, so they hold on a machine without a GPU.
    import ctypes
    L = engine.lib()
    nul = None
    buf = (ctypes.c_double * 8)()
    ibuf = (ctypes.c_int * 8)()

    def err():
        return L.pss_last_error().decode()

    assert L.pss_ctx_destroy(nul) == 0 and L.pss_sheet_destroy(nul) == 0
    assert L.pss_sheet_clear_cache(nul) == -1 and "null" in err()
    assert L.pss_partial_gsms_adj(nul, 1, buf, buf, buf, 1, 1.0, 1, buf, buf, 1, buf, buf, buf, buf, 0, nul,
                                  *([nul] * 9), 0, buf, nul, ibuf) == -1 and "null" in err()
    assert L.pss_partial_gsms(nul, 1, buf, buf, buf, 1, 1.0, 1, buf, buf, 1, buf, buf, buf, buf, 0,
                              buf, ibuf) == -1 and "null" in err()
    assert L.pss_partial_gsms_lin(nul, 1, buf, buf, buf, 1, 1.0, 1, buf, buf, 1, buf, buf, buf, buf, 0, nul,
                                  *([nul] * 9), 0, buf, nul, ibuf) == -1 and "null" in err()
    assert L.pss_fill_matrix(nul, 1, buf, buf, buf, 1, 1.0, 1.0, 0.0, 0.0, buf,
                             ctypes.byref(ctypes.c_int())) == -1 and "null" in err()
    assert L.pss_face_integrals(nul, 1.0, 0.0, 0.0, *([buf] * 9)) == -1 and "null" in err()
    assert L.pss_basis_transforms(nul, 1, buf, 0.0, 0.0, buf) == -1 and "invalid" in err()
    assert L.pss_lu_solve(nul, 4, buf, 1, buf, 0, buf, ibuf) == -1 and "invalid" in err()
    assert L.pss_profile(nul, 1) == -1 and L.pss_last_timings(nul, buf) == -1
    h = ctypes.c_void_p()
    assert L.pss_sheet_create(nul, b"J", 1.0, buf, buf, buf, buf, 0, buf, 0, ibuf, ibuf, buf, 0, 0, ibuf,
                              ibuf, ibuf, 0, ibuf, ibuf, ctypes.byref(h)) == -1 and "null" in err()
    # the no-allocation LU: invalid shapes and orders beyond its fixed scratch array
    assert L.pss_lu_factor_noalloc(0, buf, 1, ibuf, ibuf, nul) == -1 and "invalid" in err()
    assert L.pss_lu_factor_noalloc(4, buf, 2, ibuf, ibuf, nul) == -1 and "invalid" in err()
    assert L.pss_lu_factor_noalloc(9000, buf, 9000, ibuf, ibuf, nul) == -1 and "exceeds" in err()


def test_device_sheet_cache_is_bounded_and_reuses_entries(monkeypatch):
    # Host logic of the binding: an uploaded sheet is reused while cached, and the least
    # recently used one is released once more than SHEET_CACHE sheets were uploaded.
    import ctypes
    made, freed = [], []

    class FakeDeviceSheet:
        def __init__(self, ctx, sheet, rwg):
            self.sheet, self.rwg = sheet, rwg
            made.append(sheet)

        def __del__(self):
            freed.append(self.sheet)

    monkeypatch.setattr(engine, "context", lambda device=0, nworkers=None: ctypes.c_void_p(1))
    monkeypatch.setattr(engine, "DeviceSheet", FakeDeviceSheet)
    monkeypatch.setattr(engine, "SHEET_CACHE", 2)
    monkeypatch.setattr(engine, "_sheets", engine.collections.OrderedDict())
    s = [object() for _ in range(3)]
    r = object()
    a = engine.device_sheet(s[0], r)
    assert engine.device_sheet(s[0], r) is a and made == [s[0]]
    engine.device_sheet(s[1], r)
    engine.device_sheet(s[0], r)          # s[0] becomes the most recent
    engine.device_sheet(s[2], r)          # evicts s[1]
    assert made == [s[0], s[1], s[2]] and freed == [s[1]]
    assert [v.sheet for v in engine._sheets.values()] == [s[0], s[2]]
    del a


def test_linearized_binding_packs_the_header_layout(monkeypatch):
    # Host side of engine.partial_gsms_linearized without a device: the arrays handed to
    # pss_partial_gsms_lin follow the header's layout (perturbed set k, point i, mode j at
    # (k*npts + i)*nmodes + j), and the outputs come back per point, transposed.
    import ctypes
    import types
    import numpy as np
    from pssfss_b200.layers import Layer

    npts, nm, K, nl = 3, 2, 2, 3
    rng = np.random.default_rng(0)

    def io(seed):
        r = np.random.default_rng(seed)
        return types.SimpleNamespace(kvec=r.normal(size=(nm, 2)), src=r.normal(size=(nm, 2)) + 1j * r.normal(size=(nm, 2)),
                                     tobs=r.normal(size=(nm, 2)), wobs=r.normal(size=nm) + 1j * r.normal(size=nm),
                                     psi1=float(r.normal()), psi2=float(r.normal()))
    layers = [Layer(), Layer(epsr=2.2), Layer()]
    pts = [types.SimpleNamespace(layers=layers, k0=100.0 + i) for i in range(npts)]
    ios = [io(i) for i in range(npts)]
    pert = [(object(), object(), pts, 7.0 + k, [io(100 * (k + 1) + i) for i in range(npts)]) for k in range(K)]
    seen = {}

    def fake_call(*a):
        names = ["sh", "nl", "eps", "mu", "width", "s", "u", "npts", "k0", "psi", "nm", "kvec", "src", "tobs", "wobs",
                 "npert", "psh", "peps", "pmu", "pwidth", "pu", "ppsi", "pkvec", "psrc", "ptobs", "pwobs", "prec",
                 "dS", "dSp", "status"]
        seen.update(zip(names, a))
        seen["dS"][:] = rng.normal(size=seen["dS"].shape)
        seen["dSp"][:] = rng.normal(size=seen["dSp"].shape)
        return 0

    monkeypatch.setattr(engine, "_p", lambda x: x)
    monkeypatch.setattr(engine, "lib", lambda: types.SimpleNamespace(pss_partial_gsms_lin=fake_call))
    monkeypatch.setattr(engine, "device_sheet", lambda sh, rw, device=0: types.SimpleNamespace(h=ctypes.c_void_p(7)))
    dS, lin = engine.partial_gsms_linearized(object(), object(), pts, (1, 3), 1, 5.0, ios, pert)
    assert seen["nl"] == nl and seen["npert"] == K and seen["npts"] == npts and seen["nm"] == nm
    pk = seen["pkvec"].reshape(K, npts, nm, 2)
    ps = seen["psrc"].reshape(K, npts, nm, 2)
    for k in range(K):
        assert seen["pu"][k] == 7.0 + k
        for i in range(npts):
            assert np.array_equal(pk[k, i], pert[k][4][i].kvec) and np.array_equal(ps[k, i], pert[k][4][i].src)
            assert tuple(seen["ppsi"][k, i]) == (pert[k][4][i].psi1, pert[k][4][i].psi2)
    assert seen["peps"].shape == (K, nl) and seen["peps"][0, 1] == layers[1].epsr
    assert np.array_equal(dS[1], seen["dS"][1].T) and np.array_equal(lin[1][2], seen["dSp"][1, 2].T)


def _julia_stub_sheet_arrays(sheet, rwg):
    """The arguments INTEGRATION.md's Julia stub hands to pss_sheet_create, built from
    RWGSheet/RWGData-shaped fields the way the stub builds them: every index array passes
    unchanged (Int64, 1-based, column-major), ufp_rep = first.(rwgdat.ufp2fp)."""
    import numpy as np
    jl = {"fv": np.asarray(sheet.fv, np.int64), "fe": np.asarray(sheet.fe, np.int64),
          "bff": np.asarray(rwg.bff, np.int64), "ebf": np.asarray(rwg.ebf, np.int64),
          "eci": np.asarray(rwg.eci, np.int64), "ufpm": np.asarray(rwg.ufpm, np.int64),
          "ufp2fp": rwg.ufp2fp}
    col = (lambda a: np.ascontiguousarray(a.ravel(order="F")))  # Julia's memory order
    return {"fv": col(jl["fv"]), "fe": col(jl["fe"]), "bff": col(jl["bff"]), "ebf": col(jl["ebf"]),
            "eci": col(jl["eci"]), "ufpm": col(jl["ufpm"]),
            "ufp_rep": np.array([int(v[0]) for v in jl["ufp2fp"]], np.int64)}


def test_julia_stub_arrays_are_one_based_and_match_the_binding(pkg):
    # No device needed: the stub's arrays are exactly the 1-based arrays the Python binding
    # uploads (engine.DeviceSheet), so the library's 1-based checks accept both.
    import numpy as np
    from pssfss_b200.rwg import setup_rwg
    sheet = pkg.rectstrip(Lx=8, Ly=8, Px=10, Py=10, Nx=4, Ny=4, units=pkg.mm)
    rwg = setup_rwg(sheet)
    a = _julia_stub_sheet_arrays(sheet, rwg)
    assert a["fv"].min() == 1 and a["fv"].max() == sheet.nnode
    assert a["fe"].min() == 1 and a["fe"].max() == sheet.nedge
    assert a["ufpm"].min() == 1 and a["ufpm"].max() == rwg.nufp
    assert a["ebf"].min() == 0 and a["ebf"].max() == rwg.nbf  # 0: edge without a basis function
    assert np.array_equal(a["ufp_rep"], rwg.ufp_rep)
    assert np.array_equal(a["fv"], sheet.fv.ravel(order="F"))
    assert np.array_equal(a["bff"], rwg.bff.ravel(order="F"))


@pytest.mark.gpu
def test_julia_stub_arrays_upload_and_fill_like_the_binding(pkg):
    # The library accepts the stub's 1-based arrays, and the sheet they make fills the same
    # matrix as the binding's upload; the same arrays made 0-based (the old stub) are refused.
    import ctypes
    import numpy as np
    from pssfss_b200.layers import Layer
    from pssfss_b200.rwg import setup_rwg
    sheet = pkg.rectstrip(Lx=8, Ly=8, Px=10, Py=10, Nx=4, Ny=4, units=pkg.mm)
    rwg = setup_rwg(sheet)
    a = _julia_stub_sheet_arrays(sheet, rwg)
    L = engine.lib()
    ctx = engine.context(0)
    f64 = engine._f64

    def create(arr):
        h = ctypes.c_void_p()
        rc = L.pss_sheet_create(ctx, b"J", sheet.units.units_per_meter, engine._p(f64(sheet.s1)),
                                engine._p(f64(sheet.s2)), engine._p(f64(sheet.beta1)), engine._p(f64(sheet.beta2)),
                                sheet.nnode, engine._p(f64(sheet.rho)), sheet.nface, engine._p(arr["fv"]),
                                engine._p(arr["fe"]), engine._p(f64(sheet.fr)), sheet.nedge, rwg.nbf,
                                engine._p(arr["bff"]), engine._p(arr["ebf"]), engine._p(arr["eci"]), rwg.nufp,
                                engine._p(arr["ufpm"]), engine._p(arr["ufp_rep"]), ctypes.byref(h))
        return rc, h

    zero_based = {k: (v - 1 if k != "eci" else v) for k, v in a.items()}
    rc, _ = create(zero_based)
    assert rc == -1 and "out of range" in L.pss_last_error().decode()
    rc, h = create(a)
    assert rc == 0, L.pss_last_error().decode()
    try:
        layers = [Layer(), Layer()]
        eps, mu, w = engine.region_arrays(layers)
        n = rwg.nbf
        Z = np.zeros((n, n), complex, order="F")
        mm = ctypes.c_int()
        k0 = 2 * np.pi * 15e9 / 299792458.0
        u = 2 * np.pi / 0.01
        assert L.pss_fill_matrix(h, 2, engine._p(eps), engine._p(mu), engine._p(w), 1, u, k0, 0.0, 0.0,
                                 Z.ctypes.data_as(ctypes.c_void_p), ctypes.byref(mm)) == 0
        Zb, _ = engine.fill_matrix(sheet, rwg, layers, 1, u, k0, 0.0, 0.0)
        assert np.array_equal(Z, Zb)
    finally:
        L.pss_sheet_destroy(h)

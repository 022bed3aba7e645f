"""TEST INFRASTRUCTURE ONLY -- CPU oracle for the PSSFSS fill-and-solve path.

ctypes front end of ``pssfss_oracle.c`` (a plain-C FP64 restatement of PSSFSS.jl's
``PGF.jl``, ``Zint.jl``, ``FillZY.jl`` and ``RWG.jl:rwgbfft!``) plus the LAPACK LU/solve
and the modal projection of ``PSSFSS.jl:362-587``.  Only tests, ``__graft_entry__.smoke``
and the CPU-baseline leg of ``bench.py`` import this package; the product never does.

``analyze`` runs the whole reference analysis with the oracle's own host restatements
(``host.py``: modal and GSM algebra; ``select.py``: Gblocks, layer modes, duplicate Gblocks;
``rwg.py``: basis topology) around this fill and solve, so no code of the package under test
takes part in its numbers.

Parity is pinned against the golden values hard-coded in the reference's own tests
(test/FillZY_test.jl:45-46,77-78, test/PGF_test.jl:40-44,56-60, test/RWGData_test.jl:46-48,56-58,
collected in tests/golden/reference_golden.json) and the analytic grating of
test/full_test.jl:65-91.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.path.join(_HERE, "liboracle_pssfss.so")
_lib = None

MMAX_CAP = 2048
TWOPI = 2 * math.pi
C0 = 299792458.0


def build():
    """Compile the C restatement (``make`` in this directory)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIBPATH) or (
                os.path.getmtime(_LIBPATH) < os.path.getmtime(os.path.join(_HERE, "pssfss_oracle.c"))):
            build()
        _lib = ctypes.CDLL(_LIBPATH)
        _declare(_lib)
    return _lib


_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_L = ctypes.c_int64


def _declare(L):
    L.ora_jksums.argtypes = [_P, _D, _D, _P, _P, _I, _D, _P, _P]
    L.ora_jksums.restype = _I
    L.ora_modal_tables.argtypes = [_I, _D, _D, _D, _D, _I, _P, _P, _P, _I, _P, _P, _P, _D, _P, _P, _P]
    L.ora_modal_tables.restype = _I
    L.ora_filljk.argtypes = [_L, _P, _P, _L, _P, _D, _D, _D, _P, _P] + [_P] * 8 + [_P]
    L.ora_filljk.restype = None
    L.ora_fill.argtypes = ([_I, _D, _D, _I, _P, _P, _I, _D, _D, _L, _P, _P, _P, _P, _L, _P, _P, _P,
                            _P, _L, _P, _D, _P, _P] + [_P] * 8 + [_P, _P, _I, _P])
    L.ora_fill.restype = None
    L.ora_rwgbfft.argtypes = [_L, _P, _P, _P, _L, _P, _P, _P, _D, _P, _D, _D, _P]
    L.ora_rwgbfft.restype = None
    L.ora_sigma.argtypes = [_P, _I, _P, _P, _D, _D, _P]
    L.ora_sigma.restype = None  # returns double complex; wrapped below via a helper


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f64(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def _c128(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.complex128))


def _i64(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.int64))


def jksums(urho, psi1, psi2, us1, us2, extract=True, convtest=1e-8):
    """``PGF.jksums`` (PGF.jl:67)."""
    j = np.zeros(1, complex)
    k = np.zeros(1, complex)
    lib().ora_jksums(_p(_f64(urho)), psi1, psi2, _p(_f64(us1)), _p(_f64(us2)), int(extract),
                     convtest, _p(j), _p(k))
    return j[0], k[0]


class ModalTables:
    """Padded interpolation tables of ``electric_/magnetic_modal_sum_funcs``."""

    def __init__(self, mmax, t1, t2, b1, b2, psi1, psi2, converged):
        self.mmax, self.t1, self.t2 = mmax, t1, t2
        self.b1, self.b2, self.psi1, self.psi2 = _f64(b1), _f64(b2), psi1, psi2
        self.converged = converged

    def sigma(self, which, rho):
        """``Σm_func(ρdif)`` (PGF.jl:396-441) evaluated in numpy, same arithmetic."""
        T = self.t1 if which == 1 else self.t2
        return sigma_np(T, self.mmax, self.b1, self.b2, self.psi1, self.psi2, rho)


def sigma_np(T, mmax, b1, b2, psi1, psi2, rho):
    x1o = (b1[0] * rho[0] + b1[1] * rho[1]) / TWOPI
    x1o = 0.0 if abs(x1o) < 1e-8 else x1o
    x2o = (b2[0] * rho[0] + b2[1] * rho[1]) / TWOPI
    x2o = 0.0 if abs(x2o) < 1e-8 else x2o

    def jmod(x):
        r = math.fmod(x, 1.0)
        if r == 0:
            return 0.0
        return r + 1.0 if r < 0 else r

    x1, x2 = jmod(x1o), jmod(x2o)
    ms, ns = round(x1o - x1), round(x2o - x2)
    m = int(mmax * x1)
    p = mmax * x1 - m
    n = int(mmax * x2)
    q = mmax * x2 - n
    L = mmax + 2
    tab = T.reshape((L, L), order="F")

    def t(a, b):
        return tab[a + 1, b + 1]

    p2, q2, pq = p * p, q * q, p * q
    s = 0.5 * (q2 - q) * t(m, n - 1)
    s = s + 0.5 * (p2 - p) * t(m - 1, n)
    s = s + (((1 + pq) - p2) - q2) * t(m, n)
    s = s + 0.5 * ((p2 - 2 * pq) + p) * t(m + 1, n)
    s = s + 0.5 * ((q2 - 2 * pq) + q) * t(m, n + 1)
    s = s + pq * t(m + 1, n + 1)
    if ms != 0 or ns != 0:
        ph = -(ms * psi1 + ns * psi2)
        s = s * complex(math.cos(ph), math.sin(ph))
    return s


def _layer_arrays(layers):
    eps = _c128([l.epsr for l in layers])
    mu = _c128([l.mur for l in layers])
    w = _f64([l.width for l in layers])
    return eps, mu, w


def modal_tables(magnetic, k0, u, psi1, psi2, layers, s, b1, b2, b00, convtest=5e-12):
    """``electric_modal_sum_funcs`` / ``magnetic_modal_sum_funcs`` (PGF.jl:196, 478)."""
    eps, mu, w = _layer_arrays(layers)
    cap = (MMAX_CAP + 2) ** 2
    t1 = np.zeros(cap, complex)
    t2 = np.zeros(cap, complex)
    conv = np.zeros(1, np.int32)
    mmax = lib().ora_modal_tables(int(magnetic), k0, u, psi1, psi2, len(layers), _p(eps), _p(mu),
                                  _p(w), s, _p(_f64(b1)), _p(_f64(b2)), _p(_f64(b00)), convtest,
                                  _p(t1), _p(t2), _p(conv))
    L = (mmax + 2) ** 2
    return ModalTables(mmax, t1[:L].copy(), t2[:L].copy(), b1, b2, psi1, psi2, bool(conv[0]))


class JKCache:
    """Frequency-independent face-pair integrals of ``filljk!`` (Zint.jl:54)."""
    __slots__ = ("J", "Jxi", "Jeta", "K", "Kxi", "Keta", "rho_r", "rinv", "psi1", "psi2", "u",
                 "nonconv")


def sheet_arrays(sheet, rwg):
    return dict(rho=_f64(sheet.rho), fv=_i64(sheet.fv.ravel(order="F")),
                fe=_i64(sheet.fe.ravel(order="F")), fr=_f64(sheet.fr),
                bff=_i64(rwg.bff.ravel(order="F")), ebf=_i64(rwg.ebf), eci=_i64(rwg.eci),
                ufpm=_i64(rwg.ufpm.ravel(order="F")), rep=_i64(rwg.ufp_rep))


def filljk(sheet, rwg, ulocal, psi1, psi2):
    a = sheet_arrays(sheet, rwg)
    n = rwg.nufp
    c = JKCache()
    c.J, c.Jxi, c.Jeta, c.K, c.Kxi, c.Keta = (np.zeros(n, complex) for _ in range(6))
    c.rho_r = np.zeros(2 * n)
    c.rinv = np.zeros(n)
    nc = np.zeros(1, np.int32)
    lib().ora_filljk(sheet.nface, _p(a["rho"]), _p(a["fv"]), n, _p(a["rep"]), ulocal, psi1, psi2,
                     _p(_f64(sheet.s1)), _p(_f64(sheet.s2)), _p(c.J), _p(c.Jxi), _p(c.Jeta),
                     _p(c.K), _p(c.Kxi), _p(c.Keta), _p(c.rho_r), _p(c.rinv), _p(nc))
    c.psi1, c.psi2, c.u, c.nonconv = psi1, psi2, ulocal, int(nc[0])
    return c


_jk_cache = {}


def prime_jk_cache(sheet, jk):
    """Make ``jk`` (from ``filljk``) the cached face integrals of ``sheet`` for ``fill``."""
    _jk_cache[id(sheet)] = (sheet, jk)


def fill(k0, u, layers, s, psi1, psi2, sheet, rwg, jk=None):
    """``fillz`` (FillZY.jl:50) for class 'J' sheets, ``filly`` (FillZY.jl:273) for 'M'.

    ``layers`` are the Gblock's layers, ``s`` the 1-based interface of the sheet.
    Returns ``(Z, info)`` with Z an nbf x nbf complex128 array.
    """
    magnetic = sheet.cls == "M"
    upm = sheet.units.units_per_meter
    b1 = sheet.beta1 * upm
    b2 = sheet.beta2 * upm
    b00 = (psi1 * b1 + psi2 * b2) / TWOPI
    tabs = modal_tables(magnetic, k0, u, psi1, psi2, layers, s, b1, b2, b00, 1e-7)
    key = id(sheet)
    if jk is None:
        # the entry keeps its sheet alive, so a hit is this very sheet (an id is reused only
        # after its object is gone)
        held, jk = _jk_cache.get(key, (None, None))
        if held is not sheet:
            jk = None
        # FillZY.jl:97-99 cache test
        if (jk is None or psi1 != jk.psi1 or psi2 != jk.psi2 or jk.u == 0
                or abs((u / upm - jk.u) / jk.u) > 1e-4):
            jk = filljk(sheet, rwg, u / upm, psi1, psi2)
            if len(_jk_cache) >= 4:
                _jk_cache.clear()
            _jk_cache[key] = (sheet, jk)
    a = sheet_arrays(sheet, rwg)
    eps, mu, w = _layer_arrays(layers)
    nbf = rwg.nbf
    Z = np.zeros((nbf, nbf), complex, order="F")
    lib().ora_fill(int(magnetic), k0, u, len(layers), _p(eps), _p(mu), s, psi1, psi2, sheet.nface,
                   _p(a["rho"]), _p(a["fv"]), _p(a["fe"]), _p(a["fr"]), nbf, _p(a["bff"]),
                   _p(a["ebf"]), _p(a["eci"]), _p(a["ufpm"]), rwg.nufp, _p(a["rep"]), upm,
                   _p(_f64(b1)), _p(_f64(b2)), _p(jk.J), _p(jk.Jxi), _p(jk.Jeta), _p(jk.K),
                   _p(jk.Kxi), _p(jk.Keta), _p(jk.rho_r), _p(jk.rinv), _p(tabs.t1), _p(tabs.t2),
                   tabs.mmax, Z.ctypes.data_as(ctypes.c_void_p))
    return Z, dict(mmax=tabs.mmax, converged=tabs.converged, jk=jk)


def rwgbfft(rwg, sheet, k, psi1, psi2):
    """``rwgbfft!`` (RWG.jl:428): (nbf, 2) complex array of basis-function transforms."""
    a = sheet_arrays(sheet, rwg)
    ft = np.zeros((rwg.nbf, 2), complex)
    lib().ora_rwgbfft(sheet.nface, _p(a["rho"]), _p(a["fv"]), _p(a["fe"]), rwg.nbf, _p(a["bff"]),
                      _p(a["ebf"]), _p(a["eci"]), sheet.units.units_per_meter, _p(_f64(k)), psi1,
                      psi2, _p(ft))
    return ft


def lu_solve(Z, rhs):
    """``lu!`` + ``ldiv!`` (PSSFSS.jl:401,439): LAPACK zgetrf/zgetrs via scipy."""
    import scipy.linalg as sl
    lu, piv = sl.lu_factor(Z, check_finite=False)
    return sl.lu_solve((lu, piv), rhs, check_finite=False)


def partial_dS(sheet, rwg, region, s, k0, u, io):
    """Scattered part of one sheet's partial GSM at one point (PSSFSS.jl:391-457 for 'J',
    :516-584 for 'M'), in the host's generic mode form (see ``SheetIO``)."""
    Z, info = fill(k0, u, region, s, io.psi1, io.psi2, sheet, rwg)
    nm = len(io.wobs)
    bf = [rwgbfft(rwg, sheet, io.kvec[j], io.psi1, io.psi2) for j in range(nm)]
    rhs = np.stack([np.conj(bf[j]) @ io.src[j] for j in range(nm)], axis=1)
    X = lu_solve(Z, rhs)
    P = np.stack([bf[i] @ io.tobs[i] for i in range(nm)])
    return io.wobs[:, None] * (P @ X), Z, X


def analyze(strata, flist, steering):
    """Oracle ``analyze`` (PSSFSS.jl:114-334), independent of the package's host code.

    The selection steps - Gblocks, layer mode lists, duplicate-Gblock map - are the oracle's
    own (``select.py``: ``choose_gblocks``, ``choose_layer_modes!``, ``get_gbldup``, pinned to
    the reference's golden values of test/GSMs_test.jl and test/Modes_test.jl), and so is
    everything numeric: modal constants, incident GSMs and transmission-line Green's
    functions, source and projection factors (``host.py``), the basis-function topology
    (``rwg.py``: ``setup_rwg``, pinned by test/RWGData_test.jl), the fill and basis transforms
    (``pssfss_oracle.c``), LAPACK's LU, the cascade.  Nothing of the package runs; only its
    ``Result`` and ``GSM`` containers hold the output, so outputs can be taken from them."""
    import importlib
    from . import host
    from . import rwg as R
    from . import select as S
    O = importlib.import_module("pssfss_b200.outputs")
    Gm = importlib.import_module("pssfss_b200.gsms")
    freqs = [float(f) for f in np.atleast_1d(np.asarray(flist, float))]
    junc1, gbls, modes, gbldup = S.select(strata, freqs, lambda x: not hasattr(x, "style"))
    junc = junc1[1:]
    layers = [x for x in strata if not hasattr(x, "style")]
    sheets = [x for x in strata if hasattr(x, "style")]
    rwgdat = [None if sh.style == "NULL" else R.setup(sh) for sh in sheets]
    none = {"modes": [], "b1": np.zeros(2), "b2": np.zeros(2)}
    base = []
    for l, m in zip(layers, modes[1:]):
        m = none if m is None else m
        base.append(host.ModalLayer(l.epsr, l.mur, l.width, [p for p, _, _ in m["modes"]],
                                    [a for _, a, _ in m["modes"]], [b for _, _, b in m["modes"]],
                                    np.array(m["b1"], float), np.array(m["b2"], float)))
    sh0 = sheets[0]
    upm0 = sh0.units.units_per_meter
    points = host.steering_points(base, freqs, steering, (sh0.beta1 * upm0, sh0.beta2 * upm0))
    uvec = [0.0 if sh.style == "NULL" else
            0.5 * sh.units.units_per_meter * max(np.linalg.norm(sh.beta1), np.linalg.norm(sh.beta2))
            for sh in sheets]
    saved = {}

    def sheet_gsm(ig, p, region, s, k0):
        gj = gbls[ig][2]
        sheet = sheets[junc[gj - 1] - 1]
        if gbldup[ig] > 0:
            gb = {k: v.copy() for k, v in saved[(gbldup[ig] - 1, p)].items()}
        else:
            if sheet.cls == "E":
                gb = host.pec(region[0].nmodes, region[-1].nmodes)
            elif sheet.cls == "H":
                gb = host.pmc(region[0].nmodes, region[-1].nmodes)
            elif sheet.style == "NULL":
                gb = (host.electric_gblock if sheet.cls == "J" else host.magnetic_gblock)(region, s, k0)[0]
            else:
                upm = sheet.units.units_per_meter
                rwg = rwgdat[junc[gj - 1] - 1]
                b00 = points[p][3]
                psi1 = float(b00 @ np.asarray(sheet.s1, float)) / upm
                psi2 = float(b00 @ np.asarray(sheet.s2, float)) / upm
                Z, _ = fill(k0, uvec[junc[gj - 1] - 1], region, s, psi1, psi2, sheet, rwg)
                import scipy.linalg as sl
                lu = sl.lu_factor(Z, check_finite=False)
                ends = (region[0], region[-1])
                area = abs(sheet.s1[0] * sheet.s2[1] - sheet.s1[1] * sheet.s2[0]) / upm ** 2
                gb = host.sheet_partial_gsm(
                    sheet.cls, region, s, k0, area, lambda b: sl.lu_solve(lu, b, check_finite=False),
                    lambda r, q: rwgbfft(rwg, sheet, ends[r].beta[q], psi1, psi2))
            if gbldup[ig] < 0:
                saved[(ig, p)] = {k: v.copy() for k, v in gb.items()}
        if sheet.dx != 0 or sheet.dy != 0:
            upm = sheet.units.units_per_meter
            host.translate(gb, sheet.dx / upm, sheet.dy / upm, region[0], region[-1])
        return gb

    out = []
    for steer, f, b00, g, L in host.cascade_points(points, gbls, junc, sheet_gsm):
        gsm = Gm.GSM(g["s11"], g["s12"], g["s21"], g["s22"])
        out.append(O.Result(gsm, steer, np.array(b00, float), f, L[0].epsr, L[0].mur, L[0].beta1.copy(),
                            L[0].beta2.copy(), L[-1].epsr, L[-1].mur, L[-1].beta1.copy(), L[-1].beta2.copy()))
    return out


def partial_dS_linearized(sheet, rwg, region, s, k0, u, io, perturbed, tangent=False, form=None):
    """Scattered partial GSM at a point and, for each perturbed input set, its first-order
    (in the perturbation) value from the unperturbed factorisation:

        dS_k = wobs_k * (P_k Z^-1 R_k - Lambda^T (Z_k - Z) X),  X = Z^-1 R,  Lambda = Z^-T P^T,

    exact to O(h^2), so central differences of dS_k give dS/dp to O(h^2) with one
    factorisation.  ``tangent``: the same through forward solves only, Lambda^T (Z_k - Z) X
    = P Z^-1 (Z_k X - R).  ``form="adjoint"``: the fully linearised form
    dS_k = wobs_k * (P_k X + Lambda^T (R_k - Z_k X)), which needs no solve per set.  ``perturbed``: list of (sheet_k, rwg_k, region_k, u_k, io_k) with the
    topology of ``sheet``.  The same projection as ``partial_dS`` (PSSFSS.jl:391-457)."""
    import scipy.linalg as sl
    Z, _ = fill(k0, u, region, s, io.psi1, io.psi2, sheet, rwg)
    nm = len(io.wobs)

    def rp(sh, rw, io_):
        bf = [rwgbfft(rw, sh, io_.kvec[j], io_.psi1, io_.psi2) for j in range(nm)]
        R = np.stack([np.conj(bf[j]) @ io_.src[j] for j in range(nm)], axis=1)
        P = np.stack([bf[i] @ io_.tobs[i] for i in range(nm)])
        return R, P

    R, P = rp(sheet, rwg, io)
    lu = sl.lu_factor(Z, check_finite=False)
    X = sl.lu_solve(lu, R, check_finite=False)
    Lam = sl.lu_solve(lu, P.T, trans=1, check_finite=False)  # Z^T Lambda = P^T
    dS = io.wobs[:, None] * (P @ X)
    out = []
    for sh_k, rw_k, region_k, u_k, io_k in perturbed:
        Zk, _ = fill(k0, u_k, region_k, s, io_k.psi1, io_k.psi2, sh_k, rw_k)
        Rk, Pk = rp(sh_k, rw_k, io_k)
        Xk = sl.lu_solve(lu, Rk, check_finite=False)
        if form == "adjoint":
            out.append(io_k.wobs[:, None] * (Pk @ X + Lam.T @ (Rk - Zk @ X)))
        elif tangent:  # no transposed solve: Lambda^T (Z_k - Z) X = P Z^-1 (Z_k X - R)
            Wk = sl.lu_solve(lu, R - Zk @ X, check_finite=False)
            out.append(io_k.wobs[:, None] * (Pk @ Xk + P @ Wk))
        else:
            out.append(io_k.wobs[:, None] * (Pk @ Xk - Lam.T @ ((Zk - Z) @ X)))
    return dS, out


def partial_gsms_linearized(sheet, rwg, points, region_rng, s, u, ios, perturbed, tangent=False, form=None):
    """``partial_dS_linearized`` over the points of one sheet Gblock.  ``perturbed``: list
    of (sheet_k, rwg_k, points_k, u_k, ios_k).  Returns (dS per point, [dS_k per point])."""
    i1, i2 = region_rng
    dS, lin = [], [[] for _ in perturbed]
    for p, pt in enumerate(points):
        pk = [(sh_k, rw_k, pts_k[p].layers[i1 - 1:i2], u_k, ios_k[p])
              for sh_k, rw_k, pts_k, u_k, ios_k in perturbed]
        d, ds_k = partial_dS_linearized(sheet, rwg, pt.layers[i1 - 1:i2], s, pt.k0, u, ios[p], pk, tangent, form)
        dS.append(d)
        for k, v in enumerate(ds_k):
            lin[k].append(v)
    return dS, lin

"""TEST INFRASTRUCTURE ONLY -- independent FP64 restatement of the host-side modal and GSM
algebra of PSSFSS.jl v0.1.4, used by the oracle's ``analyze`` as a second, separately written
path next to the package's own host code.

Nothing here imports the package under test: every function works on plain numbers and
numpy arrays (a layer is a ``ModalLayer``), restated from the reference's Julia:

* ``modal_layer``             setup_modes!            (src/Modes.jl:298-322)
* ``electric_gblock``         gsm_electric_gblock     (src/GSMs.jl:213-370)
* ``magnetic_gblock``         gsm_magnetic_gblock     (src/GSMs.jl:401-526)
* ``slab_interface``          gsm_slab_interface      (src/GSMs.jl:545-620)
* ``cascade``, ``propagate``  cascade, cascade!       (src/GSMs.jl:125-176)
* ``translate``               translate_gsm!          (src/GSMs.jl:717-750)
* ``pec``, ``pmc``            pecgsm, pmcgsm          (src/GSMs.jl:47-63)
* ``sheet_partial_gsm``       the projection of calculate_jtype_gsm / calculate_mtype_gsm
                              (src/PSSFSS.jl:362-460, 486-587), given a solver callback
* ``steering_points``         the steering x frequency loop of _analyze (src/PSSFSS.jl:226-255)
* ``cascade_points``          the Gblock walk of _analyze (src/PSSFSS.jl:256-312)

A GSM is a dict {"s11", "s12", "s21", "s22"} of complex matrices.
"""
import cmath
import math
from dataclasses import dataclass

import numpy as np

MU0 = 1.25663706212e-6             # Constants.jl:6
C0 = 299792458.0                   # Constants.jl:9
EPS0 = 1.0 / (MU0 * C0 * C0)       # Constants.jl:12
ETA0 = math.sqrt(MU0 / EPS0)       # Constants.jl:15
TWOPI = 2.0 * math.pi
TE, TM = 1, 2                      # polarisation codes of the mode lists


def mysqrt(z):
    """PGF.jl:116-120: principal square root, with a purely negative-imaginary root negated."""
    r = cmath.sqrt(complex(z))
    return -r if (r.real == 0.0 and r.imag < 0.0) else r


def cross2(a, b):
    return a[0] * b[1] - a[1] * b[0]


def zhat_cross(v):
    return np.array([-v[1], v[0]], dtype=np.result_type(v, float))


def sinh_cosh(x):
    """GSMs.jl:893-901: both from one exponential."""
    e = cmath.exp(x)
    em = 1.0 / e
    return 0.5 * (e - em), 0.5 * (e + em)


@dataclass
class ModalLayer:
    """One layer's constitutive data, mode list and (after ``modal_layer``) modal constants."""
    epsr: complex
    mur: complex
    width: float                 # metres
    P: list
    M: list
    N: list
    beta1: np.ndarray            # 1/m
    beta2: np.ndarray
    beta: np.ndarray = None      # (nmodes, 2) 1/m
    gamma: np.ndarray = None
    Y: np.ndarray = None
    c: np.ndarray = None
    tvec: np.ndarray = None

    @property
    def nmodes(self):
        return len(self.P)

    def find(self, p, m, n):
        """find_mode_index (GSMs.jl:884-891), 0-based, -1 when absent."""
        for i in range(len(self.P)):
            if self.P[i] == p and self.M[i] == m and self.N[i] == n:
                return i
        return -1


def modal_layer(L, k0, b00):
    """setup_modes! (Modes.jl:298-322) on a copy of ``L``: transverse wavevector, attenuation
    constant, admittance, unit field vector and normalisation constant of every mode."""
    b00 = np.asarray(b00, float)
    nm = len(L.P)
    # layers inside a Gblock carry no modes (and no lattice): nothing to set up
    area = TWOPI ** 2 / abs(cross2(L.beta1, L.beta2)) if nm else math.inf
    ksq = k0 ** 2 * L.epsr * L.mur
    beta = np.zeros((nm, 2))
    gamma = np.zeros(nm, complex)
    Y = np.zeros(nm, complex)
    c = np.zeros(nm, complex)
    tvec = np.zeros((nm, 2))
    for i in range(nm):
        b = b00 + L.M[i] * np.asarray(L.beta1, float) + L.N[i] * np.asarray(L.beta2, float)
        bb = float(b[0] * b[0] + b[1] * b[1])
        bhat = np.array([1.0, 0.0]) if bb * area < 1e-14 else b / math.sqrt(bb)
        g = mysqrt(bb - ksq)
        if L.P[i] == TE:
            y = g / (1j * (k0 * ETA0) * L.mur)
            t = zhat_cross(bhat)
        else:
            y = 1j * (k0 / ETA0) * L.epsr / g
            t = bhat
        beta[i], gamma[i], Y[i], tvec[i] = b, g, y, t
        c[i] = mysqrt(1.0 / (area * y))
    return ModalLayer(L.epsr, L.mur, L.width, list(L.P), list(L.M), list(L.N), np.array(L.beta1, float),
                      np.array(L.beta2, float), beta, gamma, Y, c, tvec)


def _line_impedance(pol, k0, layer, gamma):
    """Modal characteristic impedance of a layer for a mode of attenuation constant gamma."""
    if pol == TE:
        return (1j * (k0 * ETA0) * layer.mur) / gamma
    return gamma / (1j * (k0 / ETA0) * layer.epsr)


def _transform(Z0, Zload, t):
    """Input impedance of a line section (Z0, tanh t) terminated in Zload."""
    return Z0 * (Zload + Z0 * t) / (Z0 + Zload * t)


def new_gsm(n1, n2):
    """GSM(n1, n2) (GSMs.jl:23-29): zero reflections, ones on the transmission diagonals."""
    s12 = np.zeros((n1, n2), complex)
    s21 = np.zeros((n2, n1), complex)
    k = min(n1, n2)
    s12[np.arange(k), np.arange(k)] = 1.0
    s21[np.arange(k), np.arange(k)] = 1.0
    return {"s11": np.zeros((n1, n1), complex), "s12": s12, "s21": s21, "s22": np.zeros((n2, n2), complex)}


def _section_params(region, pol, beta_sq, k0, idx):
    """Z0, sinh, cosh, tanh of the layers idx (0-based) for one mode (Eqs. 6.4, 6.12); the
    two semi-infinite end layers get their impedance only (their width plays no part)."""
    out = {}
    last = len(region) - 1
    for i in idx:
        L = region[i]
        g = mysqrt(beta_sq - k0 * k0 * L.mur * L.epsr)
        z = _line_impedance(pol, k0, L, g)
        if i == 0 or i == last:
            out[i] = (z, None, None, None)
            continue
        sh, ch = sinh_cosh(L.width * g)
        out[i] = (z, sh, ch, sh / ch)
    return out


def electric_gblock(region, s, k0):
    """gsm_electric_gblock (GSMs.jl:213-370).  ``region``: ModalLayers (0-based list, the
    reference's 1..N); ``s``: 1-based interface of the sheet.  Returns (gsm, tlgf, vinc), the
    last two of shape (max(n1, n2), 2)."""
    N = len(region)
    n1, n2 = region[0].nmodes, region[-1].nmodes
    gsm = new_gsm(n1, n2)
    nmax = max(n1, n2)
    vinc = np.zeros((nmax, 2), complex)
    tlgf = np.zeros((nmax, 2), complex)
    root_area = math.sqrt(abs(cross2(region[-1].beta1, region[-1].beta2) / cross2(region[0].beta1, region[0].beta2)))
    # 1-based layer numbers below, as in the reference; layer i is region[i - 1]
    for q1 in range(n1):
        pol = region[0].P[q1]
        bsq = float(region[0].beta[q1] @ region[0].beta[q1])
        sec = _section_params(region, pol, bsq, k0, range(1, N))  # layers 2..N
        Z0 = {1: 1.0 / region[0].Y[q1]}
        Z0.update({i + 1: sec[i][0] for i in sec})
        sh = {i + 1: sec[i][1] for i in sec}
        ch = {i + 1: sec[i][2] for i in sec}
        th = {i + 1: sec[i][3] for i in sec}
        Zl = {1: Z0[1]}
        for i in range(2, N):
            Zl[i] = _transform(Z0[i], Zl[i - 1], th[i])
        Zr = {N - 1: Z0[N]}
        for i in range(N - 2, 0, -1):
            Zr[i] = _transform(Z0[i + 1], Zr[i + 1], th[i + 1])
        cur = 2.0 / (Zr[1] + Z0[1])
        vol = cur * Zr[1]
        gsm["s11"][q1, q1] = vol - 1.0
        for i in range(2, s + 1):
            vol = vol * ch[i] - Z0[i] * cur * sh[i]
            cur = vol / Zr[i]
        vinc[q1, 0] = vol
        q2 = region[-1].find(pol, region[0].M[q1], region[0].N[q1])
        if q2 >= 0:
            for i in range(s + 1, N):
                vol = vol * ch[i] - Z0[i] * cur * sh[i]
                cur = vol / Zr[i]
            gsm["s21"][q2, q1] = vol * region[0].c[q1] / region[-1].c[q2] * root_area
        cur = -Zr[s] / (Zl[s] + Zr[s])
        vol = -Zl[s] * cur
        for i in range(s - 1, 0, -1):
            vol = vol * ch[i + 1] + Z0[i + 1] * cur * sh[i + 1]
            cur = -vol / Zl[i]
        tlgf[q1, 0] = vol
    for q2 in range(n2):
        pol = region[-1].P[q2]
        bsq = float(region[-1].beta[q2] @ region[-1].beta[q2])
        sec = _section_params(region, pol, bsq, k0, range(0, N - 1))  # layers 1..N-1
        Z0 = {N: 1.0 / region[-1].Y[q2]}
        Z0.update({i + 1: sec[i][0] for i in sec})
        sh = {i + 1: sec[i][1] for i in sec}
        ch = {i + 1: sec[i][2] for i in sec}
        th = {i + 1: sec[i][3] for i in sec}
        Zr = {N - 1: Z0[N]}
        for i in range(N - 1, 1, -1):
            Zr[i - 1] = _transform(Z0[i], Zr[i], th[i])
        Zl = {1: Z0[1]}
        for i in range(2, N):
            Zl[i] = _transform(Z0[i], Zl[i - 1], th[i])
        cur = -2.0 / (Zl[N - 1] + Z0[N])
        vol = -cur * Zl[N - 1]
        gsm["s22"][q2, q2] = vol - 1.0
        for i in range(N - 2, s - 1, -1):
            vol = vol * ch[i + 1] + Z0[i + 1] * cur * sh[i + 1]
            cur = -vol / Zl[i]
        vinc[q2, 1] = vol
        q1 = region[0].find(pol, region[-1].M[q2], region[-1].N[q2])
        if q1 >= 0:
            for i in range(s - 1, 0, -1):
                vol = vol * ch[i + 1] + Z0[i + 1] * cur * sh[i + 1]
                cur = -vol / Zl[i]
            gsm["s12"][q1, q2] = vol * region[-1].c[q2] / region[0].c[q1] / root_area
        cur = Zl[s] / (Zl[s] + Zr[s])
        vol = Zr[s] * cur
        for i in range(s + 1, N):
            vol = vol * ch[i] - Z0[i] * cur * sh[i]
            cur = vol / Zr[i]
        tlgf[q2, 1] = vol
    return gsm, tlgf, vinc


def magnetic_gblock(region, s, k0):
    """gsm_magnetic_gblock (GSMs.jl:401-526): the sheet is a short circuit between the two
    halves; returns (gsm, tlgf_iv, iinc)."""
    N = len(region)
    n1, n2 = region[0].nmodes, region[-1].nmodes
    gsm = new_gsm(n1, n2)
    gsm["s12"][:] = 0.0
    gsm["s21"][:] = 0.0
    nmax = max(n1, n2)
    iinc = np.zeros((nmax, 2), complex)
    tlgf = np.zeros((nmax, 2), complex)
    for q1 in range(n1):
        pol = region[0].P[q1]
        bsq = float(region[0].beta[q1] @ region[0].beta[q1])
        sec = _section_params(region, pol, bsq, k0, range(1, s))  # layers 2..s
        Z0 = {1: 1.0 / region[0].Y[q1]}
        Z0.update({i + 1: sec[i][0] for i in sec})
        sh = {i + 1: sec[i][1] for i in sec}
        ch = {i + 1: sec[i][2] for i in sec}
        th = {i + 1: sec[i][3] for i in sec}
        Zl = {1: Z0[1]}
        for i in range(2, s + 1):
            Zl[i] = _transform(Z0[i], Zl[i - 1], th[i])
        Zr = {s: 0.0 + 0.0j}
        for i in range(s - 1, 0, -1):
            Zr[i] = _transform(Z0[i + 1], Zr[i + 1], th[i + 1])
        cur = 2.0 / (1.0 + Zr[1] / Z0[1])
        vol = cur * Zr[1]
        gsm["s11"][q1, q1] = 1.0 - cur
        for i in range(2, s + 1):
            cur = cur * ch[i] - vol * sh[i] / Z0[i]
            vol = cur * Zr[i]
        iinc[q1, 0] = cur
        cur = 1.0 / Zl[s]
        vol = -1.0 + 0.0j
        for i in range(s - 1, 0, -1):
            cur = cur * ch[i + 1] + vol * sh[i + 1] / Z0[i + 1]
            vol = -cur * Zl[i]
        tlgf[q1, 0] = cur
    for q2 in range(n2):
        pol = region[-1].P[q2]
        bsq = float(region[-1].beta[q2] @ region[-1].beta[q2])
        sec = _section_params(region, pol, bsq, k0, range(s, N - 1))  # layers s+1..N-1
        Z0 = {N: 1.0 / region[-1].Y[q2]}
        Z0.update({i + 1: sec[i][0] for i in sec})
        sh = {i + 1: sec[i][1] for i in sec}
        ch = {i + 1: sec[i][2] for i in sec}
        th = {i + 1: sec[i][3] for i in sec}
        Zr = {N - 1: Z0[N]}
        for i in range(N - 1, s, -1):
            Zr[i - 1] = _transform(Z0[i], Zr[i], th[i])
        Zl = {s: 0.0 + 0.0j}
        for i in range(s + 1, N):
            Zl[i] = _transform(Z0[i], Zl[i - 1], th[i])
        cur = -2.0 / (1.0 + Zl[N - 1] / Z0[N])
        vol = -cur * Zl[N - 1]
        gsm["s22"][q2, q2] = 1.0 + cur
        for i in range(N - 2, s - 1, -1):
            cur = cur * ch[i + 1] + vol * sh[i + 1] / Z0[i + 1]
            vol = -cur * Zl[i]
        iinc[q2, 1] = cur
        cur = 1.0 / Zr[s]
        vol = 1.0 + 0.0j
        for i in range(s + 1, N):
            cur = cur * ch[i] - vol * sh[i] / Z0[i]
            vol = cur * Zr[i]
        tlgf[q2, 1] = cur
    return gsm, tlgf, iinc


def _admittance(pol, k0, layer, gamma):
    if pol == TE:
        return gamma / (1j * (k0 * ETA0) * layer.mur)
    return 1j * (k0 / ETA0) * layer.epsr / gamma


def slab_interface(L1, L2, k0):
    """gsm_slab_interface (GSMs.jl:545-620): Eqs. 3.23/3.24 per mode; a mode absent on the
    other side gets its admittance there from that side's wavenumber."""
    n1, n2 = L1.nmodes, L2.nmodes
    g = new_gsm(n1, n2)

    def other_y(src, i, dst):
        j = dst.find(src.P[i], src.M[i], src.N[i])
        if j >= 0:
            return dst.Y[j], j
        ksq = float(dst.beta[0] @ dst.beta[0]) - dst.gamma[0] ** 2
        gam = mysqrt(float(src.beta[i] @ src.beta[i]) - ksq)
        return _admittance(src.P[i], k0, dst, gam), -1

    for i1 in range(n1):
        Y1 = L1.Y[i1]
        Y2, i2 = other_y(L1, i1, L2)
        g["s11"][i1, i1] = (Y1 - Y2) / (Y2 + Y1)
        if i2 >= 0:
            g["s21"][i2, i1] = 2 * mysqrt(Y2) * mysqrt(Y1) / (Y2 + Y1)
    for i2 in range(n2):
        Y2 = L2.Y[i2]
        Y1, i1 = other_y(L2, i2, L1)
        g["s22"][i2, i2] = -((Y1 - Y2) / (Y2 + Y1))
        if i1 >= 0:
            g["s12"][i1, i2] = 2 * mysqrt(Y2) * mysqrt(Y1) / (Y2 + Y1)
    return g


def cascade(a, b):
    """Redheffer product of two GSMs (GSMs.jl:125-141, theory Eq. 3.35)."""
    I = np.eye(a["s22"].shape[0])
    g1 = np.linalg.solve(I - a["s22"] @ b["s11"], a["s21"])
    g2 = np.linalg.solve(np.eye(b["s11"].shape[0]) - b["s11"] @ a["s22"], b["s12"])
    return {"s11": a["s11"] + a["s12"] @ (b["s11"] @ g1), "s12": a["s12"] @ g2,
            "s21": b["s21"] @ g1, "s22": b["s22"] + b["s21"] @ (a["s22"] @ g2)}


def propagate(g, layer):
    """cascade!(g, layer) (GSMs.jl:154-176): the region-2 ports advanced through the layer."""
    d = layer.width
    if d == 0:
        return g
    p = np.exp(-layer.gamma * d)
    g["s12"] = g["s12"] * p[None, :]
    g["s21"] = g["s21"] * p[:, None]
    g["s22"] = g["s22"] * p[None, :] * p[:, None]
    return g


def translate(g, dx, dy, L1, L2):
    """translate_gsm! (GSMs.jl:717-750)."""
    t1 = np.exp(1j * (L1.beta @ np.array([dx, dy])))
    t2 = np.exp(1j * (L2.beta @ np.array([dx, dy])))
    g["s11"] = g["s11"] * (t1[None, :] / t1[:, None])
    g["s12"] = g["s12"] * (t2[None, :] / t1[:, None])
    g["s21"] = g["s21"] * (t1[None, :] / t2[:, None])
    g["s22"] = g["s22"] * (t2[None, :] / t2[:, None])
    return g


def pec(n1, n2):
    g = new_gsm(n1, n2)
    g["s11"][np.diag_indices(n1)] = -1.0
    g["s22"][np.diag_indices(n2)] = -1.0
    g["s12"][:] = 0.0
    g["s21"][:] = 0.0
    return g


def pmc(n1, n2):
    g = pec(n1, n2)
    g["s11"] = -g["s11"]
    g["s22"] = -g["s22"]
    return g


def sheet_partial_gsm(cls, region, s, k0, area, solve, transforms):
    """calculate_jtype_gsm (PSSFSS.jl:362-460) for cls 'J', calculate_mtype_gsm
    (PSSFSS.jl:486-587) for 'M': the incident partial GSM of the Gblock plus the scattered
    part of the sheet, written in the reference's own terms (vinc·c·acf·t source vectors,
    Eq. 6.18 projection with tlgfvi/(c·acf·A); iinc·c·Y·(ẑ×t) and Eq. 6.37 with σ·tlgfiv·c).

    ``area``: unit-cell area (m²); ``solve(rhs)`` returns Z⁻¹ rhs for an (nbf, k) block;
    ``transforms(r, q)`` the basis-function transforms (nbf, 2) at mode q of end region r
    (0: region 1, 1: region N)."""
    ends = (region[0], region[-1])
    acf = [math.sqrt((TWOPI * TWOPI / abs(cross2(l.beta1, l.beta2))) / area) for l in ends]
    if cls == "J":
        gsm, tlgf, vinc = electric_gblock(region, s, k0)
    else:
        gsm, tlgf, vinc = magnetic_gblock(region, s, k0)
    F = [[transforms(r, q) for q in range(l.nmodes)] for r, l in enumerate(ends)]
    blocks = {(0, 0): "s11", (0, 1): "s12", (1, 0): "s21", (1, 1): "s22"}
    for sr, ls in enumerate(ends):
        sigma = 1.0 if sr == 0 else -1.0
        cols = []
        for qp in range(ls.nmodes):
            if cls == "J":
                src = vinc[qp, sr] * ls.c[qp] * acf[sr] * ls.tvec[qp]
            else:
                src = vinc[qp, sr] * ls.c[qp] * ls.Y[qp] * zhat_cross(ls.tvec[qp])
            cols.append(np.conj(F[sr][qp]) @ src)  # b ⋅ sourcevec conjugates b
        X = solve(np.stack(cols, axis=1))
        for orr, lo in enumerate(ends):
            S = gsm[blocks[(orr, sr)]]
            for q in range(lo.nmodes):
                FT = F[orr][q].T @ X  # (2, nmodes of sr): transform of each solution's current
                if cls == "J":
                    S[q, :] -= (lo.tvec[q] @ FT) * (tlgf[q, orr] / (lo.c[q] * acf[orr] * area))
                else:
                    S[q, :] += (zhat_cross(lo.tvec[q]) @ FT) * (sigma * tlgf[q, orr] * lo.c[q])
    return gsm


def steering_points(layers, freqs, steering, sheet0_beta):
    """The steering x frequency loop of _analyze (PSSFSS.jl:226-255): per kept point
    (steer, fghz, k0, beta00, modal layers).  ``layers``: ModalLayers with mode lists;
    ``steering``: ordered dict of two keys ((θ, ϕ) or (ψ₁, ψ₂), degrees; the first is the
    outer loop); ``sheet0_beta``: (β₁, β₂) of the first sheet in 1/m, for ψ steering."""
    keys = list(steering.keys())
    vals = [list(np.atleast_1d(np.asarray(steering[k], float))) for k in keys]
    phi_keys = ("phi", "ϕ", "Phi", "PHI", "Φ")
    psi1_keys = ("psi1", "Psi1", "PSI1", "ψ₁", "Ψ₁", "ψ1", "Ψ1")
    out = []
    for vo in vals[0]:
        for vi in vals[1]:
            if keys[0] in phi_keys:
                steer = {"θ": vi, "ϕ": vo}
            elif keys[1] in phi_keys:
                steer = {"θ": vo, "ϕ": vi}
            elif keys[0] in psi1_keys:
                steer = {"ψ₁": vo, "ψ₂": vi}
            else:
                steer = {"ψ₁": vi, "ψ₂": vo}
            for f in freqs:
                k0 = TWOPI * float(f) * 1e9 / C0
                if "θ" in steer:
                    k1 = k0 * math.sqrt((layers[0].epsr * layers[0].mur).real)
                    th = math.radians(steer["θ"])
                    ph = math.radians(steer["ϕ"])
                    st = 0.0 if steer["θ"] % 180 == 0 else math.sin(th)
                    sp = 0.0 if steer["ϕ"] % 180 == 0 else math.sin(ph)
                    cp = 0.0 if (steer["ϕ"] - 90) % 180 == 0 else math.cos(ph)
                    b00 = np.array([k1 * st * cp, k1 * st * sp])
                else:
                    p1, p2 = math.radians(steer["ψ₁"]), math.radians(steer["ψ₂"])
                    b00 = (p1 * np.asarray(sheet0_beta[0]) + p2 * np.asarray(sheet0_beta[1])) / TWOPI
                ml = [modal_layer(l, k0, b00) for l in layers]
                a0, a1 = cmath.phase(ml[0].gamma[0]), cmath.phase(ml[-1].gamma[0])
                if not (math.isclose(a0, a1, rel_tol=math.sqrt(np.finfo(float).eps))
                        and math.isclose(a1, math.pi / 2, rel_tol=math.sqrt(np.finfo(float).eps))):
                    continue
                out.append((steer, float(f), k0, b00, ml))
    return out


def cascade_points(points, gbls, junc, sheet_gsm):
    """The Gblock walk of _analyze (PSSFSS.jl:256-312) for every point.  ``gbls``: list of
    (first, last, j) 1-based layer range and junction (j = 0: bare interface); ``junc``: the
    sheet index (1-based, 0 none) per junction; ``sheet_gsm(ig, p, region, s, k0)`` returns
    the Gblock's GSM (the sheet's partial GSM, or a PEC/PMC one), already translated."""
    out = []
    for p, (steer, f, k0, b00, L) in enumerate(points):
        n1 = L[0].nmodes
        ga = propagate(new_gsm(n1, n1), L[0])
        gc = ga
        for ig, (first, last, j) in enumerate(gbls):
            i1, i2 = first, last + 1
            if j != 0:
                gb = sheet_gsm(ig, p, L[i1 - 1:i2], j - i1 + 1, k0)
            else:
                gb = slab_interface(L[i1 - 1], L[i2 - 1], k0)
            gc = propagate(cascade(ga, gb), L[i2 - 1])
            ga = gc
        out.append((steer, f, b00, gc, L))
    return out

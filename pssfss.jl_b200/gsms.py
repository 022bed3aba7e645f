"""Generalized scattering matrices (PSSFSS.jl ``src/GSMs.jl``).

Host-side: ``GSM`` (``:16-29``), ``cascade`` (``:125-141``), ``cascade_layer``
(``cascade!``, ``:155-176``), the incident partial GSMs and transmission-line Green's
functions of a Gblock (``gsm_electric_gblock`` ``:213-370``, ``gsm_magnetic_gblock``
``:401-526``), ``gsm_slab_interface`` (``:545-620``), ``translate_gsm`` (``:717-750``),
``choose_gblocks`` (``:771-868``), ``find_mode_index`` (``:884-891``) and the GSM files
(``:623-696``).  These are
per-mode scalar recursions and n_modes-sized dense algebra; the O(N^2)/O(N^3) work of a
sheet's partial GSM is done by the CUDA library.
"""
import cmath
import math

import numpy as np

from .constants import ETA0, MIN_ELENGTH
from .layers import TE, TM


def mysqrt(z):
    """``PGF.mysqrt`` (PGF.jl:116-120): principal root, flipped if pure negative imaginary."""
    z = complex(z)
    a = cmath.sqrt(z)
    if a.real == 0 and a.imag < 0:
        a = complex(-a.real, -a.imag)
    return a


def _rsubc(x, z):
    """Julia ``Real - Complex`` (keeps the sign of the zero imaginary part)."""
    return complex(x - z.real, -z.imag)


def _rmulc(x, z):
    """Julia ``Real * Complex`` (no promotion of ``x`` to complex, keeps signed zeros)."""
    return complex(x * z.real, x * z.imag)


class GSM:
    def __init__(self, s11, s12, s21, s22):
        self.s11, self.s12, self.s21, self.s22 = s11, s12, s21, s22

    @classmethod
    def identity(cls, n1, n2):
        """``GSM(n1, n2)`` (GSMs.jl:23-29): zero reflection, unit-diagonal transmission."""
        s12 = np.zeros((n1, n2), complex)
        s21 = np.zeros((n2, n1), complex)
        k = min(n1, n2)
        s12[range(k), range(k)] = 1
        s21[range(k), range(k)] = 1
        return cls(np.zeros((n1, n1), complex), s12, s21, np.zeros((n2, n2), complex))

    def __getitem__(self, ij):
        return {(1, 1): self.s11, (1, 2): self.s12, (2, 1): self.s21, (2, 2): self.s22}[ij]

    def copy(self):
        return GSM(self.s11.copy(), self.s12.copy(), self.s21.copy(), self.s22.copy())


def pecgsm(n1, n2):
    g = GSM.identity(n1, n2)
    g.s11[np.diag_indices(n1)] = -1
    g.s22[np.diag_indices(n2)] = -1
    g.s12[:] = 0
    g.s21[:] = 0
    return g


def pmcgsm(n1, n2):
    g = GSM.identity(n1, n2)
    g.s11[np.diag_indices(n1)] = 1
    g.s22[np.diag_indices(n2)] = 1
    g.s12[:] = 0
    g.s21[:] = 0
    return g


def cascade(a, b):
    """Redheffer star product of two GSMs (GSMs.jl:125-141, Eq. 3.35)."""
    n2a = a.s22.shape[1]
    n1b = b.s11.shape[0]
    if n1b != n2a:
        raise ValueError("Non-conformable arrays")
    I = np.eye(n1b)
    g1 = np.linalg.solve(I - a.s22 @ b.s11, a.s21)
    s21 = b.s21 @ g1
    s11 = a.s11 + a.s12 @ (b.s11 @ g1)
    g2 = np.linalg.solve(I - b.s11 @ a.s22, b.s12)
    s12 = a.s12 @ g2
    s22 = b.s22 + b.s21 @ (a.s22 @ g2)
    return GSM(s11, s12, s21, s22)


def cascade_layer(a, layer, t=None):
    """``cascade!`` (GSMs.jl:155-176): propagate side-2 ports through ``layer``."""
    n2 = a.s22.shape[0]
    if n2 != len(layer.gamma):
        raise ValueError("# modes not consistent")
    d = layer.width if t is None else layer.user_width.unit.to_meters(t)
    if d == 0:
        return a
    for i in range(n2):
        p = cmath.exp(-layer.gamma[i] * d)
        a.s12[:, i] *= p
        a.s21[i, :] *= p
        a.s22[:, i] *= p
        a.s22[i, :] *= p
    return a


def find_mode_index(p, m, n, layer):
    for i in range(len(layer.P)):
        if layer.P[i] == p and layer.M[i] == m and layer.N[i] == n:
            return i + 1
    return 0


def sinhcosh(x):
    """GSMs.jl:893-901."""
    ex = cmath.exp(x)
    emx = 1 / ex
    return 0.5 * (ex - emx), 0.5 * (ex + emx)


def _zdotcross(a, b):
    return a[0] * b[1] - a[1] * b[0]


def gsm_electric_gblock(layers, s, k0):
    """Incident partial GSM, ``tlgfvi`` and ``vincs`` of a J-type Gblock (GSMs.jl:213-370).

    ``layers`` is the Gblock's layer list, ``s`` the 1-based sheet interface.
    """
    N = len(layers)
    cosha = [0j] * (N + 1)
    sinha = [0j] * (N + 1)
    tanha = [0j] * (N + 1)
    Z0 = [0j] * (N + 1)
    Zleft = [0j] * (N + 1)
    Zright = [0j] * (N + 1)
    k0sq = k0 * k0
    L1, LN = layers[0], layers[N - 1]
    n1, n2 = len(L1.P), len(LN.P)
    gsm = GSM.identity(n1, n2)
    nmax = max(n1, n2)
    vincs = np.zeros((nmax, 2), complex)
    tlgfvi = np.zeros((nmax, 2), complex)
    root_area1oN = math.sqrt(abs(_zdotcross(LN.beta1, LN.beta2) / _zdotcross(L1.beta1, L1.beta2)))
    for q1 in range(n1):
        Z0[1] = 1 / L1.Y[q1]
        Zleft[1] = Z0[1]
        bsq = L1.beta[q1][0] * L1.beta[q1][0] + L1.beta[q1][1] * L1.beta[q1][1]
        for i in range(2, N + 1):
            Li = layers[i - 1]
            ksq = _rmulc(k0sq, Li.mur) * Li.epsr
            g = mysqrt(_rsubc(bsq, ksq))
            if L1.P[q1] == TE:
                Z0[i] = (1j * (k0 * ETA0) * Li.mur) / g
            else:
                Z0[i] = g / (1j * (k0 / ETA0) * Li.epsr)
            if i < N:
                sinha[i], cosha[i] = sinhcosh(Li.width * g)
                tanha[i] = sinha[i] / cosha[i]
                Zleft[i] = Z0[i] * (Zleft[i - 1] + Z0[i] * tanha[i]) / (Z0[i] + Zleft[i - 1] * tanha[i])
        Zright[N - 1] = Z0[N]
        for i in range(N - 2, 0, -1):
            Zright[i] = Z0[i + 1] * (Zright[i + 1] + Z0[i + 1] * tanha[i + 1]) / \
                (Z0[i + 1] + Zright[i + 1] * tanha[i + 1])
        current = 2 / (Zright[1] + Z0[1])
        voltage = current * Zright[1]
        gsm.s11[q1, q1] = voltage - 1
        for i in range(2, s + 1):
            voltage = voltage * cosha[i] - Z0[i] * current * sinha[i]
            current = voltage / Zright[i]
        vincs[q1, 0] = voltage
        q2 = find_mode_index(L1.P[q1], L1.M[q1], L1.N[q1], LN)
        if q2 != 0:
            for i in range(s + 1, N):
                voltage = voltage * cosha[i] - Z0[i] * current * sinha[i]
                current = voltage / Zright[i]
            gsm.s21[q2 - 1, q1] = voltage * L1.c[q1] / LN.c[q2 - 1] * root_area1oN
        current = -Zright[s] / (Zleft[s] + Zright[s])
        voltage = -Zleft[s] * current
        for i in range(s - 1, 0, -1):
            voltage = voltage * cosha[i + 1] + Z0[i + 1] * current * sinha[i + 1]
            current = -voltage / Zleft[i]
        tlgfvi[q1, 0] = voltage
    for q2 in range(n2):
        Z0[N] = 1 / LN.Y[q2]
        Zright[N - 1] = Z0[N]
        bsq = LN.beta[q2][0] * LN.beta[q2][0] + LN.beta[q2][1] * LN.beta[q2][1]
        for i in range(N - 1, 0, -1):
            Li = layers[i - 1]
            ksq = _rmulc(k0sq, Li.mur) * Li.epsr
            g = mysqrt(_rsubc(bsq, ksq))
            if LN.P[q2] == TE:
                Z0[i] = (1j * (k0 * ETA0) * Li.mur) / g
            else:
                Z0[i] = g / (1j * (k0 / ETA0) * Li.epsr)
            if i > 1:
                sinha[i], cosha[i] = sinhcosh(Li.width * g)
                tanha[i] = sinha[i] / cosha[i]
                Zright[i - 1] = Z0[i] * (Zright[i] + Z0[i] * tanha[i]) / (Z0[i] + Zright[i] * tanha[i])
        Zleft[1] = Z0[1]
        for i in range(2, N):
            Zleft[i] = Z0[i] * (Zleft[i - 1] + Z0[i] * tanha[i]) / (Z0[i] + Zleft[i - 1] * tanha[i])
        current = -2 / (Zleft[N - 1] + Z0[N])
        voltage = -current * Zleft[N - 1]
        gsm.s22[q2, q2] = voltage - 1
        for i in range(N - 2, s - 1, -1):
            voltage = voltage * cosha[i + 1] + Z0[i + 1] * current * sinha[i + 1]
            current = -voltage / Zleft[i]
        vincs[q2, 1] = voltage
        q1 = find_mode_index(LN.P[q2], LN.M[q2], LN.N[q2], L1)
        if q1 != 0:
            for i in range(s - 1, 0, -1):
                voltage = voltage * cosha[i + 1] + Z0[i + 1] * current * sinha[i + 1]
                current = -voltage / Zleft[i]
            gsm.s12[q1 - 1, q2] = voltage * LN.c[q2] / L1.c[q1 - 1] / root_area1oN
        current = Zleft[s] / (Zleft[s] + Zright[s])
        voltage = Zright[s] * current
        for i in range(s + 1, N):
            voltage = voltage * cosha[i] - Z0[i] * current * sinha[i]
            current = voltage / Zright[i]
        tlgfvi[q2, 1] = voltage
    return gsm, tlgfvi, vincs


def gsm_magnetic_gblock(layers, s, k0):
    """Incident partial GSM, ``tlgfiv`` and ``iincs`` of an M-type Gblock (GSMs.jl:401-526)."""
    N = len(layers)
    cosha = [0j] * (N + 1)
    sinha = [0j] * (N + 1)
    tanha = [0j] * (N + 1)
    Z0 = [0j] * (N + 1)
    Zleft = [0j] * (N + 1)
    Zright = [0j] * (N + 1)
    k0sq = k0 * k0
    L1, LN = layers[0], layers[N - 1]
    n1, n2 = len(L1.P), len(LN.P)
    gsm = GSM.identity(n1, n2)
    gsm.s12[:] = 0
    gsm.s21[:] = 0
    nmax = max(n1, n2)
    iincs = np.zeros((nmax, 2), complex)
    tlgfiv = np.zeros((nmax, 2), complex)
    for q1 in range(n1):
        Z0[1] = 1 / L1.Y[q1]
        Zleft[1] = Z0[1]
        bsq = L1.beta[q1][0] * L1.beta[q1][0] + L1.beta[q1][1] * L1.beta[q1][1]
        for i in range(2, s + 1):
            Li = layers[i - 1]
            ksq = _rmulc(k0sq, Li.mur) * Li.epsr
            g = mysqrt(_rsubc(bsq, ksq))
            if L1.P[q1] == TE:
                Z0[i] = (1j * (k0 * ETA0) * Li.mur) / g
            else:
                Z0[i] = g / (1j * (k0 / ETA0) * Li.epsr)
            sinha[i], cosha[i] = sinhcosh(Li.width * g)
            tanha[i] = sinha[i] / cosha[i]
            Zleft[i] = Z0[i] * (Zleft[i - 1] + Z0[i] * tanha[i]) / (Z0[i] + Zleft[i - 1] * tanha[i])
        Zright[s] = 0j
        for i in range(s - 1, 0, -1):
            Zright[i] = Z0[i + 1] * (Zright[i + 1] + Z0[i + 1] * tanha[i + 1]) / \
                (Z0[i + 1] + Zright[i + 1] * tanha[i + 1])
        current = 2 / (1 + Zright[1] / Z0[1])
        voltage = current * Zright[1]
        gsm.s11[q1, q1] = 1 - current
        for i in range(2, s + 1):
            current = current * cosha[i] - voltage * sinha[i] / Z0[i]
            voltage = current * Zright[i]
        iincs[q1, 0] = current
        current = 1 / Zleft[s]
        voltage = -1 + 0j
        for i in range(s - 1, 0, -1):
            current = current * cosha[i + 1] + voltage * sinha[i + 1] / Z0[i + 1]
            voltage = -current * Zleft[i]
        tlgfiv[q1, 0] = current
    for q2 in range(n2):
        Z0[N] = 1 / LN.Y[q2]
        Zright[N - 1] = Z0[N]
        bsq = LN.beta[q2][0] * LN.beta[q2][0] + LN.beta[q2][1] * LN.beta[q2][1]
        for i in range(N - 1, s, -1):
            Li = layers[i - 1]
            ksq = _rmulc(k0sq, Li.mur) * Li.epsr
            g = mysqrt(_rsubc(bsq, ksq))
            if LN.P[q2] == TE:
                Z0[i] = (1j * (k0 * ETA0) * Li.mur) / g
            else:
                Z0[i] = g / (1j * k0 / ETA0 * Li.epsr)
            sinha[i], cosha[i] = sinhcosh(Li.width * g)
            tanha[i] = sinha[i] / cosha[i]
            Zright[i - 1] = Z0[i] * (Zright[i] + Z0[i] * tanha[i]) / (Z0[i] + Zright[i] * tanha[i])
        Zleft[s] = 0j
        for i in range(s + 1, N):
            Zleft[i] = Z0[i] * (Zleft[i - 1] + Z0[i] * tanha[i]) / (Z0[i] + Zleft[i - 1] * tanha[i])
        current = -2 / (1 + Zleft[N - 1] / Z0[N])
        voltage = -current * Zleft[N - 1]
        gsm.s22[q2, q2] = 1 + current
        for i in range(N - 2, s - 1, -1):
            current = current * cosha[i + 1] + voltage * sinha[i + 1] / Z0[i + 1]
            voltage = -current * Zleft[i]
        iincs[q2, 1] = current
        current = 1 / Zright[s]
        voltage = 1 + 0j
        for i in range(s + 1, N):
            current = current * cosha[i] - voltage * sinha[i] / Z0[i]
            voltage = current * Zright[i]
        tlgfiv[q2, 1] = current
    return gsm, tlgfiv, iincs


def gsm_slab_interface(L1, L2, k0):
    """GSM of a bare dielectric junction (GSMs.jl:545-620, Eqs. 3.23-3.24)."""
    n1, n2 = len(L1.P), len(L2.P)
    g = GSM.identity(n1, n2)
    for i1 in range(n1):
        Y1 = L1.Y[i1]
        i2 = find_mode_index(L1.P[i1], L1.M[i1], L1.N[i1], L2)
        if i2 == 0:
            k2sq = (L2.beta[0][0] * L2.beta[0][0] + L2.beta[0][1] * L2.beta[0][1]) - L2.gamma[0] ** 2
            bsq = L1.beta[i1][0] * L1.beta[i1][0] + L1.beta[i1][1] * L1.beta[i1][1]
            gm = mysqrt(bsq - k2sq)
            Y2 = gm / (1j * (k0 * ETA0) * L2.mur) if L1.P[i1] == TE else 1j * (k0 / ETA0) * L2.epsr / gm
        else:
            Y2 = L2.Y[i2 - 1]
        g.s11[i1, i1] = (Y1 - Y2) / (Y2 + Y1)
        if i2 != 0:
            g.s21[i2 - 1, i1] = 2 * mysqrt(Y2) * mysqrt(Y1) / (Y2 + Y1)
    for i2 in range(n2):
        Y2 = L2.Y[i2]
        i1 = find_mode_index(L2.P[i2], L2.M[i2], L2.N[i2], L1)
        if i1 == 0:
            k1sq = (L1.beta[0][0] * L1.beta[0][0] + L1.beta[0][1] * L1.beta[0][1]) - L1.gamma[0] ** 2
            bsq = L2.beta[i2][0] * L2.beta[i2][0] + L2.beta[i2][1] * L2.beta[i2][1]
            gm = mysqrt(bsq - k1sq)
            Y1 = gm / (1j * (k0 * ETA0) * L1.mur) if L2.P[i2] == TE else 1j * (k0 / ETA0) * L1.epsr / gm
        else:
            Y1 = L1.Y[i1 - 1]
        g.s22[i2, i2] = -(Y1 - Y2) / (Y2 + Y1)
        if i1 != 0:
            g.s12[i1 - 1, i2] = 2 * mysqrt(Y2) * mysqrt(Y1) / (Y2 + Y1)
    return g


def translate_gsm(g, dx, dy, layer1, layer2):
    """Phase shift a GSM for a translated structure (GSMs.jl:717-750)."""
    t1 = np.array([cmath.exp(1j * (b[0] * dx + b[1] * dy)) for b in layer1.beta])
    t2 = np.array([cmath.exp(1j * (b[0] * dx + b[1] * dy)) for b in layer2.beta])
    g.s11 *= t1[None, :] / t1[:, None]
    g.s12 *= t2[None, :] / t1[:, None]
    g.s21 *= t1[None, :] / t2[:, None]
    g.s22 *= t2[None, :] / t2[:, None]
    return g


class Gblock:
    """A GSM building block (GSMs.jl:91-107): interfaces ``rng`` (1-based, inclusive
    range as (first, last)) with the sheet at interface ``j`` (0 if none)."""

    def __init__(self, first, last, j):
        if last < first:
            raise ValueError("rng must have positive length")
        if j < 0:
            raise ValueError(f"negative integer j = {j}")
        if j == 0 and last != first:
            raise ValueError("length(rng) must be 1 when j==0")
        if j != 0 and not first <= j <= last:
            raise ValueError(f"j={j} is not a member of rng")
        self.first, self.last, self.j = first, last, j

    @property
    def rng(self):
        return range(self.first, self.last + 1)

    def __eq__(self, o):
        return (self.first, self.last, self.j) == (o.first, o.last, o.j)

    def __repr__(self):
        return f"Gblock({self.first}:{self.last}, {self.j})"


def find_unique_periods(junc, sheets):
    """``find_unique_periods`` (Sheets.jl:139-169)."""
    rows = []
    for sh in sheets:
        upm = sh.units.units_per_meter
        v = [sh.s1[0] / upm, sh.s1[1] / upm, sh.s2[0] / upm, sh.s2[1] / upm]
        rows.append(tuple(float(f"{x:.8g}") for x in v))
    upa = [0] * len(junc)
    nup = 0
    for i in range(len(upa)):
        isht = junc[i]
        if isht == 0 or sheets[isht - 1].style == "NULL":
            continue
        found = False
        for n in range(1, nup + 1):
            nsht = junc[upa.index(n)]
            if rows[isht - 1] == rows[nsht - 1]:
                upa[i] = n
                found = True
                break
        if not found:
            nup += 1
            upa[i] = nup
    return upa


def choose_gblocks(layers, sheets, junc, k0min):
    """Partition the interfaces into Gblocks (GSMs.jl:771-868).  ``junc`` is 1-based sheet
    numbers per interface (0 for none)."""
    nl = len(layers)
    nj = nl - 1
    ns = len(sheets)
    if ns == 0 or all(t.style == "NULL" for t in sheets):
        return [Gblock(i, i, 0 if junc[i - 1] == 0 else i) for i in range(1, nj + 1)]
    elength = [k0min * l.width * math.sqrt((l.epsr * l.mur).real) for l in layers]
    sint = [i + 1 for i in range(nj) if junc[i] != 0]
    owner = list(range(1, nj + 1))
    E = lambda j: elength[j - 1]

    def sty(j):
        return sheets[junc[j - 1] - 1].style

    if sheets[0].style != "NULL":
        for j in range(sint[0], 1, -1):
            if E(j) > MIN_ELENGTH:
                break
            owner[j - 2] = sint[0]
    if sheets[-1].style != "NULL":
        for j in range(1 + sint[ns - 1], nj + 1):
            if E(j) > MIN_ELENGTH:
                break
            owner[j - 1] = sint[-1]
    for i in range(ns - 1):
        j1, j2 = sint[i], sint[i + 1]
        nwide = sum(1 for j in range(j1 + 1, j2 + 1) if E(j) > MIN_ELENGTH)
        if nwide > 0:
            for j in range(j2, j1, -1):
                if E(j) > MIN_ELENGTH or sty(j2) == "NULL":
                    break
                owner[j - 2] = j2
            for j in range(j1 + 1, j2 + 1):
                if E(j) > MIN_ELENGTH or sty(j1) == "NULL":
                    break
                owner[j - 1] = j1
        else:
            if sty(j1) == "NULL" and sty(j2) != "NULL":
                for j in range(j1 + 1, j2 + 1):
                    owner[j - 1] = j2
                continue
            elif sty(j1) != "NULL" and sty(j2) == "NULL":
                for j in range(j1, j2):
                    owner[j - 1] = j1
                continue
            elif sty(j1) == "NULL" and sty(j2) == "NULL":
                continue
            elmax = max(E(j) for j in range(j1 + 1, j2 + 1))
            best = [j for j in range(1, nl + 1) if E(j) == elmax and j1 + 1 <= j <= j2]
            mid = (j1 + j2 + 1) // 2
            dist = [abs(b - mid) for b in best]
            lb = best[dist.index(min(dist))]
            for j in range(j1, lb):
                owner[j - 1] = j1
            for j in range(lb, j2 + 1):
                owner[j - 1] = j2
    ngbl = 1 + sum(1 for j in range(2, nj + 1) if owner[j - 1] != owner[j - 2])
    gbl = [[1, 1, 0] for _ in range(ngbl)]
    jg = 0
    for j in range(1, nj + 1):
        if owner[j - 1] == owner[gbl[jg][0] - 1]:
            gbl[jg][1] = j
        else:
            jg += 1
            gbl[jg] = [j, j, 0]
        if junc[j - 1] != 0:
            gbl[jg][2] = j
    out = [Gblock(a, b, c) for a, b, c in gbl]
    cover = [j for g in out for j in g.rng]
    if cover != list(range(1, nj + 1)):
        raise RuntimeError(f"Bad Gblock vector: {out}")
    return out


# GSM files (GSMs.jl:623-700): a header with the end regions' unit cells and mode lists, then
# one group per frequency / scan case.  The reference writes JLD2; here the same keys are
# kept in a pickled dict.
def _load_gsm_dict(fname):
    import pickle
    with open(fname, "rb") as f:
        return pickle.load(f)


def _save_gsm_dict(fname, dat):
    import pickle
    with open(fname, "wb") as f:
        pickle.dump(dat, f)


def initialize_gsm_file(fname, layer1, layer2, sh1=None, sh2=None):
    """Start a GSM file with the unit cells of the input and output regions (a 1 m square
    cell when no sheets are given) and their mode lists (``GSMs.jl:623-665``)."""
    if (sh1 is None) != (sh2 is None):
        raise ValueError("give both sheets or neither")
    cells = []
    for sh in (sh1, sh2):
        if sh is None:
            cells.append((np.array([1.0, 0.0]), np.array([0.0, 1.0]), "m"))
        else:
            cells.append((np.array(sh.s1, float), np.array(sh.s2, float), sh.units))
    _save_gsm_dict(fname, {
        "FileType": "GSMFile", "FileTypeVersion": "0.0.1",
        "s1in": cells[0][0], "s2in": cells[0][1], "unitsin": cells[0][2],
        "s1out": cells[1][0], "s2out": cells[1][1], "unitsout": cells[1][2],
        "ModelistIn": (list(layer1.P), list(layer1.M), list(layer1.N)),
        "ModelistOut": (list(layer2.P), list(layer2.M), list(layer2.N)),
    })


def append_gsm_data(fname, gname, gsm, l1, l2, case):
    """Add the GSM of one frequency / scan case (``case``: "FGHz" and θ, ϕ or ψ₁, ψ₂) under
    group ``gname``, with the end regions' (εr, μr) (``GSMs.jl:667-690``)."""
    dat = read_gsm_file(fname)
    dat[f"{gname}/case"] = dict(case)
    dat[f"{gname}/epsmu1"] = (complex(l1.epsr), complex(l1.mur))
    dat[f"{gname}/epsmu2"] = (complex(l2.epsr), complex(l2.mur))
    dat[f"{gname}/gsm"] = gsm
    _save_gsm_dict(fname, dat)


def read_gsm_file(fname):
    """The contents of a GSM file as a dict keyed like the reference's (``GSMs.jl:692-696``)."""
    dat = _load_gsm_dict(fname)
    if dat.get("FileType") != "GSMFile":
        raise ValueError(f"{fname} is not a GSM file")
    return dat

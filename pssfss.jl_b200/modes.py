"""Floquet mode selection and per-frequency modal constants (PSSFSS.jl ``src/Modes.jl``).

``choose_layer_modes`` (``:49-275``), ``setup_modes`` (``:298-322``), ``fill_mmax_pmn``
(``:367-382``), ``select_pmn`` (``:399-431``).
"""
import math

import numpy as np

from .constants import DBMIN, ETA0, TWOPI
from .gsms import _rmulc, find_unique_periods, mysqrt
from .layers import TE, TM
from .rings import Ring

MNMAX_DEFAULT = 6


def zhatcross(v):
    return np.array([-v[1], v[0]])


def setup_modes(layer, k0, kvec):
    """Fill ``β``, ``γ``, ``Y``, ``c`` and ``tvec`` of ``layer`` (Modes.jl:298-322)."""
    b00 = np.array([kvec[0], kvec[1]], float)
    b1, b2 = layer.beta1, layer.beta2
    cross = abs(b1[0] * b2[1] - b1[1] * b2[0])
    # layers inside a Gblock carry no modes and no lattice: their area is never used
    area = TWOPI ** 2 / cross if cross != 0 else math.inf
    ksq = _rmulc(k0 * k0, layer.epsr) * layer.mur
    n = len(layer.M)
    layer.beta = np.zeros((n, 2))
    layer.gamma = np.zeros(n, complex)
    layer.Y = np.zeros(n, complex)
    layer.c = np.zeros(n, complex)
    layer.tvec = np.zeros((n, 2))
    for mode in range(n):
        m, nn, p = layer.M[mode], layer.N[mode], layer.P[mode]
        beta = np.array([(b00[0] + m * b1[0]) + nn * b2[0], (b00[1] + m * b1[1]) + nn * b2[1]])
        bsq = beta[0] * beta[0] + beta[1] * beta[1]
        if bsq * area < 1e-14:
            bhat = np.array([1.0, 0.0])
        else:
            nb = math.sqrt(bsq)
            bhat = beta / nb
        layer.beta[mode] = beta
        g = mysqrt(complex(bsq - ksq.real, -ksq.imag))
        layer.gamma[mode] = g
        if p == TE:
            Y = g / (1j * (k0 * ETA0) * layer.mur)
            tvec = zhatcross(bhat)
        else:
            Y = 1j * (k0 / ETA0) * layer.epsr / g
            tvec = bhat
        layer.Y[mode] = Y
        layer.tvec[mode] = tvec
        layer.c[mode] = mysqrt(1 / (area * Y))


def equal_layer_periodicity(l1, l2):
    n = np.linalg.norm
    denom = n(l1.beta1) + n(l1.beta2) + n(l2.beta1) + n(l2.beta2)
    return n(l1.beta1 - l2.beta1) / denom < 1e-5 and n(l1.beta2 - l2.beta2) / denom < 1e-5


def copy_betas_pmn(l1, l2):
    l1.beta1 = l2.beta1.copy()
    l1.beta2 = l2.beta2.copy()
    l1.P, l1.M, l1.N = list(l2.P), list(l2.M), list(l2.N)


def fill_mmax_pmn(layer, mnmax, k0max, dbmin):
    if mnmax < 0:
        raise ValueError("MNmax must be nonnegative")
    M, N, P = [], [], []
    for ring in range(mnmax + 1):
        for (m, n) in Ring(ring):
            M += [m, m]
            N += [n, n]
            P += [TE, TM]
    layer.M, layer.N, layer.P = M, N, P
    select_pmn(layer, k0max, dbmin)


def select_pmn(layer, k0max, dbmin=-math.inf):
    b1, b2 = layer.beta1, layer.beta2
    kmaxsq = k0max ** 2 * (layer.epsr * layer.mur)
    keep = []
    for mode in range(len(layer.P)):
        m, n = layer.M[mode], layer.N[mode]
        if math.isfinite(dbmin):
            if m == 0 and n == 0:
                keep.append(True)
                continue
            test = dbmin / 8.6859
            bv = m * b1 + n * b2
            beta = math.sqrt(bv[0] ** 2 + bv[1] ** 2)
            bmin = 0.0 if beta <= k0max else beta - k0max
            g = mysqrt(bmin ** 2 - kmaxsq)
            keep.append(g.real * layer.width < test)
        else:
            bv = m * b1 + n * b2
            g = mysqrt(bv[0] * bv[0] + bv[1] * bv[1] - kmaxsq)
            keep.append(g.imag >= g.real)
    M = [x for x, k in zip(layer.M, keep) if k]
    N = [x for x, k in zip(layer.N, keep) if k]
    uniq = []
    for mn in zip(M, N):
        if mn not in uniq:
            uniq.append(mn)
    layer.M = [mn[0] for mn in uniq for _ in range(2)]
    layer.N = [mn[1] for mn in uniq for _ in range(2)]
    layer.P = [TE, TM] * len(uniq)


def choose_layer_modes(layers, sheets, junc, gbl, k0max, dbmin=DBMIN):
    """Assign mode index lists ``P``, ``M``, ``N`` to every layer outside a Gblock
    (Modes.jl:49-275).  ``junc`` holds 1-based sheet numbers (0 = none)."""
    nl = len(layers)
    ngbl = len(gbl)
    for i in range(1, nl):
        for j in range(i):
            if layers[i] is layers[j]:
                layers[i] = layers[j].copy()
                break
    mset = [False] * (nl + 1)  # 1-based
    for g in gbl:
        for k in list(g.rng)[1:]:
            mset[k] = True
    pure_radome = not any(isht != 0 and sheets[isht - 1].style != "NULL" for isht in junc)
    if pure_radome:
        for l in layers:
            l.P, l.M, l.N = [TE, TM], [0, 0], [0, 0]
            l.beta1 = np.array([TWOPI, 0.0])
            l.beta2 = np.array([0.0, TWOPI])
        notinablock = list(range(1, nl + 1))
    else:
        good = [ig for ig, g in enumerate(gbl) if g.j != 0 and sheets[junc[g.j - 1] - 1].style != "NULL"]
        last_sheet = junc[gbl[good[-1]].j - 1]
        first_sheet = junc[gbl[good[0]].j - 1]
        upa = find_unique_periods(junc, sheets)
        for igbl in range(ngbl):
            g = gbl[igbl]
            ijunc = g.j
            if ijunc == 0:
                continue
            isht = junc[ijunc - 1]
            sheet = sheets[isht - 1]
            if sheet.style == "NULL":
                continue
            upm = sheet.units.units_per_meter
            b1 = sheet.beta1 * upm
            b2 = sheet.beta2 * upm
            i1 = g.first
            i2 = 1 + g.last
            for i in (i1, i2):
                if i == 1 or i == nl:
                    continue
                igo = max(igbl - 1, 0) if i == i1 else min(igbl + 1, ngbl - 1)
                ijo = gbl[igo].j
                ishto = junc[ijo - 1] if ijo != 0 else 0
                if not mset[i]:
                    layers[i - 1].beta1 = b1.copy()
                    layers[i - 1].beta2 = b2.copy()
                    mnmax = MNMAX_DEFAULT
                    if ijo != 0 and upa[ijunc - 1] != upa[ijo - 1] and sheets[ishto - 1].style != "NULL":
                        mnmax = 0
                    fill_mmax_pmn(layers[i - 1], mnmax, k0max, dbmin)
                    mset[i] = True
                else:
                    if (ijo != 0 and upa[ijunc - 1] != upa[ijo - 1] and len(layers[i - 1].P) != 2
                            and sheets[ishto - 1].style != "NULL"):
                        raise ValueError(f"Unequal unit cells in sheets {isht} and {ishto}.")
        while not all(mset[2:nl]):
            for i in range(2, nl):
                if mset[i]:
                    continue
                if mset[i - 1] and mset[i + 1]:
                    L, Lm, Lp = layers[i - 1], layers[i - 2], layers[i]
                    if equal_layer_periodicity(Lm, Lp):
                        L.beta1, L.beta2 = Lp.beta1.copy(), Lp.beta2.copy()
                        L.P = Lm.P + Lp.P
                        L.M = Lm.M + Lp.M
                        L.N = Lm.N + Lp.N
                        select_pmn(L, k0max, dbmin)
                    else:
                        L.beta1, L.beta2 = Lp.beta1.copy(), Lp.beta2.copy()
                        L.P, L.M, L.N = [TE, TM], [0, 0], [0, 0]
                    mset[i] = True
                elif mset[i - 1] and not mset[i + 1]:
                    if i - 1 == 1:
                        break
                    copy_betas_pmn(layers[i - 1], layers[i - 2])
                    select_pmn(layers[i - 1], k0max, dbmin)
                    mset[i] = True
                elif not mset[i - 1] and mset[i + 1]:
                    if i + 1 == nl:
                        break
                    copy_betas_pmn(layers[i - 1], layers[i])
                    select_pmn(layers[i - 1], k0max, dbmin)
                    mset[i] = True
        for l, sh in ((layers[0], sheets[first_sheet - 1]), (layers[nl - 1], sheets[last_sheet - 1])):
            upm = sh.units.units_per_meter
            l.beta1 = sh.beta1 * upm
            l.beta2 = sh.beta2 * upm
            fill_mmax_pmn(l, 0, k0max, dbmin)
        inblock = set()
        for g in gbl:
            inblock |= set(list(g.rng)[1:])
        notinablock = sorted(set(range(1, nl + 1)) - inblock)
        for k in range(len(notinablock) - 1):
            if notinablock[k + 1] - notinablock[k] != 1:
                continue
            il = notinablock[k]
            if equal_layer_periodicity(layers[il - 1], layers[il]):
                continue
            for l in layers[il - 1:il + 1]:
                l.P, l.M, l.N = [TE, TM], [0, 0], [0, 0]
    for i in notinablock:
        n = len(layers[i - 1].P)
        L = layers[i - 1]
        L.beta = np.zeros((n, 2))
        L.gamma = np.zeros(n, complex)
        L.Y = np.zeros(n, complex)
        L.c = np.zeros(n, complex)
        L.tvec = np.zeros((n, 2))

"""TEST INFRASTRUCTURE ONLY -- independent restatement of the selection steps that come before
the numerics of PSSFSS.jl v0.1.4's ``_analyze``: which interfaces form each Gblock, which
Floquet modes every layer carries, and which Gblocks repeat an earlier one.

Nothing here imports the package under test.  The strata are read as plain data: a layer
gives ``name``, ``epsr``, ``mur`` (complex) and ``width`` (m); a sheet gives ``style``,
``s1``, ``s2``, ``beta1``, ``beta2`` (sheet units) and ``units.units_per_meter``.  Indices
are 1-based, as in the reference (entry 0 of every per-layer or per-junction list is unused).

* ``junctions``          the layer/sheet walk of _analyze         (src/PSSFSS.jl:199-214)
* ``ring``               Ring iteration order                     (src/Rings.jl:9-60)
* ``unique_periods``     find_unique_periods                      (src/Sheets.jl:139-169)
* ``gblocks``            choose_gblocks                           (src/GSMs.jl:771-868)
* ``keep_modes``         select_pmn!                              (src/Modes.jl:399-431)
* ``lattice_modes``      fill_mmax_pmn!                           (src/Modes.jl:367-382)
* ``layer_modes``        choose_layer_modes!                      (src/Modes.jl:49-275)
* ``duplicate_gblocks``  get_gbldup                               (src/PSSFSS.jl:675-704)
* ``select``             all of the above for one strata list and frequency band
"""
import cmath
import math

import numpy as np

TE, TM = 1, 2
C0 = 299792458.0            # Constants.jl:9
DBMIN = 30.0                # Constants.jl:22
MIN_ELENGTH = 0.2 * math.pi  # Constants.jl:25: twopi * 0.1
MNMAX = 6                   # Modes.jl:14


def _mysqrt(z):
    r = cmath.sqrt(complex(z))
    return -r if (r.real == 0.0 and r.imag < 0.0) else r


def _null(sheet):
    return sheet.style == "NULL"


def junctions(strata, is_layer):
    """Split the strata list into layers and sheets; ``junc[k]`` (k = 1..nl-1) is the 1-based
    number of the sheet at the junction after layer k, 0 where there is none
    (src/PSSFSS.jl:122-125: the k-th sheet sits at the interface after the layers before it)."""
    layers, sheets = [], []
    for item in strata:
        (layers if is_layer(item) else sheets).append(item)
    junc = [0] * len(layers)  # junc[0] unused
    nlay = nsh = 0
    for item in strata:
        if is_layer(item):
            nlay += 1
        else:
            nsh += 1
            junc[nlay] = nsh
    return layers, sheets, junc


def ring(r):
    """The (m, n) lattice points at Chebyshev distance r, in Rings.jl's order: the row m = r
    (n ascending), the row m = -r, then the columns n = -r and n = r (m from 1-r to r-1)."""
    if r == 0:
        return [(0, 0)]
    pts = [(r, n) for n in range(-r, r + 1)] + [(-r, n) for n in range(-r, r + 1)]
    pts += [(m, -r) for m in range(1 - r, r)] + [(m, r) for m in range(1 - r, r)]
    return pts


def unique_periods(junc, sheets):
    """Equivalence class (1, 2, ...) of each junction's unit cell, 0 for a junction without a
    non-null sheet.  Cells compare by s1, s2 in metres at 8 significant digits."""
    def cell(sh):
        upm = sh.units.units_per_meter
        return tuple(float(f"{float(v) / upm:.7e}") for v in (*sh.s1, *sh.s2))

    reps, upa = [], [0] * len(junc)
    for i in range(1, len(junc)):
        if junc[i] == 0 or _null(sheets[junc[i] - 1]):
            continue
        c = cell(sheets[junc[i] - 1])
        if c not in reps:
            reps.append(c)
        upa[i] = reps.index(c) + 1
    return upa


def gblocks(layers, sheets, junc, k0min):
    """Partition of the junctions 1..nl-1 into Gblocks, as (first, last, j) with j the sheet's
    junction (0 for none): thin layers (electrical length at k0min at most 2pi/10) next to a
    sheet go into that sheet's block; two sheets without a thick layer between them are split
    at the electrically thickest intervening layer (the one nearest the middle on a tie)."""
    nl = len(layers)
    nj = nl - 1
    if not sheets or all(_null(s) for s in sheets):
        return [(i, i, i if junc[i] else 0) for i in range(1, nj + 1)]
    el = [0.0] + [k0min * l.width * math.sqrt((l.epsr * l.mur).real) for l in layers]  # el[1..nl]
    sint = [j for j in range(1, nj + 1) if junc[j] != 0]
    owner = list(range(nj + 1))  # owner[j] = junction whose block holds junction j
    ns = len(sheets)
    if not _null(sheets[0]):
        for lay in range(sint[0], 1, -1):
            if el[lay] > MIN_ELENGTH:
                break
            owner[lay - 1] = sint[0]
    if not _null(sheets[-1]):
        for lay in range(sint[ns - 1] + 1, nj + 1):
            if el[lay] > MIN_ELENGTH:
                break
            owner[lay] = sint[-1]
    for a, b in zip(sint[:-1], sint[1:]):
        na, nb = _null(sheets[junc[a] - 1]), _null(sheets[junc[b] - 1])
        between = range(a + 1, b + 1)  # layers between junctions a and b
        if any(el[lay] > MIN_ELENGTH for lay in between):
            for lay in range(b, a, -1):
                if el[lay] > MIN_ELENGTH or nb:
                    break
                owner[lay - 1] = b
            for lay in range(a + 1, b + 1):
                if el[lay] > MIN_ELENGTH or na:
                    break
                owner[lay] = a
            continue
        if na and not nb:
            for j in range(a + 1, b + 1):
                owner[j] = b
            continue
        if nb and not na:
            for j in range(a, b):
                owner[j] = a
            continue
        if na and nb:
            continue
        top = max(el[lay] for lay in between)
        ties = [lay for lay in between if el[lay] == top]
        mid = (a + b + 1) // 2
        best = min(ties, key=lambda lay: abs(lay - mid))  # first of equal distances
        for j in range(a, best):
            owner[j] = a
        for j in range(best, b + 1):
            owner[j] = b
    out = []
    for j in range(1, nj + 1):
        if out and owner[j] == owner[out[-1][0]]:
            out[-1][1] = j
        else:
            out.append([j, j, 0])
        if junc[j] != 0:
            out[-1][2] = j
    return [tuple(g) for g in out]


def keep_modes(modes, b1, b2, epsr, mur, width, k0max, dbmin=DBMIN):
    """Accessible modes among the candidates ``modes`` [(p, m, n)]: the (0, 0) pair always, any
    other (m, n) whose least possible attenuation through the layer at k0max (any incidence)
    stays below dbmin (dbmin = -inf: propagating modes only); each surviving (m, n) once, in
    first-appearance order, as a TE, TM pair."""
    ksq = k0max * k0max * (complex(epsr) * complex(mur))
    kept = []
    for p, m, n in modes:
        bx, by = m * b1[0] + n * b2[0], m * b1[1] + n * b2[1]
        if math.isfinite(dbmin):
            if m == 0 and n == 0:
                ok = True
            else:
                beta = math.hypot(bx, by)
                bmin = 0.0 if beta <= k0max else beta - k0max
                ok = _mysqrt(bmin * bmin - ksq).real * width < dbmin / 8.6859
        else:
            g = _mysqrt(bx * bx + by * by - ksq)
            ok = g.imag >= g.real
        if ok:
            kept.append((m, n))
    pairs = list(dict.fromkeys(kept))
    return [(pol, m, n) for m, n in pairs for pol in (TE, TM)]


def lattice_modes(mnmax, b1, b2, epsr, mur, width, k0max, dbmin=DBMIN):
    """Candidates of rings 0..mnmax (TE then TM at each lattice point), then ``keep_modes``."""
    cand = [(pol, m, n) for r in range(mnmax + 1) for m, n in ring(r) for pol in (TE, TM)]
    return keep_modes(cand, b1, b2, epsr, mur, width, k0max, dbmin)


def _same_cell(a, b):
    """equal_layer_periodicity (Modes.jl:335-338)."""
    den = (np.linalg.norm(a["b1"]) + np.linalg.norm(a["b2"]) + np.linalg.norm(b["b1"])
           + np.linalg.norm(b["b2"]))
    return (np.linalg.norm(np.subtract(a["b1"], b["b1"])) / den < 1e-5
            and np.linalg.norm(np.subtract(a["b2"], b["b2"])) / den < 1e-5)


def layer_modes(layers, sheets, junc, gbls, k0max, dbmin=DBMIN):
    """Mode list and reciprocal lattice of every layer: a list (index 1..nl) of dicts with
    ``modes`` [(p, m, n)], ``b1``, ``b2`` (rad/m), None for layers inside a Gblock."""
    nl = len(layers)
    st = [None] + [{"modes": [], "b1": np.zeros(2), "b2": np.zeros(2)} for _ in layers]
    inside = set()
    for first, last, _ in gbls:
        inside.update(range(first + 1, last + 1))
    done = [False] * (nl + 1)
    for lay in inside:
        done[lay] = True

    def active(g):
        return g[2] != 0 and not _null(sheets[junc[g[2]] - 1])

    def fill(lay, mnmax, b1, b2):
        L = layers[lay - 1]
        st[lay] = {"modes": lattice_modes(mnmax, b1, b2, L.epsr, L.mur, L.width, k0max, dbmin),
                   "b1": np.array(b1, float), "b2": np.array(b2, float)}

    def reselect(lay, modes, b1, b2):
        L = layers[lay - 1]
        st[lay] = {"modes": keep_modes(modes, b1, b2, L.epsr, L.mur, L.width, k0max, dbmin),
                   "b1": np.array(b1, float), "b2": np.array(b2, float)}

    two = [(TE, 0, 0), (TM, 0, 0)]
    if not any(junc[j] != 0 and not _null(sheets[junc[j] - 1]) for j in range(1, nl)):
        for lay in range(1, nl + 1):  # pure radome: dominant modes on a 1 m square cell
            st[lay] = {"modes": list(two), "b1": np.array([2 * math.pi, 0.0]), "b2": np.array([0.0, 2 * math.pi])}
        return st
    act = [k for k, g in enumerate(gbls) if active(g)]
    first_sheet = sheets[junc[gbls[act[0]][2]] - 1]
    last_sheet = sheets[junc[gbls[act[-1]][2]] - 1]
    upa = unique_periods(junc, sheets)
    ng = len(gbls)
    for k, g in enumerate(gbls):
        if not active(g):
            continue
        jk = g[2]
        sh = sheets[junc[jk] - 1]
        upm = sh.units.units_per_meter
        b1, b2 = np.asarray(sh.beta1, float) * upm, np.asarray(sh.beta2, float) * upm
        for lay, other in ((g[0], max(k - 1, 0)), (g[1] + 1, min(k + 1, ng - 1))):
            if lay == 1 or lay == nl:
                continue
            jo = gbls[other][2]
            clash = jo != 0 and upa[jk] != upa[jo] and not _null(sheets[junc[jo] - 1])
            if not done[lay]:
                fill(lay, 0 if clash else MNMAX, b1, b2)
                done[lay] = True
            elif clash and len(st[lay]["modes"]) != 2:
                raise ValueError(f"unequal unit cells in sheets {junc[jk]} and {junc[jo]}")
    while not all(done[2:nl]):
        before = sum(done)
        for lay in range(2, nl):
            if done[lay]:
                continue
            left, right = done[lay - 1], done[lay + 1]
            if left and right:
                if _same_cell(st[lay - 1], st[lay + 1]):
                    reselect(lay, st[lay - 1]["modes"] + st[lay + 1]["modes"], st[lay + 1]["b1"], st[lay + 1]["b2"])
                else:
                    st[lay] = {"modes": list(two), "b1": st[lay + 1]["b1"].copy(), "b2": st[lay + 1]["b2"].copy()}
                done[lay] = True
            elif left:
                if lay - 1 == 1:
                    break  # an end layer's modes are not chosen yet: go round again
                reselect(lay, st[lay - 1]["modes"], st[lay - 1]["b1"], st[lay - 1]["b2"])
                done[lay] = True
            elif right:
                if lay + 1 == nl:
                    break
                reselect(lay, st[lay + 1]["modes"], st[lay + 1]["b1"], st[lay + 1]["b2"])
                done[lay] = True
        if sum(done) == before:
            raise RuntimeError("interior layers whose modes no neighbour decides")
    for lay, sh in ((1, first_sheet), (nl, last_sheet)):
        upm = sh.units.units_per_meter
        fill(lay, 0, np.asarray(sh.beta1, float) * upm, np.asarray(sh.beta2, float) * upm)
    outside = [lay for lay in range(1, nl + 1) if lay not in inside]
    for a, b in zip(outside[:-1], outside[1:]):
        if b - a == 1 and not _same_cell(st[a], st[b]):
            st[a]["modes"] = list(two)
            st[b]["modes"] = list(two)
    for lay in inside:
        st[lay] = None
    return st


def duplicate_gblocks(gbls, layers, sheets, junc, modes):
    """gbldup: -1 for a Gblock whose GSM a later identical one reuses, g1 (1-based) for a
    Gblock that takes block g1's GSM, 0 otherwise.  Identical: the same sheet object, the
    same position of the sheet in the block, the same end-layer mode counts and equal
    interior layers (name, constants, width)."""
    def nm(lay):
        return len(modes[lay]["modes"]) if modes[lay] is not None else 0

    def same_layer(x, y):
        return (x.name == y.name and complex(x.epsr) == complex(y.epsr) and complex(x.mur) == complex(y.mur)
                and float(x.width) == float(y.width))

    dup = [0] * len(gbls)
    for a, (f1, l1, j1) in enumerate(gbls):
        if dup[a] != 0 or j1 == 0:
            continue
        n1, n2 = nm(f1), nm(l1 + 1)
        for b in range(a + 1, len(gbls)):
            f2, l2, j2 = gbls[b]
            if dup[b] != 0 or j2 == 0:
                continue
            if sheets[junc[j1] - 1] is not sheets[junc[j2] - 1]:
                continue
            if l1 - j1 != l2 - j2 or l1 - f1 != l2 - f2:
                continue
            if n1 != nm(f2) or n2 != nm(l2 + 1):
                continue
            if not all(same_layer(layers[x - 1], layers[y - 1])
                       for x, y in zip(range(f1 + 1, l1 + 1), range(f2 + 1, l2 + 1))):
                continue
            dup[a] = -1
            dup[b] = a + 1
    return dup


def select(strata, flist, is_layer):
    """Everything chosen before the numerics, for ``strata`` swept over ``flist`` (GHz):
    (junc, gbls [(first, last, j)], modes per layer (index 1..nl; None inside a Gblock),
    gbldup)."""
    layers, sheets, junc = junctions(strata, is_layer)
    f = [float(x) for x in np.atleast_1d(np.asarray(flist, float))]
    k0min = 2 * math.pi * 1e9 / C0 * min(f)
    k0max = 2 * math.pi * 1e9 / C0 * max(f)
    gbls = gblocks(layers, sheets, junc, k0min)
    modes = layer_modes(layers, sheets, junc, gbls, k0max)
    dup = duplicate_gblocks(gbls, layers, sheets, junc, modes)
    return junc, gbls, modes, dup

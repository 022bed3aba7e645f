"""``analyze``: the public entry point (PSSFSS.jl ``src/PSSFSS.jl:114-334``).

The reference walks steering x frequency and, per Gblock holding a sheet, calls
``calculate_jtype_gsm`` / ``calculate_mtype_gsm`` (``PSSFSS.jl:362-587``): fill, LU,
basis-function transforms, one solve per incident mode and the modal projection.  Here
the loop is reordered without changing any result: every (steering, frequency) point
is independent, so all points of one sheet go to the CUDA library in one batched call
(``pss_partial_gsms``), and the host then cascades each point's GSMs exactly as the
reference does.

Host-side per point (cheap scalar work, reference order kept): ``setup_modes!``
(Modes.jl:298), ``gsm_electric_gblock`` / ``gsm_magnetic_gblock`` (GSMs.jl:213/401), the
source vectors and projection weights of ``PSSFSS.jl:431-457`` / ``:557-584``, and the
cascade (``PSSFSS.jl:256-305``).

``getsttuple`` (PSSFSS.jl:607-617) reads an undefined global for ψ steering in
reference v0.1.4; here ψ steering works as its docstring describes.
"""
import cmath
import math
from dataclasses import dataclass, field

import numpy as np

from .constants import C0, DBMIN, TWOPI, UFACTOR
from .gsms import (GSM, cascade, cascade_layer, choose_gblocks, gsm_electric_gblock,
                   gsm_magnetic_gblock, gsm_slab_interface, pecgsm, pmcgsm, translate_gsm)
from .layers import Layer
from .modes import choose_layer_modes, setup_modes, zhatcross
from .outputs import Result
from .rwg import setup_rwg
from .sheets import RWGSheet

RTOL_APPROX = math.sqrt(np.finfo(float).eps)
PHI_KEYS = ("phi", "ϕ", "Phi", "PHI", "Φ")
THETA_KEYS = ("theta", "θ", "Theta", "THETA", "Θ")
PSI1_KEYS = ("psi1", "Psi1", "PSI1", "ψ₁", "Ψ₁", "ψ1", "Ψ1")
PSI2_KEYS = ("psi2", "Psi2", "PSI2", "ψ₂", "Ψ₂", "ψ2", "Ψ2")


def getsttuple(stkeys, stout, stin):
    """Steering dict for one (outer, inner) pair (PSSFSS.jl:607-617, ψ branch fixed)."""
    if stkeys[0] in PHI_KEYS:
        return {"θ": stin, "ϕ": stout}
    if stkeys[1] in PHI_KEYS:
        return {"θ": stout, "ϕ": stin}
    if stkeys[0] in PSI1_KEYS:
        return {"ψ₁": stout, "ψ₂": stin}
    return {"ψ₁": stin, "ψ₂": stout}


def check_inputs(layers):
    """PSSFSS.jl:619-633."""
    a, b = layers[0], layers[-1]
    if not (a.epsr.imag == b.epsr.imag == a.mur.imag == b.mur.imag == 0):
        raise ValueError("First and last layers must be lossless")
    if not (a.epsr == b.epsr and a.mur == b.mur):
        raise ValueError("First and last layers must have identical electrical parameters")


def _sind(x):
    if x % 180 == 0:
        return 0.0
    return math.sin(math.radians(x))


def _sincosd(x):
    from .sheets import _sincosd as sc
    return sc(x)


@dataclass
class Point:
    steer: dict
    fghz: float
    k0: float
    beta00: np.ndarray
    layers: list            # per-point deep copy with modal constants filled


@dataclass
class Plan:
    layers: list
    sheets: list
    junc: list              # 1-based sheet number per interface, 0 = none
    gbls: list
    gbldup: list
    rwgdat: list
    uvec: list
    points: list = field(default_factory=list)


def get_gbldup(gbls, layers, sheets, junc):
    """PSSFSS.jl:675-704."""
    gd = [0] * len(gbls)
    for g1, b1 in enumerate(gbls):
        if gd[g1] != 0 or b1.j == 0:
            continue
        n1 = len(layers[b1.first - 1].P)
        n2 = len(layers[b1.last].P)
        for g2 in range(g1 + 1, len(gbls)):
            b2 = gbls[g2]
            if gd[g2] != 0 or b2.j == 0:
                continue
            if sheets[junc[b1.j - 1] - 1] is not sheets[junc[b2.j - 1] - 1]:
                continue
            if b1.last - b1.j != b2.last - b2.j:
                continue
            if len(b1.rng) != len(b2.rng):
                continue
            if n1 != len(layers[b2.first - 1].P) or n2 != len(layers[b2.last].P):
                continue
            same = all(i1 == b1.first or layers[i1 - 1].same_as(layers[i2 - 1])
                       for i1, i2 in zip(b1.rng, b2.rng))
            if not same:
                continue
            gd[g1] = -1
            gd[g2] = g1 + 1
    return gd


def _geometry_key(sh):
    return (sh.rho.tobytes(), np.asarray(sh.fv).tobytes(), np.asarray(sh.fe).tobytes(), bool(sh.fufp),
            bool(sh.xi_eta_check), tuple(np.asarray(sh.s1, float)), tuple(np.asarray(sh.s2, float)))


def make_plan(strata, flist, steering, plan_flist=None, rwg_cache=None):
    """Everything of ``_analyze`` (PSSFSS.jl:199-255) before the per-Gblock GSMs.

    ``plan_flist`` (default ``flist``): the frequencies whose extremes choose the Gblocks
    and layer modes (PSSFSS.jl:215-221) - the whole sweep when ``flist`` is one shard.
    ``rwg_cache``: a dict reused across calls so that sheets of identical geometry share one
    basis-function setup (gradients perturb layers as well as geometry)."""
    layers = [s.copy() for s in strata if isinstance(s, Layer)]
    sheets = [s for s in strata if isinstance(s, RWGSheet)]
    nl = len(layers)
    junc = [0] * (nl - 1)
    nlay = 0
    ns = 0
    for s in strata:
        if isinstance(s, Layer):
            nlay += 1
        elif isinstance(s, RWGSheet):
            ns += 1
            junc[nlay - 1] = ns
    freqs = [float(f) for f in np.atleast_1d(np.asarray(flist, float))]
    stkeys = tuple(steering.keys())
    stvalues = [[float(v) for v in np.atleast_1d(np.asarray(steering[k], float))] for k in stkeys]
    check_inputs(layers)
    pfreqs = freqs if plan_flist is None else [float(f) for f in np.atleast_1d(np.asarray(plan_flist, float))]
    k0min = TWOPI * 1e9 / C0 * min(pfreqs)
    k0max = TWOPI * 1e9 / C0 * max(pfreqs)
    gbls = choose_gblocks(layers, sheets, junc, k0min)
    choose_layer_modes(layers, sheets, junc, gbls, k0max, DBMIN)
    gbldup = get_gbldup(gbls, layers, sheets, junc)
    rwgdat = []
    for sh in sheets:
        if sh.style == "NULL":
            rwgdat.append(None)
        elif rwg_cache is None:
            rwgdat.append(setup_rwg(sh))
        else:
            key = _geometry_key(sh)
            if key not in rwg_cache:
                rwg_cache[key] = setup_rwg(sh)
            rwgdat.append(rwg_cache[key])
    uvec = []
    for sh in sheets:
        if sh.style == "NULL":
            uvec.append(0.0)
        else:
            uf = UFACTOR * sh.units.units_per_meter
            uvec.append(uf * max(np.linalg.norm(sh.beta1), np.linalg.norm(sh.beta2)))
    plan = Plan(layers, sheets, junc, gbls, gbldup, rwgdat, uvec)
    for stout in stvalues[0]:
        for stin in stvalues[1]:
            steer = getsttuple(stkeys, stout, stin)
            if "ψ₁" in steer:
                p1, p2 = math.radians(steer["ψ₁"]), math.radians(steer["ψ₂"])
                upm = sheets[0].units.units_per_meter
                b1, b2 = sheets[0].beta1 * upm, sheets[0].beta2 * upm
                b00 = (p1 * b1 + p2 * b2) / TWOPI
            else:
                st = _sind(steer["θ"])
                sp, cp = _sincosd(steer["ϕ"])
            for fghz in freqs:
                k0 = TWOPI * fghz * 1e9 / C0
                if "θ" in steer:
                    k1 = k0 * math.sqrt((layers[0].epsr * layers[0].mur).real)
                    b00 = np.array([k1 * st * cp, k1 * st * sp])
                pl = [l.copy() for l in layers]
                for l in pl:
                    setup_modes(l, k0, b00)
                a0 = np.angle(pl[0].gamma[0])
                a1 = np.angle(pl[-1].gamma[0])
                # Julia's a ≈ b ≈ c: default rtol = sqrt(eps(Float64))
                if not (math.isclose(a0, a1, rel_tol=RTOL_APPROX)
                        and math.isclose(a1, math.pi / 2, rel_tol=RTOL_APPROX)):
                    continue  # principal modes cut off in the ambient medium (PSSFSS.jl:252)
                plan.points.append(Point(steer, fghz, k0, np.array(b00, float), pl))
    return plan


@dataclass
class SheetIO:
    """Inputs of one sheet's partial GSM at one point, in the library's generic form.

    For mode j (region-1 modes first, then region-N modes): ``kvec[j]`` is the transform
    variable of its basis-function FT, ``src[j]`` the complex incident field vector so
    that ``rhs[n, j] = conj(bfft_j[n]) . src[j]``, and ``tobs[j]``/``wobs[j]`` give
    ``dS[i, j] = wobs[i] * sum_n x[n, j] (tobs[i] . bfft_i[n])``.
    """
    gsm: GSM
    n1: int
    n2: int
    kvec: np.ndarray
    src: np.ndarray
    tobs: np.ndarray
    wobs: np.ndarray
    psi1: float
    psi2: float


def sheet_io(region, sheet, s, k0, beta00):
    """Host part of ``calculate_jtype_gsm`` (PSSFSS.jl:362-460) / ``calculate_mtype_gsm``
    (PSSFSS.jl:486-587): incident GSM, source vectors and projection weights."""
    upm = sheet.units.units_per_meter
    area = abs(sheet.s1[0] * sheet.s2[1] - sheet.s1[1] * sheet.s2[0]) / upm ** 2
    ends = (region[0], region[-1])
    acf = []
    for l in ends:
        ai = TWOPI * TWOPI / abs(l.beta1[0] * l.beta2[1] - l.beta1[1] * l.beta2[0])
        acf.append(math.sqrt(ai / area))
    if sheet.cls == "J":
        gsm, tlgf, vinc = gsm_electric_gblock(region, s, k0)
    else:
        gsm, tlgf, vinc = gsm_magnetic_gblock(region, s, k0)
    psi1 = (beta00[0] * sheet.s1[0] + beta00[1] * sheet.s1[1]) / upm
    psi2 = (beta00[0] * sheet.s2[0] + beta00[1] * sheet.s2[1]) / upm
    n1, n2 = len(ends[0].P), len(ends[1].P)
    nm = n1 + n2
    kvec = np.zeros((nm, 2))
    src = np.zeros((nm, 2), complex)
    tobs = np.zeros((nm, 2))
    wobs = np.zeros(nm, complex)
    j = 0
    for r, l in enumerate(ends):
        sigma = 1.0 if r == 0 else -1.0
        for q in range(len(l.P)):
            kvec[j] = l.beta[q]
            if sheet.cls == "J":
                src[j] = vinc[q, r] * l.c[q] * acf[r] * l.tvec[q]
                tobs[j] = l.tvec[q]
                wobs[j] = -(tlgf[q, r] / (l.c[q] * acf[r] * area))
            else:
                src[j] = sigma * (vinc[q, r] * l.c[q] * l.Y[q] * zhatcross(l.tvec[q]))
                tobs[j] = zhatcross(l.tvec[q])
                wobs[j] = tlgf[q, r] * l.c[q]
            j += 1
    return SheetIO(gsm, n1, n2, kvec, src, tobs, wobs, psi1, psi2)


def add_scattered(io, dS):
    """Add the scattered part ``dS`` ((n1+n2)^2) to the incident partial GSM."""
    g = io.gsm
    n1 = io.n1
    g.s11 += dS[:n1, :n1]
    g.s12 += dS[:n1, n1:]
    g.s21 += dS[n1:, :n1]
    g.s22 += dS[n1:, n1:]
    return g


def sheet_gblocks(plan):
    """(Gblock index, region slice, sheet index, s) of every Gblock whose GSM comes from a
    non-null sheet and is not a copy of an earlier one."""
    out = []
    for ig, g in enumerate(plan.gbls):
        if g.j == 0:
            continue
        isht = plan.junc[g.j - 1]
        sheet = plan.sheets[isht - 1]
        if plan.gbldup[ig] > 0 or sheet.style == "NULL" or sheet.cls not in ("J", "M"):
            continue
        i1, i2 = g.first, g.last + 1
        out.append((ig, (i1, i2), isht, g.j - i1 + 1))
    return out


def _propagation(layer):
    """exp(-γ d) of every mode of ``layer`` (``cascade!``, GSMs.jl:154-176); ones when d = 0."""
    if layer.width == 0:
        return np.ones(len(layer.gamma), complex)
    return np.array([cmath.exp(-g * layer.width) for g in layer.gamma], complex)


def _gblock_chain(plan, partial, p, gsm_save):
    """The GSM of every Gblock at point ``p`` (sheet partial GSMs, PEC/PMC, or bare slab
    interfaces; translations applied), each with the propagation factors of the layer
    behind it (PSSFSS.jl:256-305)."""
    pt = plan.points[p]
    L = pt.layers
    chain = [_propagation(L[0])]
    for ig, g in enumerate(plan.gbls):
        i1, i2 = g.first, g.last + 1
        if g.j != 0:
            isht = plan.junc[g.j - 1]
            sheet = plan.sheets[isht - 1]
            if plan.gbldup[ig] > 0:
                gsmb = gsm_save[plan.gbldup[ig] - 1].copy()
            else:
                if sheet.cls in ("J", "M") and sheet.style != "NULL":
                    gsmb = partial[ig][p].copy()
                elif sheet.cls == "E":
                    gsmb = pecgsm(len(L[i1 - 1].P), len(L[i2 - 1].P))
                elif sheet.cls == "H":
                    gsmb = pmcgsm(len(L[i1 - 1].P), len(L[i2 - 1].P))
                else:
                    raise ValueError(f"Illegal sheet class: {sheet.cls}")
                if plan.gbldup[ig] < 0:
                    gsm_save[ig] = gsmb.copy()
            if sheet.dx != 0 or sheet.dy != 0:
                upm = sheet.units.units_per_meter
                translate_gsm(gsmb, sheet.dx / upm, sheet.dy / upm, L[i1 - 1], L[i2 - 1])
        else:
            gsmb = gsm_slab_interface(L[i1 - 1], L[i2 - 1], pt.k0)
        chain.append((gsmb, _propagation(L[i2 - 1])))
    return chain


def _result(pt, gsmc):
    L = pt.layers
    return Result(gsmc, pt.steer, pt.beta00, pt.fghz, L[0].epsr, L[0].mur, L[0].beta1.copy(), L[0].beta2.copy(),
                  L[-1].epsr, L[-1].mur, L[-1].beta1.copy(), L[-1].beta2.copy())


def assemble(plan, partial, where="auto", device=0):
    """Cascade each point's Gblock GSMs (PSSFSS.jl:256-312).  ``partial[ig][p]`` is the
    partial GSM of sheet Gblock ``ig`` at point ``p``.  ``where``: ``"device"`` runs the
    star products of every point in one ``pss_cascade`` call, ``"host"`` in numpy,
    ``"auto"`` (default) the device when a GPU is there and every region has at most 64
    modes."""
    if not plan.points:
        return []
    gsm_save = {}
    chains = [_gblock_chain(plan, partial, p, gsm_save) for p in range(len(plan.points))]
    use_device = where == "device"
    if where == "auto":
        from . import engine
        dims = [len(chains[0][0])] + [len(pv) for _, pv in chains[0][1:]]
        use_device = max(dims) <= engine.CASCADE_MAX_MODES and engine.device_available()
    if use_device:
        from . import engine
        out = engine.cascade_points(chains, device=device)
        return [_result(pt, GSM(*o)) for pt, o in zip(plan.points, out)]
    results = []
    for pt, chain in zip(plan.points, chains):
        n1 = len(pt.layers[0].P)
        gsma = cascade_layer(GSM.identity(n1, n1), pt.layers[0])
        gsmc = gsma
        for (gsmb, _), g in zip(chain[1:], plan.gbls):
            gsmc = cascade(gsma, gsmb)
            cascade_layer(gsmc, pt.layers[g.last])
            gsma = gsmc
        results.append(_result(pt, gsmc))
    return results


class AnalysisLog:
    """The ``logfile`` of ``analyze`` (``Log.jl``; messages of ``PSSFSS.jl:212-332`` and the
    layer / sheet report of ``:706-745``).  Without a file name every call is a no-op."""

    def __init__(self, logfile):
        self.fname = logfile
        if logfile:
            open(logfile, "w").close()

    def __call__(self, msg):
        if self.fname:
            with open(self.fname, "a", encoding="utf-8") as f:
                f.write(msg + "\n")

    def start(self):
        import datetime
        now = datetime.datetime.now()
        self(f"\n\nStarting pssfss_b200 analysis on {now:%Y-%m-%d} at {now:%H:%M:%S}\n\n")

    def report(self, plan):
        """Layer and sheet tables of ``report_layers_sheets`` (PSSFSS.jl:706-745)."""
        if not self.fname:
            return
        from .gsms import find_unique_periods
        usi = find_unique_periods(plan.junc, plan.sheets)
        usi = [usi[plan.junc.index(k + 1)] if (k + 1) in plan.junc else 0 for k in range(len(plan.sheets))]
        self("Dielectric layer information... \n")
        self(" Layer  Width  units  epsr   tandel   mur  mtandel modes  beta1x  beta1y  beta2x  beta2y")
        self(" ----- ------------- ------- ------ ------- ------ ----- ------- ------- ------- -------")
        for jl, l in enumerate(plan.layers, 1):
            eps, mu = l.epsr.real, l.mur.real
            uw = l.user_width
            units = "in" if uw.unit.name == "inch" else uw.unit.name
            self(" %5i %9.4f %3s %7.2f %6.4f %7.2f %6.4f %5i %7.1f %7.1f %7.1f %7.1f" % (
                jl, float(uw.value), units, eps, -l.epsr.imag / eps, mu, -l.mur.imag / mu, len(l.P),
                l.beta1[0], l.beta1[1], l.beta2[0], l.beta2[1]))
            if jl < len(plan.layers) and plan.junc[jl - 1] != 0:
                js = plan.junc[jl - 1]
                sh = plan.sheets[js - 1]
                om = sh.units.units_per_meter
                self(" ==================  Sheet %3i  ======================== %7.1f %7.1f %7.1f %7.1f" % (
                    usi[js - 1], sh.beta1[0] * om, sh.beta1[1] * om, sh.beta2[0] * om, sh.beta2[1] * om))
        sint = [i + 1 for i, j in enumerate(plan.junc) if j != 0]
        self("\n\n\nPSS/FSS sheet information...\n")
        self("Sheet  Loc         Style      Rot  J/M Faces Edges Nodes Unknowns  NUFP")
        self("-----  ---  ---------------- ----- --- ----- ----- ----- -------- ------")
        for js, sh in enumerate(plan.sheets, 1):
            rw = plan.rwgdat[js - 1]
            self("%4i   %3i  %16s %5.1f  %1s  %5i %5i %5i  %6i %7i" % (
                usi[js - 1], sint[js - 1], sh.style, sh.rot, sh.cls, sh.nface, sh.nedge, sh.nnode,
                rw.nbf if rw is not None else 0, rw.nufp if rw is not None else 0))
        self("\n\n")

    def skipped(self, plan, flist):
        planned = {pt.fghz for pt in plan.points}
        for f in np.atleast_1d(np.asarray(flist, float)):
            if float(f) not in planned:
                self(f"  Skipping {float(f)} GHz due to cutoff principal modes in ambient medium")

    def sheet_sweep(self, isht, npts, timings):
        self(f"    Sheet {isht}: {npts} points on the GPU")
        for k, v in (timings or {}).items():
            self(f"      {v:.3f} ms {k}")

    def finish(self):
        import datetime
        now = datetime.datetime.now()
        self(f"\n\n pssfss_b200 analysis exiting on {now:%Y-%m-%d} at {now:%H:%M:%S}\n\n")


def analyze(strata, flist, steering, *, precision="fp64", device=0, outlist=(),
            logfile=None, resultfile=None, showprogress=False, stats=None, plan_flist=None):
    """Analyze a layered FSS/PSS over frequencies and steering (PSSFSS.jl:114).

    ``strata``: list of ``Layer`` and ``RWGSheet`` (first and last must be layers).
    ``flist``: frequencies in GHz.  ``steering``: dict with keys (θ, ϕ) or (ψ₁, ψ₂) in
    degrees (first key = outer loop).  ``precision``: ``"fp64"`` (plain FP64 LU) or
    ``"fp32r"`` (complex64 LU with FP64 iterative refinement).
    ``logfile``: a log of the layers, sheets and per-sheet device timings (none by default).
    ``outlist``: (csv file name, ``outputs(...)`` tuple) pairs, each written as a header of
    output labels and one row per result (PSSFSS.jl:316-325).  ``resultfile``: where to
    save the results for ``read_result_file`` / ``extract_result_file`` (none by default;
    the reference's JLD2 file is not written).
    Returns a list of ``Result``.
    """
    from . import engine
    from .outputs import write_outlist
    log = AnalysisLog(logfile)
    log.start()
    plan = make_plan(strata, flist, steering, plan_flist)
    log.report(plan)
    log.skipped(plan, flist)
    partial = {}
    for ig, (i1, i2), isht, s in sheet_gblocks(plan):
        sheet = plan.sheets[isht - 1]
        ios = [sheet_io(pt.layers[i1 - 1:i2], sheet, s, pt.k0, pt.beta00) for pt in plan.points]
        st = stats if stats is not None else ({} if logfile else None)
        dS = engine.partial_gsms(sheet, plan.rwgdat[isht - 1], plan.points, (i1, i2), s,
                                 plan.uvec[isht - 1], ios, precision=precision, device=device,
                                 stats=st)
        log.sheet_sweep(isht, len(plan.points), (st or {}).get("timings_ms"))
        partial[ig] = [add_scattered(io, d) for io, d in zip(ios, dS)]
    results = assemble(plan, partial)
    write_outlist(results, outlist, resultfile)
    log.finish()
    return results


def analyze_many(cases, *, precision="fp32r", device=0, tuning=None, stats=None):
    """Many independent analyses in one device call (``pss_partial_gsms_multi``).

    ``cases``: list of ``(strata, flist, steering)`` as ``analyze`` takes them.  Every sheet
    sweep of every case goes into one shared work list on the device - batches of like-N
    points, largest matrices first - instead of one library call per sheet and case.
    ``tuning``: a callable ``n -> dict(batch=, panel_w=, outer_nb=)`` choosing the batch size
    and the FP32 LU tile shape per unknown count (``autotune.lookup`` reads the stored
    table); ``None`` keeps the library defaults.  Returns one list of ``Result`` per case."""
    from . import engine
    plans, jobs, problems = [], [], []
    for strata, flist, steering in cases:
        plan = make_plan(strata, flist, steering)
        plans.append(plan)
        for ig, (i1, i2), isht, s in sheet_gblocks(plan):
            sheet, rwg = plan.sheets[isht - 1], plan.rwgdat[isht - 1]
            ios = [sheet_io(pt.layers[i1 - 1:i2], sheet, s, pt.k0, pt.beta00) for pt in plan.points]
            pr = dict(sheet=sheet, rwg=rwg, points=plan.points, region_rng=(i1, i2), s=s, u=plan.uvec[isht - 1],
                      ios=ios)
            if tuning is not None:
                pr.update(tuning(rwg.nbf))
            jobs.append((len(plans) - 1, ig, ios))
            problems.append(pr)
    out = engine.partial_gsms_multi(problems, precision=precision, device=device, stats=stats) if problems else []
    partial = [dict() for _ in plans]
    for (c, ig, ios), dS in zip(jobs, out):
        partial[c][ig] = [add_scattered(io, d) for io, d in zip(ios, dS)]
    return [assemble(plan, partial[c]) for c, plan in enumerate(plans)]

"""Analysis results and their extraction (PSSFSS.jl ``src/Outputs.jl``).

``Result`` carries the full GSM of the structure for one (steering, frequency) point
plus the end-region media and lattices, exactly the fields of the reference's struct.
Outputs are requested as in the reference's ``@outputs`` (``Outputs.jl:366``): ``outputs(
"FGHz", "theta", "s21db(te,te)", "ar21db(h)")`` returns functors that ``extract_result``
applies to results.  Polarisation indices are ``TE``/``TM`` (the modal basis), ``H``/``V``
(Ludwig-3 linear) or ``R``/``L`` (circular), converted by the 2 x 2 basis changes of
``Outputs.jl:99-197``.
"""
import cmath
import math
import re
from dataclasses import dataclass
from enum import IntEnum

import numpy as np

from .constants import C0, TWOPI
from .gsms import GSM
from .layers import TE, TM


@dataclass
class Result:
    gsm: GSM
    steering: dict          # {"θ": deg, "ϕ": deg} or {"ψ₁": deg, "ψ₂": deg}
    beta00: np.ndarray      # radians/meter
    FGHz: float
    epsr_in: complex
    mur_in: complex
    beta1_in: np.ndarray
    beta2_in: np.ndarray
    epsr_out: complex
    mur_out: complex
    beta1_out: np.ndarray
    beta2_out: np.ndarray

    def __repr__(self):
        return f"Result: {self.FGHz} GHz, {self.steering}, GSM{self.gsm.s12.shape}"


class HorV(IntEnum):
    """Ludwig-3 horizontal / vertical polarisation (``Outputs.jl:15``)."""
    H = 1
    V = 2


class RorL(IntEnum):
    """Right / left circular polarisation (``Outputs.jl:16``)."""
    R = 1
    L = 2


H, V = HorV.H, HorV.V
R, L = RorL.R, RorL.L


def _sincosd(x):
    return math.sin(math.radians(x)), math.cos(math.radians(x))


def theta_phi(o):
    """Steering angles (degrees) of a result, from its β00 and the input medium
    (``θϕ``, ``Outputs.jl:319-337``)."""
    b00 = np.asarray(o.beta00, float)
    b2 = float(b00 @ b00)
    if b2 == 0:
        return 0.0, float(o.steering.get("ϕ", 0.0))
    k2 = (TWOPI * o.FGHz * 1e9 / C0) ** 2 * (o.epsr_in * o.mur_in).real
    if b2 > k2:
        raise ValueError("Cut-off dominant mode")
    kz = math.sqrt(k2 - b2)
    return math.degrees(math.acos(kz / math.sqrt(k2))), math.degrees(math.atan2(b00[1], b00[0]))


def hv_hat(theta, phi):
    """Ludwig-3 unit vectors ĥ, v̂ at (θ, ϕ) in degrees (``Outputs.jl:344-354``)."""
    st, ct = _sincosd(theta)
    sp, cp = _sincosd(phi)
    th = np.array([ct * cp, ct * sp, -st])
    ph = np.array([-sp, cp, 0.0])
    return th * cp - ph * sp, th * sp + ph * cp


def _region_angles(j, o, incident):
    th1, ph1 = theta_phi(o)
    if j == 1:
        return th1, (ph1 if incident else ph1 + 180), 1
    n1 = math.sqrt(o.epsr_in.real * o.mur_in.real)
    n2 = math.sqrt(o.epsr_out.real * o.mur_out.real)
    th = math.degrees(math.asin(n1 / n2 * math.sin(math.radians(th1))))  # Snell's law
    return th, (ph1 + 180 if incident else ph1), -1


def _tangents(o):
    b00 = np.asarray(o.beta00, float)
    nb = float(np.linalg.norm(b00))
    bh = np.array([1.0, 0.0]) if nb == 0 else b00 / nb
    return np.array([-bh[1], bh[0]]), bh  # t̂1 = ẑ × β̂00, t̂2 = β̂00


def sourcemat(j, n, o):
    """2 x 2 change from the TE/TM basis to H/V or R/L for the incident wave of region j
    (right factor of ``o.gsm[i, j]``; ``Outputs.jl:99-144``).  Kept term for term as the
    reference writes it, including its 1/cos θ on the TM row, so oblique-incidence H/V and
    R/L outputs are the reference's numbers."""
    th, ph, sgn = _region_angles(j, o, incident=True)
    h, v = hv_hat(th, ph)
    t1, t2 = _tangents(o)
    ct = math.cos(math.radians(th))
    if isinstance(n, HorV):
        return np.array([[h[:2] @ t1, v[:2] @ t1], [h[:2] @ t2 / ct, v[:2] @ t2 / ct]], complex)
    lv = (h + sgn * 1j * v) / math.sqrt(2)
    rv = (h - sgn * 1j * v) / math.sqrt(2)
    return np.array([[t1 @ rv[:2], t1 @ lv[:2]], [t2 @ rv[:2] / ct, t2 @ lv[:2] / ct]])


def obsmat(i, m, o):
    """2 x 2 change to H/V or R/L for the wave leaving region i (left factor of
    ``o.gsm[i, j]``; ``Outputs.jl:154-197``)."""
    th, ph, sgn = _region_angles(i, o, incident=False)
    h, v = hv_hat(th, ph)
    t1, t2 = _tangents(o)
    t13 = np.array([t1[0], t1[1], 0.0])
    t23 = np.array([t2[0], t2[1], sgn * math.tan(math.radians(th))])
    if isinstance(m, HorV):
        return np.array([[h @ t13, h @ t23], [v @ t13, v @ t23]], complex)
    lv = (h - sgn * 1j * v) / math.sqrt(2)
    rv = (h + sgn * 1j * v) / math.sqrt(2)
    rc, lc = np.conj(rv), np.conj(lv)  # the observed component: conjugated projection
    return np.array([[rc @ t13, rc @ t23], [lc @ t13, lc @ t23]])


def _changed(x):
    return isinstance(x, (HorV, RorL))


def getsijmn(i, j, m, n, r):
    """Entry (m, n) of partition (i, j) of ``r.gsm`` (``Outputs.jl:73-89``): m, n are 1-based
    mode indices or TE/TM, or H/V, R/L for the polarisation basis changes."""
    g = r.gsm[(i, j)]
    if not _changed(m) and not _changed(n):
        return g[int(m) - 1, int(n) - 1]
    g2 = np.asarray(g[:2, :2])
    if _changed(n):
        g2 = g2 @ sourcemat(j, n, r)
    if _changed(m):
        g2 = obsmat(i, m, r) @ g2
    return g2[int(m) - 1, int(n) - 1]


def s_parameters(results, i, j, m, n):
    """Vector of ``S{i}{j}(m,n)`` over a list of results."""
    return np.array([getsijmn(i, j, m, n, r) for r in results])


class Outfun:
    """A labelled output request applied to a ``Result`` (``Outputs.jl:40-45``)."""

    def __init__(self, f, label):
        self.f, self.label = f, label

    def __call__(self, r):
        return self.f(r)

    def __repr__(self):
        return f"Outfun: {self.label}"


def _db(x2):
    return 10 * math.log10(x2) if x2 > 0 else -math.inf


def _sij(i, j, kind):
    conv = {"": lambda z: z, "MAG": abs, "DB": lambda z: _db(abs(z) ** 2),
            "ANG": lambda z: math.degrees(cmath.phase(z)), "REAL": lambda z: z.real,
            "IMAG": lambda z: z.imag}[kind]

    def make(m, n):
        return Outfun(lambda o: conv(complex(getsijmn(i, j, m, n, o))), f"S{i}{j}{kind}({_name(m)},{_name(n)})")
    return make


def _name(x):
    if isinstance(x, (HorV, RorL)):
        return x.name
    return {TE: "TE", TM: "TM"}.get(int(x), str(int(x)))


def _ardb(i, j):
    def make(n):
        def f(o):
            jp = 1j * getsijmn(i, j, 1, n, o) / getsijmn(i, j, 2, n, o)  # modified linear pol. ratio
            q = abs((1 - jp) / (1 + jp))                                  # circular pol. ratio
            q = 1 / q if q > 1 else q
            return math.inf if q >= 1 else 20 * math.log10((1 + q) / (1 - q))
        return Outfun(f, f"AR{i}{j}({_name(n)})dB")
    return make


def _ratio(i, j, kind):
    def f(o):
        z = getsijmn(i, j, 1, 1, o) / getsijmn(i, j, 2, 2, o)
        return math.degrees(cmath.phase(z)) if kind == "IPD" else _db(abs(z) ** 2)
    return Outfun(f, "ΔIPD" if kind == "IPD" else "ΔIL")


OUTPUTS = {}
for _i in (1, 2):
    for _j in (1, 2):
        for _k in ("", "MAG", "DB", "ANG", "REAL", "IMAG"):
            OUTPUTS[f"S{_i}{_j}{_k}"] = _sij(_i, _j, _k)
        OUTPUTS[f"AR{_i}{_j}DB"] = _ardb(_i, _j)
OUTPUTS.update({
    "ΔIPD21": _ratio(2, 1, "IPD"), "DIPD21": _ratio(2, 1, "IPD"),
    "ΔIPD12": _ratio(1, 2, "IPD"), "DIPD12": _ratio(1, 2, "IPD"),
    "ΔIL21": _ratio(2, 1, "IL"), "DIL21": _ratio(2, 1, "IL"),
    "ΔIL12": _ratio(1, 2, "IL"), "DIL12": _ratio(1, 2, "IL"),
    "FGHZ": Outfun(lambda o: o.FGHz, "FGHZ"),
    "FMHZ": Outfun(lambda o: o.FGHz * 1000, "FMHZ"),
    "THETA": Outfun(lambda o: o.steering.get("θ", math.nan), "THETA"),
    "PHI": Outfun(lambda o: o.steering.get("ϕ", math.nan), "PHI"),
    "PSI1": Outfun(lambda o: o.steering.get("ψ₁", math.nan), "PSI1"),
    "PSI2": Outfun(lambda o: o.steering.get("ψ₂", math.nan), "PSI2"),
})
OUTPUTS.update({"Θ": OUTPUTS["THETA"], "Φ": OUTPUTS["PHI"], "Ψ₁": OUTPUTS["PSI1"], "Ψ₂": OUTPUTS["PSI2"]})
_POL = {"TE": TE, "TM": TM, "H": H, "V": V, "R": R, "L": L}


def outputs(*specs):
    """Output functors from request strings, case-insensitive as ``@outputs``
    (``Outputs.jl:366-384``): e.g. ``outputs("FGHz", "theta", "s11db(te,te)",
    "S21ang(R,H)", "ar21db(h)", "dipd21")``."""
    out = []
    for spec in specs:
        m = re.fullmatch(r"\s*([^\s(]+)\s*(?:\((.*)\))?\s*", spec)
        if not m:
            raise ValueError(f"Illegal outputs construction: {spec!r}")
        name = m.group(1).upper()
        if name not in OUTPUTS:
            raise ValueError(f"unknown output {m.group(1)!r}")
        f = OUTPUTS[name]
        if m.group(2) is None:
            if not isinstance(f, Outfun):
                raise ValueError(f"{m.group(1)} needs arguments")
            out.append(f)
            continue
        args = []
        for a in m.group(2).split(","):
            a = a.strip().upper()
            args.append(_POL[a] if a in _POL else int(a))
        out.append(f(*args))
    return tuple(out)


def extract_result(results, ops):
    """Matrix of outputs: one row per result, one column per functor of ``ops``
    (``Outputs.jl:446-453``); a single ``Result`` gives one row."""
    if isinstance(results, Result):
        results = [results]
    return np.array([[o(r) for o in ops] for r in results])


def _cell(v):
    if isinstance(v, complex):
        return f"{v.real!r}{'+' if v.imag >= 0 else '-'}{abs(v.imag)!r}im"
    return repr(float(v))


def write_outputs_csv(fname, results, ops):
    """A CSV of the outputs ``ops`` of ``results``: a header of their labels, then one row
    per result (the reference's ``outlist`` files, ``PSSFSS.jl:316-325``)."""
    with open(fname, "w", encoding="utf-8") as f:
        f.write(",".join(o.label for o in ops) + "\n")
        for r in results:
            f.write(",".join(_cell(o(r)) for o in ops) + "\n")


def save_results(fname, results):
    """Save results for ``read_result_file`` (a pickle of the list; the reference's file is
    JLD2, ``Outputs.jl:396-409``)."""
    import pickle
    with open(fname, "wb") as f:
        pickle.dump(list(results), f)


def read_result_file(fname):
    """The results saved by ``save_results`` (``Outputs.jl:411-421``)."""
    import pickle
    with open(fname, "rb") as f:
        return pickle.load(f)


def extract_result_file(fname, ops):
    """``extract_result`` of the results in a result file (``Outputs.jl:428-431``)."""
    return extract_result(read_result_file(fname), ops)


def write_outlist(results, outlist=(), resultfile=None):
    """The file outputs of ``analyze``: every (csv name, ops) of ``outlist``, and the result
    file when one is named."""
    for fname, ops in outlist:
        write_outputs_csv(fname, results, ops)
    if resultfile:
        save_results(resultfile, results)

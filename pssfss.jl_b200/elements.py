"""Sheet constructors with structured meshes (PSSFSS.jl ``src/Elements.jl``).

``rectstrip`` (``:149-186``) and ``meander`` (``:617-729``) are built from ``recttri``
and ``combine`` exactly as in the reference, so node numbering, edge numbering and
coordinates are identical.  ``pecsheet``/``pmcsheet`` (``:108-126``) are the null
sheets.  Constructors that call Shewchuk's Triangle in the reference (``polyring``,
``diagstrip`` end caps, ``loadedcross``, ``jerusalemcross``) are not provided: their
meshes cannot be reproduced without that third-party mesher.
"""
import math

import numpy as np

from .sheets import RWGSheet, combine, recttri, rotate, s1s2_to_b1b2

_DEFAULTS = dict(cls="J", dx=0.0, dy=0.0, rot=0.0, Rsheet=0.0, save="", fufp=False)


def _check_kwargs(kwargs):
    """``check_optional_kw_arguments!`` (``Elements.jl:46-71``)."""
    if "class" in kwargs:
        kwargs["cls"] = kwargs.pop("class")
    bad = set(kwargs) - set(_DEFAULTS)
    if bad:
        raise ValueError("Illegal keywords: " + ", ".join(sorted(bad)))
    for k, v in _DEFAULTS.items():
        kwargs.setdefault(k, v)
    if kwargs["cls"] not in ("J", "M"):
        raise ValueError(f"Illegal value {kwargs['cls']} for class")
    for k in ("dx", "dy", "rot", "Rsheet"):
        if not isinstance(kwargs[k], (int, float)):
            raise ValueError(f"{k} must be a Real")
    if kwargs["Rsheet"] < 0:
        raise ValueError("Rsheet must be nonnegative")
    if not isinstance(kwargs["save"], str):
        raise ValueError("save must be an AbstractString")
    return kwargs


def _testpos(**kw):
    for k, v in kw.items():
        if not v > 0:
            raise ValueError(f"{k} must be positive!")


def pecsheet():
    """Perfect electric conducting sheet (``Elements.jl:108``)."""
    sh = RWGSheet()
    sh.style = "NULL"
    sh.cls = "E"
    return sh


def pmcsheet():
    """Perfect magnetic conducting sheet (``Elements.jl:121``)."""
    sh = RWGSheet()
    sh.style = "NULL"
    sh.cls = "H"
    return sh


def rectstrip(*, Lx, Ly, Nx, Ny, Px, Py, units, **kwarg):
    """Rectangular strip in a rectangular cell (``Elements.jl:149-186``)."""
    kwargs = dict(kwarg)
    kwargs.setdefault("fufp", True)
    _check_kwargs(kwargs)
    _testpos(Lx=Lx, Ly=Ly, Nx=Nx, Ny=Ny, Px=Px, Py=Py)
    x0 = 0.5 * (Px - Lx)
    y0 = 0.5 * (Py - Ly)
    sheet = recttri([x0, y0], [x0 + Lx, y0 + Ly], Nx, Ny)
    sheet.style = "rectstrip"
    sheet.units = units
    sheet.s1 = np.array([float(Px), 0.0])
    sheet.s2 = np.array([0.0, float(Py)])
    sheet.beta1, sheet.beta2 = s1s2_to_b1b2(sheet.s1, sheet.s2)
    sheet.fr = np.full(sheet.nface, float(kwargs["Rsheet"]))
    sheet.fufp = kwargs["fufp"]
    sheet.cls = kwargs["cls"]
    rotate(sheet, kwargs["rot"])
    if kwargs["dx"] != 0 or kwargs["dy"] != 0:
        sheet.rho = np.array([[kwargs["dx"] + x, kwargs["dy"] + y] for x, y in sheet.rho])
    sheet.xi_eta_check = (Lx == Px or Ly == Py)
    return sheet


def meander_counts(a, b, h, w1, w2, ntri):
    """Segment counts ``(nx1, nx2, ny1, ny2)`` and triangle total (``Elements.jl:635-646``)."""
    hm = h - 2 * w2
    t1 = w2 * (a + 2 * w1) / (2 * (hm * hm))
    t2 = w1 / hm
    fny2 = math.sqrt(ntri / (4 * (t1 + t2)))
    ny2 = round(fny2)
    ny2 = 1 if ny2 <= 0 else ny2
    ny1 = round(fny2 * w2 / (h - 2 * w2))
    ny1 = 1 if ny1 <= 0 else ny1
    nx1 = round(fny2 * (a - 2 * w1) / (4 * (h - 2 * w2)))
    nx1 = 1 if nx1 <= 0 else nx1
    nx2 = round(fny2 * w1 / (h - 2 * w2))
    nx2 = 1 if nx2 <= 0 else nx2
    ntotal = 4 * (2 * ny1 * (nx1 + nx2) + nx2 * ny2)
    return nx1, nx2, ny1, ny2, ntotal


def meander(*, a, b, h, w1, w2, ntri, units, orient=0.0, **kwarg):
    """Meanderline strip (``Elements.jl:617-729``)."""
    kwargs = dict(kwarg)
    kwargs.setdefault("fufp", True)
    _check_kwargs(kwargs)
    _testpos(a=a, b=b, h=h, w1=w1, w2=w2, ntri=ntri)
    if orient != 0 and a != b:
        raise ValueError("Nonzero orient only allowed for square unit cell")
    morient = orient % 360
    if morient not in (0, 90, 180, 270):
        raise ValueError("orient must be a multiple of 90")
    nx1, nx2, ny1, ny2, _ = meander_counts(a, b, h, w1, w2, ntri)
    yoffset = (b - h) / 2
    Lx = (a / 2 - w1) / 2
    Ly = h - 2 * w2

    def rt(bl, d):
        return [bl[0] + d[0], bl[1] + d[1]]

    bl = [0.0, yoffset]
    sh1 = recttri(bl, rt(bl, [Lx, w2]), nx1, ny1)
    bl = [Lx, yoffset]
    sh2 = recttri(bl, rt(bl, [w1, w2]), nx2, ny1)
    sh3 = combine(sh1, sh2, "x", Lx)
    bl = [Lx, yoffset + w2]
    sh1 = recttri(bl, rt(bl, [w1, Ly]), nx2, ny2)
    sh2 = combine(sh3, sh1, "y", bl[1])
    bl = [Lx, yoffset + w2 + Ly]
    sh1 = recttri(bl, rt(bl, [w1, w2]), nx2, ny1)
    sh3 = combine(sh2, sh1, "y", bl[1])
    bl = [Lx + w1, yoffset + w2 + Ly]
    tr = rt(bl, [2 * Lx, w2])
    sh1 = recttri(bl, tr, 2 * nx1, ny1)
    sh2 = combine(sh3, sh1, "x", bl[0])
    bl = [tr[0], bl[1]]
    tr = rt(bl, [w1, w2])
    sh1 = recttri(bl, tr, nx2, ny1)
    sh3 = combine(sh2, sh1, "x", bl[0])
    bl = [bl[0], yoffset + w2]
    tr = rt(bl, [w1, Ly])
    sh1 = recttri(bl, tr, nx2, ny2)
    sh2 = combine(sh3, sh1, "y", tr[1])
    bl = [bl[0], yoffset]
    tr = rt(bl, [w1, w2])
    sh1 = recttri(bl, tr, nx2, ny1)
    sh3 = combine(sh2, sh1, "y", tr[1])
    bl = [tr[0], yoffset]
    tr = rt(bl, [Lx, w2])
    sh1 = recttri(bl, tr, nx1, ny1)
    sheet = combine(sh3, sh1, "x", bl[0])
    if morient != 0:
        if morient == 90:
            xf = lambda x, y: (b - y, x)
        elif morient == 180:
            xf = lambda x, y: (a - x, b - y)
        else:
            xf = lambda x, y: (y, a - x)
        sheet.rho = np.array([xf(x, y) for x, y in sheet.rho], float)
    sheet.fr = np.full(sheet.nface, float(kwargs["Rsheet"]))
    sheet.fufp = kwargs["fufp"]
    sheet.cls = kwargs["cls"]
    sheet.style = "meander"
    sheet.units = units
    sheet.s1 = np.array([float(a), 0.0])
    sheet.s2 = np.array([0.0, float(b)])
    sheet.beta1, sheet.beta2 = s1s2_to_b1b2(sheet.s1, sheet.s2)
    rotate(sheet, kwargs["rot"])
    if kwargs["dx"] != 0 or kwargs["dy"] != 0:
        sheet.rho = np.array([[kwargs["dx"] + x, kwargs["dy"] + y] for x, y in sheet.rho])
    sheet.xi_eta_check = True
    return sheet

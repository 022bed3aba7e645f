"""Dielectric layer type (PSSFSS.jl ``src/Layers.jl:85-121``).

``Layer(width=..., epsr=..., tandel=..., mur=..., mtandel=...)`` builds the complex
constitutive parameters exactly as the reference does: ``ϵᵣ*complex(1,-tanδ)``, so a
lossless layer carries ``imag == -0.0`` (the sign of that zero decides branch cuts in
the modal square roots downstream).
"""
import numpy as np

from .units import Length, mm

TE = 1
TM = 2


def _creal_times(x, z):
    """Julia ``Real * Complex``: ``Complex(x*re, x*im)`` (keeps signed zeros)."""
    return complex(x * z.real, x * z.imag)


class Layer:
    def __init__(self, name="Layer", width=None, epsr=1.0, tandel=0.0, mur=1.0, mtandel=0.0,
                 **kw):
        # Greek keyword spellings accepted like the reference (Layers.jl:107-113)
        epsr = kw.pop("ϵᵣ", epsr)
        tandel = kw.pop("tanδ", tandel)
        mur = kw.pop("μᵣ", mur)
        mtandel = kw.pop("mtanδ", mtandel)
        if kw:
            raise TypeError(f"unexpected keyword(s): {sorted(kw)}")
        if width is None:
            width = Length(0, mm)
        self.name = name
        self.epsr = _creal_times(float(epsr), complex(1.0, -float(tandel)))
        self.mur = _creal_times(float(mur), complex(1.0, -float(mtandel)))
        self.user_width = width
        self.width = float(width.meters)
        self.P = []
        self.M = []
        self.N = []
        self.beta1 = np.zeros(2)
        self.beta2 = np.zeros(2)
        self.beta = np.zeros((0, 2))
        self.gamma = np.zeros(0, complex)
        self.Y = np.zeros(0, complex)
        self.c = np.zeros(0, complex)
        self.tvec = np.zeros((0, 2))

    def copy(self):
        """An independent copy: the mode lists and modal arrays are copied; the name,
        constants and width (never changed in place) are shared."""
        c = type(self).__new__(type(self))
        d = dict(self.__dict__)
        for k, v in d.items():
            if isinstance(v, list):
                d[k] = list(v)
            elif isinstance(v, np.ndarray):
                d[k] = v.copy()
        c.__dict__.update(d)
        return c

    def same_as(self, other):
        """Field-wise equality (``Layers.jl:123``) used by the Gblock duplicate search."""
        if not isinstance(other, Layer):
            return False
        for f in ("name", "epsr", "mur", "width", "P", "M", "N"):
            if getattr(self, f) != getattr(other, f):
                return False
        for f in ("beta1", "beta2", "beta", "gamma", "Y", "c", "tvec"):
            a, b = getattr(self, f), getattr(other, f)
            if np.shape(a) != np.shape(b) or not np.array_equal(a, b):
                return False
        return True

    def __repr__(self):
        return (f"{self.name}: width={self.user_width}, ϵᵣ={self.epsr.real}, "
                f"tanδ={-self.epsr.imag / self.epsr.real}, μᵣ={self.mur.real}, "
                f"{len(self.P)} modes")

"""The benchmark workloads, built from the package's own element constructors.

* ``square_patch_sweep``: an 8 mm square patch in a 10 mm cell (structured 16 x 16 strip
  mesh, 512 triangles, N = 736) in free space, normal incidence, 11 frequencies 10-20 GHz.
* ``jerusalem_aperture_cascade``: a solid Jerusalem cross (P = 8, L1 = 6, L2 = 0.5, A = 3,
  B = 0.5, w = 0.25 mm) on 0.5 mm eps_r = 3 (tan d = 0.002), a 2 mm air gap, and a square
  aperture (M-type ``polyring``, b = 6/sqrt(2) mm, 45 deg) in the same cell; 51 frequencies
  5-25 GHz at theta = 30, phi = 45 (the face-pair integrals change with every point).
* ``meander_precision_sweep``: the meanderline a = 5, b = 10, h = 6, w1 = w2 = 0.3 mm,
  ntri = 3000 (2840 triangles, N = 3976) on 1 mm eps_r = 2.2, 101 frequencies 8-18 GHz.
* ``ring_batch``: 64 seeded ring problems of differing size: period P ~ U(6, 12) mm, outer
  radius ro ~ U(0.35, 0.45) P, width 0.05 P, 48 sides, ntri ~ U{300..3000}, theta drawn from
  {0, 15, 30, 45} deg, phi = 0, free-standing, 21 frequencies 10-20 GHz.
* ``meander_gradient_workload``: the meanderline at ntri = 4000 (3960 triangles) on the same
  substrate, 201 frequencies 8-18 GHz, with its width / pitch / eps_r parameters.

Each returns ``(strata, flist, steering)`` (``ring_batch`` a list of them) for ``analyze``.
"""
import math

import numpy as np

from .elements import jerusalemcross, meander, polyring, rectstrip
from .layers import Layer
from .units import Length, mm

NORMAL = {"θ": 0.0, "ϕ": 0.0}


def square_patch_sweep():
    sheet = rectstrip(Lx=8, Ly=8, Px=10, Py=10, Nx=16, Ny=16, units=mm)
    return [Layer(), sheet, Layer()], np.linspace(10, 20, 11), dict(NORMAL)


def jerusalem_aperture_cascade(ntri_cross=1500, ntri_aperture=1200):
    cross = jerusalemcross(P=8, L1=6, L2=0.5, A=3, B=0.5, w=0.25, ntri=ntri_cross, units=mm)
    aperture = polyring(s1=[8, 0], s2=[0, 8], a=[0], b=[6 / math.sqrt(2)], sides=4, orient=45,
                        ntri=ntri_aperture, units=mm, **{"class": "M"})
    strata = [Layer(), cross, Layer(epsr=3.0, tandel=0.002, width=Length(0.5, mm)),
              Layer(width=Length(2, mm)), aperture, Layer()]
    return strata, np.linspace(5, 25, 51), {"θ": 30.0, "ϕ": 45.0}


def meander_strata(w=0.3, a=5.0, epsr=2.2, ntri=3000):
    sheet = meander(a=a, b=10, h=6, w1=w, w2=w, ntri=ntri, units=mm)
    return [Layer(), sheet, Layer(epsr=epsr, width=Length(1, mm)), Layer()]


def meander_precision_sweep():
    return meander_strata(), np.linspace(8, 18, 101), dict(NORMAL)


def ring_batch(seed=0, count=64):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        P = float(rng.uniform(6, 12))
        ro = float(rng.uniform(0.35, 0.45)) * P
        ntri = int(rng.integers(300, 3001))
        theta = float(rng.choice([0.0, 15.0, 30.0, 45.0]))
        sheet = polyring(s1=[P, 0], s2=[0, P], a=[ro - 0.05 * P], b=[ro], sides=48, ntri=ntri, units=mm)
        out.append(([Layer(), sheet, Layer()], np.linspace(10, 20, 21), {"θ": theta, "ϕ": 0.0}))
    return out


def meander_gradient_workload():
    """Parameters, frequencies and triangle count of the differentiation workload (for
    ``gradient.meander_gradient`` / ``meander_linearized_gradient``)."""
    return {"w": 0.3, "a": 5.0, "epsr": 2.2}, np.linspace(8, 18, 201), 4000

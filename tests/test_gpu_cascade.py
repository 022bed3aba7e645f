"""GSM cascade on the device (pss_cascade) against the host's numpy cascade.

The star products of every point run in one call; per point the same Gblock walk as
_analyze (PSSFSS.jl:256-305).  Stacks: a sheet on a substrate with an air gap to a second
sheet (two sheet Gblocks and bare slab interfaces), a PEC sheet, a translated sheet and a
duplicated Gblock; the sheets' partial GSMs are seeded random matrices of the plan's shapes
(the cascade is pure algebra on them) so the test isolates the cascade.  Bar: 1e-12 relative.
The default analyze path (where="auto") runs on the device whenever a GPU is present, so
every end-to-end GPU test against the oracle covers it too.
"""
import numpy as np
import pytest

from pssfss_b200.analyze import assemble, make_plan, sheet_gblocks
from pssfss_b200.elements import pecsheet, rectstrip
from pssfss_b200.gsms import GSM
from pssfss_b200.layers import Layer
from pssfss_b200.units import Length, mm

pytestmark = pytest.mark.gpu


def random_partials(plan, seed):
    rng = np.random.default_rng(seed)
    partial = {}
    for ig, (i1, i2), isht, s in sheet_gblocks(plan):
        out = []
        for pt in plan.points:
            n1, n2 = len(pt.layers[i1 - 1].P), len(pt.layers[i2 - 1].P)
            c = lambda a, b: 0.3 * (rng.standard_normal((a, b)) + 1j * rng.standard_normal((a, b)))
            out.append(GSM(c(n1, n1), c(n1, n2), c(n2, n1), c(n2, n2)))
        partial[ig] = out
    return partial


def stacks():
    j = rectstrip(Lx=6, Ly=0.5, Px=8, Py=8, Nx=4, Ny=2, units=mm)
    m = rectstrip(Lx=6, Ly=6, Px=8, Py=8, Nx=4, Ny=4, units=mm, **{"class": "M"})
    shifted = rectstrip(Lx=6, Ly=0.5, Px=8, Py=8, Nx=4, Ny=2, units=mm, dx=1.5, dy=-0.5)
    return [
        ([Layer(), j, Layer(epsr=3.0, tandel=0.002, width=Length(0.5, mm)), Layer(width=Length(2, mm)), m, Layer()],
         [5.0, 15.0, 25.0], {"θ": 30.0, "ϕ": 45.0}),
        ([Layer(), shifted, Layer(epsr=2.2, width=Length(1, mm)), Layer(width=Length(3, mm)),
          pecsheet(), Layer()], [10.0, 20.0], {"θ": 0.0, "ϕ": 0.0}),
        ([Layer(), j, Layer(epsr=2.5, width=Length(3, mm)), j, Layer(epsr=2.5, width=Length(3, mm)), j, Layer()],
         [12.0, 18.0], {"θ": 15.0, "ϕ": 0.0}),
        # thin spacers: 338 modes in the inner layers, beyond the device cascade's 64
        ([Layer(), j, Layer(epsr=2.5, width=Length(0.3, mm)), j, Layer()], [12.0], {"θ": 0.0, "ϕ": 0.0}),
    ]


@pytest.mark.parametrize("k", [0, 1, 2])
def test_device_cascade_equals_host(k):
    strata, freqs, steer = stacks()[k]
    plan = make_plan(strata, freqs, steer)
    partial = random_partials(plan, 7 + k)
    dev = assemble(plan, partial, where="device")
    host = assemble(plan, partial, where="host")
    assert len(dev) == len(host) == len(plan.points)
    for a, b in zip(dev, host):
        for blk in ("s11", "s12", "s21", "s22"):
            x, y = getattr(a.gsm, blk), getattr(b.gsm, blk)
            assert x.shape == y.shape
            assert np.max(np.abs(x - y)) <= 1e-12 * max(1.0, np.max(np.abs(y))), (k, blk)


def test_device_cascade_rejects_too_many_modes_and_auto_uses_host():
    strata, freqs, steer = stacks()[3]
    plan = make_plan(strata, freqs, steer)
    assert max(len(l.P) for l in plan.points[0].layers) > 64
    partial = random_partials(plan, 3)
    with pytest.raises(RuntimeError, match="outside 1..64"):
        assemble(plan, partial, where="device")
    auto = assemble(plan, partial)
    host = assemble(plan, partial, where="host")
    for a, b in zip(auto, host):
        assert np.array_equal(a.gsm.s21, b.gsm.s21)

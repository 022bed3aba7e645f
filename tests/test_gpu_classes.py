"""Face-pair classing of setup_rwg on the device (pss_face_pair_classes) against the host's.

The classes (translation-equivalent pairs of faces: same source shape, same quantised offset of
the match centroid from the source's first vertex, RWG.jl:287-319) and their numbering by first
appearance in column-major order must be identical - the map, the representatives and the
count - on structured sheets of several kinds and sizes, including the benchmark meanderlines.
"""
import numpy as np
import pytest

from pssfss_b200.elements import diagstrip, meander, rectstrip
from pssfss_b200.rwg import setup_rwg, unique_face_pairs
from pssfss_b200.units import mil, mm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [
    lambda: rectstrip(Lx=8, Ly=8, Px=10, Py=10, Nx=16, Ny=16, units=mm),
    lambda: rectstrip(Nx=20, Ny=20, Lx=20, Ly=50, Px=100, Py=100, units=mil),
    lambda: rectstrip(Nx=4, Ny=6, Lx=10, Ly=3, Px=10, Py=8, units=mm),
    lambda: meander(a=5, b=10, h=6, w1=0.3, w2=0.3, ntri=3000, units=mm),
    lambda: meander(a=5, b=10, h=6, w1=0.3, w2=0.3, ntri=4000, units=mm),
    # a perturbed trace width breaks most translation equivalences: 6.1M classes of 15.7M pairs
    lambda: meander(a=5, b=10, h=6, w1=0.3 * (1 + 1e-4), w2=0.3 * (1 + 1e-4), ntri=4000, units=mm),
    lambda: diagstrip(P=10, w=1.5, orient=45, Nl=20, Nw=4, units=mm),
])
def test_device_classes_equal_host(make):
    sheet = make()
    dev = unique_face_pairs(sheet, where="device")
    host = unique_face_pairs(sheet, where="host")
    assert dev[2] == host[2]
    assert np.array_equal(dev[1], host[1])
    assert np.array_equal(dev[0], host[0])
    assert setup_rwg(sheet).nufp == host[2]  # setup_rwg takes the device path here

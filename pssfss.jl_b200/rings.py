"""Square summation rings of the (m, n) lattice (PSSFSS.jl ``src/Rings.jl:9-60``).

Ring ``r`` lists its ``8r`` points in a fixed order: the ``m = r`` column
(``n = -r..r``), the ``m = -r`` column, the ``n = -r`` row (``m = 1-r..r-1``)
and the ``n = r`` row.  That order fixes the summation order of every lattice
series, so it is the same one the CUDA kernels and the oracle use.
"""


def ring_len(r):
    return 1 if r == 0 else 8 * r


def ring_mn(r, idx):
    """(m, n) of element ``idx`` (0-based) of ring ``r``."""
    if r == 0:
        return (0, 0)
    w = 2 * r + 1
    if idx < w:
        return (r, -r + idx)
    idx -= w
    if idx < w:
        return (-r, -r + idx)
    idx -= w
    h = 2 * r - 1
    if idx < h:
        return (-r + 1 + idx, -r)
    idx -= h
    return (-r + 1 + idx, r)


class Ring:
    """Iterator over the (m, n) pairs of ring ``r`` (``Rings.jl:9``)."""

    def __init__(self, r):
        if r < 0:
            raise ValueError("ring must be non-negative")
        self.r = r

    def __len__(self):
        return ring_len(self.r)

    def __iter__(self):
        for i in range(ring_len(self.r)):
            yield ring_mn(self.r, i)

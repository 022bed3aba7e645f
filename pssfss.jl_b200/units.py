"""Length units (PSSFSS.jl ``src/PSSFSSLen.jl:141-145``).

The reference uses Unitful, whose conversions are exact rationals turned into a
Float64 at the end.  Each unit here carries its exact size in metres as a
``fractions.Fraction`` so that ``units_per_meter`` and layer widths round the
same way (``ustrip(Float64, mm, 1u"m") == 1000.0``, ``mil -> 5000000/127``).
"""
from fractions import Fraction


class LengthUnit:
    __slots__ = ("name", "meters")

    def __init__(self, name, meters):
        self.name = name
        self.meters = Fraction(meters)

    @property
    def units_per_meter(self):
        """``ustrip(Float64, unit, 1u"m")``."""
        return float(1 / self.meters)

    def to_meters(self, value):
        """``ustrip(u"m", value*unit)`` with exact-rational conversion for ints."""
        if isinstance(value, int):
            return float(Fraction(value) * self.meters)
        return float(value) * float(self.meters)

    def __rmul__(self, value):
        return Length(value, self)

    def __eq__(self, other):
        return isinstance(other, LengthUnit) and self.name == other.name

    def __hash__(self):
        return hash(self.name)

    def __repr__(self):
        return self.name


class Length:
    """A length quantity ``value*unit`` (the reference's ``Unitful.Length``)."""
    __slots__ = ("value", "unit")

    def __init__(self, value, unit):
        self.value = value
        self.unit = unit

    @property
    def meters(self):
        return self.unit.to_meters(self.value)

    def __repr__(self):
        return f"{self.value} {self.unit.name}"


m = LengthUnit("m", 1)
mm = LengthUnit("mm", Fraction(1, 1000))
cm = LengthUnit("cm", Fraction(1, 100))
inch = LengthUnit("inch", Fraction(254, 10000))
mil = LengthUnit("mil", Fraction(254, 10000000))

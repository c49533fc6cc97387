"""ORACLE-ONLY import shim for LSSTDESC.Coord (not installed here).

The reference GalSim package imports ``coord`` at module load (galsim/angle.py:22,
galsim/celestial.py).  Only the angle units are exercised by the FFT drawing path
(e.g. Kolmogorov/Airy ``scale_unit``, ``GSObject.rotate``); this shim implements those
and leaves celestial coordinates as an inert placeholder.
"""
import math


class AngleUnit(object):
    def __init__(self, value):
        self.value = float(value)

    def __rmul__(self, theta):
        return Angle(theta, self)

    def __truediv__(self, unit):
        return self.value / unit.value

    def __eq__(self, other):
        return isinstance(other, AngleUnit) and self.value == other.value

    def __hash__(self):
        return hash(self.value)

    @staticmethod
    def from_name(name):
        name = name.strip().lower()
        for key, unit in (('rad', radians), ('deg', degrees), ('hour', hours),
                          ('arcmin', arcmin), ('arcsec', arcsec)):
            if name.startswith(key):
                return unit
        raise ValueError("Unknown Angle unit: %s" % name)


radians = AngleUnit(1.)
degrees = AngleUnit(math.pi / 180.)
hours = AngleUnit(math.pi / 12.)
arcmin = AngleUnit(math.pi / 180. / 60.)
arcsec = AngleUnit(math.pi / 180. / 3600.)


class Angle(object):
    def __init__(self, theta, unit=None):
        if isinstance(theta, Angle):
            self._rad = theta._rad
        else:
            self._rad = float(theta) * (unit.value if unit is not None else 1.)

    @property
    def rad(self):
        return self._rad

    @property
    def deg(self):
        return self._rad / degrees.value

    def __truediv__(self, unit):
        if isinstance(unit, AngleUnit):
            return self._rad / unit.value
        return _Angle(self._rad / unit)

    def __mul__(self, x):
        return _Angle(self._rad * x)

    __rmul__ = __mul__

    def __add__(self, other):
        return _Angle(self._rad + other._rad)

    def __sub__(self, other):
        return _Angle(self._rad - other._rad)

    def __neg__(self):
        return _Angle(-self._rad)

    def __eq__(self, other):
        return isinstance(other, Angle) and self._rad == other._rad

    def __hash__(self):
        return hash(self._rad)

    def sin(self):
        return math.sin(self._rad)

    def cos(self):
        return math.cos(self._rad)

    def tan(self):
        return math.tan(self._rad)

    def sincos(self):
        return math.sin(self._rad), math.cos(self._rad)

    def wrap(self, center=None):
        c = 0. if center is None else center._rad
        r = self._rad - c
        r -= 2. * math.pi * math.floor((r + math.pi) / (2. * math.pi))
        return _Angle(r + c)


def _Angle(theta):
    a = Angle.__new__(Angle)
    a._rad = theta
    return a


class CelestialCoord(object):
    """Placeholder; celestial coordinates are not used on the FFT drawing path."""
    def __init__(self, *args, **kwargs):
        raise NotImplementedError("CelestialCoord is not available in the oracle shim")

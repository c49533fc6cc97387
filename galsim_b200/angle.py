"""Angle units (the reference re-exports LSSTDESC.Coord's, galsim/angle.py:22)."""
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
        for key, unit in (('rad', radians), ('deg', degrees), ('hour', hours), ('arcmin', arcmin),
                          ('arcsec', arcsec)):
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
            if unit is None:
                raise TypeError("Angle requires a unit")
            self._rad = float(theta) * unit.value

    @property
    def rad(self):
        return self._rad

    @property
    def deg(self):
        return self._rad / degrees.value

    def __truediv__(self, unit):
        return self._rad / unit.value

    def __mul__(self, x):
        return _Angle(self._rad * x)

    __rmul__ = __mul__

    def __neg__(self):
        return _Angle(-self._rad)

    def __add__(self, other):
        return _Angle(self._rad + other._rad)

    def __sub__(self, other):
        return _Angle(self._rad - other._rad)

    def __eq__(self, other):
        return isinstance(other, Angle) and self._rad == other._rad

    def __hash__(self):
        return hash(self._rad)

    def sin(self):
        return math.sin(self._rad)

    def cos(self):
        return math.cos(self._rad)

    def sincos(self):
        return math.sin(self._rad), math.cos(self._rad)

    def tan(self):
        return math.tan(self._rad)

    def __repr__(self):
        return 'galsim.Angle(%r, galsim.radians)' % self._rad


def _Angle(theta):
    a = Angle.__new__(Angle)
    a._rad = theta
    return a


__all__ = ['Angle', 'AngleUnit', '_Angle', 'radians', 'degrees', 'hours', 'arcmin', 'arcsec']

"""BoundsI / BoundsD (galsim/bounds.py), the subset the drawing path uses."""
import math

import numpy as np

from .errors import GalSimUndefinedBoundsError
from .position import PositionD, PositionI, _PositionD, _PositionI


class Bounds(object):
    def __init__(self, *args, **kwargs):
        self._isdefined = True
        if len(args) == 4 and not kwargs:
            self.xmin, self.xmax, self.ymin, self.ymax = [self._cast(a) for a in args]
        elif len(args) == 0 and not kwargs:
            self._isdefined = False
            self.xmin = self.xmax = self.ymin = self.ymax = 0
        elif len(args) == 0:
            self.xmin = self._cast(kwargs.pop('xmin'))
            self.xmax = self._cast(kwargs.pop('xmax'))
            self.ymin = self._cast(kwargs.pop('ymin'))
            self.ymax = self._cast(kwargs.pop('ymax'))
        elif len(args) == 1 and isinstance(args[0], Bounds):
            b = args[0]
            self._isdefined = b._isdefined
            self.xmin, self.xmax, self.ymin, self.ymax = b.xmin, b.xmax, b.ymin, b.ymax
        else:
            raise TypeError("Bounds requires 4 values or another Bounds")
        if self.xmin > self.xmax or self.ymin > self.ymax:
            self._isdefined = False

    def isDefined(self):
        return self._isdefined

    def _getinitargs(self):
        return (self.xmin, self.xmax, self.ymin, self.ymax)

    @property
    def true_center(self):
        if not self.isDefined():
            raise GalSimUndefinedBoundsError("true_center is invalid for an undefined Bounds")
        return _PositionD((self.xmin + self.xmax) / 2., (self.ymin + self.ymax) / 2.)

    def includes(self, *args):
        if len(args) == 1 and isinstance(args[0], Bounds):
            b = args[0]
            return (self.isDefined() and b.isDefined() and self.xmin <= b.xmin and
                    self.xmax >= b.xmax and self.ymin <= b.ymin and self.ymax >= b.ymax)
        if len(args) == 1:
            x, y = args[0].x, args[0].y
        else:
            x, y = args
        return self.isDefined() and self.xmin <= x <= self.xmax and self.ymin <= y <= self.ymax

    def __eq__(self, other):
        return (self is other or (isinstance(other, Bounds) and type(self) == type(other) and
                ((not self.isDefined() and not other.isDefined()) or
                 (self.isDefined() and other.isDefined() and
                  self._getinitargs() == other._getinitargs()))))

    def __ne__(self, other):
        return not self.__eq__(other)

    def __hash__(self):
        return hash((type(self).__name__, self._getinitargs()))

    def __repr__(self):
        if self.isDefined():
            return 'galsim.%s(xmin=%r, xmax=%r, ymin=%r, ymax=%r)' % (
                type(self).__name__, self.xmin, self.xmax, self.ymin, self.ymax)
        return 'galsim.%s()' % type(self).__name__


class BoundsD(Bounds):
    @staticmethod
    def _cast(v):
        return float(v)


class BoundsI(Bounds):
    @staticmethod
    def _cast(v):
        return int(v)

    def numpyShape(self):
        if self.isDefined():
            return (self.ymax - self.ymin + 1, self.xmax - self.xmin + 1)
        return (0, 0)

    @property
    def center(self):
        """The integer center, up and right of the true center for even sizes
        (galsim/bounds.py:448-455)."""
        if not self.isDefined():
            raise GalSimUndefinedBoundsError("center is invalid for an undefined Bounds")
        return _PositionI(self.xmin + (self.xmax - self.xmin + 1) // 2,
                          self.ymin + (self.ymax - self.ymin + 1) // 2)

    def shift(self, delta):
        return BoundsI(self.xmin + delta.x, self.xmax + delta.x, self.ymin + delta.y,
                       self.ymax + delta.y)

    def withBorder(self, dx, dy=None):
        dy = dx if dy is None else dy
        return BoundsI(self.xmin - dx, self.xmax + dx, self.ymin - dy, self.ymax + dy)


def _BoundsI(xmin, xmax, ymin, ymax):
    b = BoundsI.__new__(BoundsI)
    b.xmin, b.xmax, b.ymin, b.ymax = int(xmin), int(xmax), int(ymin), int(ymax)
    b._isdefined = xmin <= xmax and ymin <= ymax
    return b


__all__ = ['Bounds', 'BoundsD', 'BoundsI', '_BoundsI']

"""PositionD / PositionI (galsim/position.py), the subset the drawing path uses."""
import numpy as np


class Position(object):
    def __init__(self, *args, **kwargs):
        if len(kwargs) == 0:
            if len(args) == 2:
                x, y = args
            elif len(args) == 0:
                x = y = 0
            elif len(args) == 1:
                a = args[0]
                if isinstance(a, Position):
                    x, y = a.x, a.y
                else:
                    x, y = a[0], a[1]
            else:
                raise TypeError("Too many arguments for Position")
        else:
            x = kwargs.pop('x')
            y = kwargs.pop('y')
            if kwargs:
                raise TypeError("Got unexpected keyword arguments %s" % kwargs.keys())
        self.x = self._cast(x)
        self.y = self._cast(y)

    def __add__(self, other):
        return self._make(self.x + other.x, self.y + other.y)

    def __sub__(self, other):
        return self._make(self.x - other.x, self.y - other.y)

    def __neg__(self):
        return self._make(-self.x, -self.y)

    def __mul__(self, s):
        return PositionD(self.x * s, self.y * s)

    __rmul__ = __mul__

    def __eq__(self, other):
        return isinstance(other, Position) and self.x == other.x and self.y == other.y

    def __ne__(self, other):
        return not self.__eq__(other)

    def __hash__(self):
        return hash((type(self).__name__, self.x, self.y))

    def __iter__(self):
        return iter((self.x, self.y))

    def __getitem__(self, i):
        return (self.x, self.y)[i]

    def __repr__(self):
        return 'galsim.%s(x=%r, y=%r)' % (type(self).__name__, self.x, self.y)


class PositionD(Position):
    @staticmethod
    def _cast(v):
        return float(v)

    def _make(self, x, y):
        return PositionD(x, y)


class PositionI(Position):
    @staticmethod
    def _cast(v):
        if isinstance(v, (float, np.floating)) and v != int(v):
            raise TypeError("PositionI must have integer values")
        return int(v)

    def _make(self, x, y):
        if isinstance(x, (int, np.integer)) and isinstance(y, (int, np.integer)):
            return PositionI(x, y)
        return PositionD(x, y)


def _PositionD(x, y):
    p = PositionD.__new__(PositionD)
    p.x = float(x)
    p.y = float(y)
    return p


def _PositionI(x, y):
    p = PositionI.__new__(PositionI)
    p.x = int(x)
    p.y = int(y)
    return p


def parse_pos_args(args, kwargs, name1, name2, integer=False, others=[]):
    """Parse (x, y), a Position, or x=, y= keyword forms (galsim/utilities.py parse_pos_args)."""
    cls = PositionI if integer else PositionD
    other_vals = []
    if len(args) == 0:
        pos = cls(kwargs.pop(name1), kwargs.pop(name2))
    elif len(args) == 1:
        a = args[0]
        pos = a if isinstance(a, Position) else cls(a[0], a[1])
    elif len(args) == 2:
        pos = cls(args[0], args[1])
    else:
        raise TypeError("Too many arguments")
    for o in others:
        other_vals.append(kwargs.pop(o))
    if kwargs:
        raise TypeError("Received unexpected keyword arguments: %s" % kwargs)
    return (pos,) + tuple(other_vals) if others else pos


__all__ = ['Position', 'PositionD', 'PositionI', '_PositionD', '_PositionI']

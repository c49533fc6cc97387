"""Shear (galsim/shear.py): reduced shear g = g1 + i g2 and its 2x2 distortion matrix.

g1, g2 may be numpy arrays (one shear per stamp of a batch); getMatrix then returns an
array of shape (B, 2, 2)."""
import math

import numpy as np

from .angle import Angle
from .errors import GalSimIncompatibleValuesError, GalSimRangeError


class Shear(object):
    def __init__(self, *args, **kwargs):
        if len(args) == 1:
            if kwargs:
                raise TypeError("Gave both unnamed and named arguments to Shear")
            a = args[0]
            if isinstance(a, Shear):
                self._g1, self._g2 = a._g1, a._g2
                return
            if not isinstance(a, complex):
                raise TypeError("Non-keyword argument to Shear must be complex g1 + 1j * g2")
            self._g1, self._g2 = a.real, a.imag
        elif len(args) > 1:
            raise TypeError("Too many unnamed arguments to Shear")
        elif len(kwargs) == 0:
            self._g1 = self._g2 = 0.
        elif 'g1' in kwargs or 'g2' in kwargs:
            self._g1 = _arr(kwargs.pop('g1', 0.))
            self._g2 = _arr(kwargs.pop('g2', 0.))
            if np.any(self._g1 ** 2 + self._g2 ** 2 > 1.):
                raise GalSimRangeError("Requested shear exceeds 1.", self.g, 0., 1.)
        elif 'e1' in kwargs or 'e2' in kwargs:
            e1 = _arr(kwargs.pop('e1', 0.))
            e2 = _arr(kwargs.pop('e2', 0.))
            absesq = e1 ** 2 + e2 ** 2
            if np.any(absesq > 1.):
                raise GalSimRangeError("Requested distortion exceeds 1.", np.sqrt(absesq), 0., 1.)
            f = _e2g(absesq)
            self._g1, self._g2 = e1 * f, e2 * f
        elif 'eta1' in kwargs or 'eta2' in kwargs:
            eta1 = _arr(kwargs.pop('eta1', 0.))
            eta2 = _arr(kwargs.pop('eta2', 0.))
            eta = np.hypot(eta1, eta2)
            f = np.where(eta > 1.e-4, np.tanh(0.5 * eta) / np.where(eta > 0, eta, 1.), 0.5)
            self._g1, self._g2 = eta1 * f, eta2 * f
        elif 'g' in kwargs or 'e' in kwargs or 'eta' in kwargs or 'q' in kwargs:
            if 'beta' not in kwargs:
                raise GalSimIncompatibleValuesError(
                    "Shear constructor requires beta when g, e, eta or q is specified.")
            beta = kwargs.pop('beta')
            if not isinstance(beta, Angle):
                raise TypeError("beta must be an Angle instance.")
            if 'g' in kwargs:
                g = kwargs.pop('g')
                if not 0 <= g <= 1:
                    raise GalSimRangeError("Requested shear exceeds 1.", g, 0., 1.)
            elif 'e' in kwargs:
                e = kwargs.pop('e')
                if not 0 <= e <= 1:
                    raise GalSimRangeError("Requested distortion exceeds 1.", e, 0., 1.)
                g = e * _e2g(e * e)
            elif 'eta' in kwargs:
                eta = kwargs.pop('eta')
                g = math.tanh(0.5 * eta)
            else:
                q = kwargs.pop('q')
                if not 0 < q <= 1:
                    raise GalSimRangeError("Cannot use requested axis ratio.", q, 0., 1.)
                g = (1. - q) / (1. + q)
            s, c = (2. * beta).sincos()
            self._g1, self._g2 = g * c, g * s
        else:
            raise TypeError("Invalid keyword arguments for Shear: %s" % kwargs)
        if kwargs:
            raise TypeError("Shear got unexpected extra arguments: %s" % kwargs)

    @property
    def g1(self):
        return self._g1

    @property
    def g2(self):
        return self._g2

    @property
    def g(self):
        return np.hypot(self._g1, self._g2) if np.ndim(self._g1) else math.hypot(self._g1, self._g2)

    @property
    def shear(self):
        return complex(self._g1, self._g2)

    def getMatrix(self):
        """[[1+g1, g2], [g2, 1-g1]] / sqrt(1-g^2)  (galsim/shear.py:365-386)."""
        g1, g2 = self._g1, self._g2
        if np.ndim(g1) == 0 and np.ndim(g2) == 0:
            return np.array([[1. + g1, g2], [g2, 1. - g1]]) / np.sqrt(1. - (g1 ** 2 + g2 ** 2))
        g1, g2 = np.broadcast_arrays(np.asarray(g1, float), np.asarray(g2, float))
        m = np.empty(g1.shape + (2, 2))
        m[..., 0, 0] = 1. + g1
        m[..., 0, 1] = g2
        m[..., 1, 0] = g2
        m[..., 1, 1] = 1. - g1
        return m / np.sqrt(1. - (g1 ** 2 + g2 ** 2))[..., None, None]

    def __eq__(self, other):
        return (isinstance(other, Shear) and np.array_equal(self._g1, other._g1) and
                np.array_equal(self._g2, other._g2))

    def __repr__(self):
        return 'galsim.Shear(g1=%r, g2=%r)' % (self._g1, self._g2)


def _arr(v):
    return np.asarray(v, float) if np.ndim(v) else float(v)


def _e2g(absesq):
    absesq = np.asarray(absesq, float)
    out = np.where(absesq > 1.e-4, 1. / (1. + np.sqrt(np.clip(1. - absesq, 0., None))), 0.5 + absesq * (0.125 + absesq * (0.0625 + absesq * 0.0390625)))
    return float(out) if out.ndim == 0 else out


def _Shear(shear):
    s = Shear.__new__(Shear)
    s._g1, s._g2 = shear.real, shear.imag
    return s


__all__ = ['Shear', '_Shear']

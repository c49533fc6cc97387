"""Box and Pixel (box.py:30-175): flux * sinc(kx w / 2 pi) sinc(ky h / 2 pi) in k space."""
import numpy as np

from . import _lib
from .gsobject import _as_param, _plen
from .gsparams import GSParams
from .profiles import _Leaf, _eq


class Box(_Leaf):
    _has_hard_edges = True
    _is_axisymmetric = False
    _type = _lib.BOX

    def __init__(self, width, height, flux=1., gsparams=None):
        self._width = _as_param(width)
        self._height = _as_param(height)
        self._flux = _as_param(flux)
        self._gsparams = GSParams.check(gsparams)
        self._batch = _plen(self._width, self._height, self._flux)

    width = property(lambda self: self._width)
    height = property(lambda self: self._height)

    def _params(self):
        return (self._width, self._height)

    def withFlux(self, flux):
        return Box(width=self.width, height=self.height, flux=flux, gsparams=self.gsparams)

    def __eq__(self, other):
        return self is other or (isinstance(other, Box) and _eq(self.width, other.width) and
                                 _eq(self.height, other.height) and _eq(self.flux, other.flux) and
                                 self.gsparams == other.gsparams)

    def __hash__(self):
        return hash(("galsim.Box", str(self.width), str(self.height), str(self.flux), self.gsparams))

    def __repr__(self):
        return 'galsim.Box(width=%r, height=%r, flux=%r, gsparams=%r)' % (
            self.width, self.height, self.flux, self.gsparams)


class Pixel(Box):
    """A square Box of side ``scale`` (box.py:139-175)."""

    def __init__(self, scale, flux=1., gsparams=None):
        super(Pixel, self).__init__(width=scale, height=scale, flux=flux, gsparams=gsparams)

    @property
    def scale(self):
        return self.width

    def withFlux(self, flux):
        return Pixel(scale=self.scale, flux=flux, gsparams=self.gsparams)

    def __repr__(self):
        return 'galsim.Pixel(scale=%r, flux=%r, gsparams=%r)' % (self.scale, self.flux, self.gsparams)


__all__ = ['Box', 'Pixel']

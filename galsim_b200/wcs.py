"""PixelScale WCS (galsim/wcs.py:1489-1606): the uniform pixel scale the FFT path needs."""
import numpy as np

from .position import PositionD, _PositionD


class BaseWCS(object):
    _isPixelScale = False
    _isUniform = False


class PixelScale(BaseWCS):
    """u = x * scale, v = y * scale."""
    _isPixelScale = True
    _isUniform = True
    _isLocal = True

    def __init__(self, scale):
        self._scale = float(scale)

    @property
    def scale(self):
        return self._scale

    def local(self, image_pos=None, world_pos=None, color=None):
        return self

    def pixelArea(self):
        return self._scale ** 2

    def shiftOrigin(self, origin, world_origin=None):
        # Only the scale matters for drawing in image coordinates.
        return self

    def profileToImage(self, world_profile, image_pos=None, world_pos=None, color=None,
                       flux_ratio=1., offset=(0, 0)):
        """The profile in image coordinates (wcs.py:386-403, 1550-1558)."""
        from .compound import _Transform
        if self._scale == 1.:
            j = None
        else:
            inv = 1. / self._scale
            j = np.array(((inv, 0.), (0., inv)))
        offset = PositionD(offset)
        return _Transform(world_profile, j, flux_ratio=self._scale ** 2 * flux_ratio,
                          offset=(offset.x, offset.y))

    toImage = profileToImage

    def __eq__(self, other):
        return isinstance(other, PixelScale) and self._scale == other._scale

    def __hash__(self):
        return hash(('galsim.PixelScale', self._scale))

    def __repr__(self):
        return 'galsim.PixelScale(%r)' % self._scale


__all__ = ['BaseWCS', 'PixelScale']

"""Interpolants for InterpolatedImage (galsim/interpolant.py).

The classes carry what InterpolatedImage needs on the host: the kernel's support (xrange,
ixrange), its Fourier extent (urange, krange), GSParams handling, equality and names.  Their
kernels run on the GPU (galsim_b200/csrc/gsb_interp.cuh): Delta (as x interpolant only),
Nearest, Linear, Cubic and Quintic.  Lanczos and SincInterpolant can be constructed, but an
InterpolatedImage using them raises GalSimNotImplementedError when it is sized or drawn.
"""
import math

from . import _lib
from .errors import GalSimValueError
from .gsparams import GSParams


class Interpolant(object):
    """Base class (interpolant.py:33-220)."""
    _code = None          # GSB_INTERP_* of the kernels built on the GPU, or None

    def __init__(self, gsparams=None):
        self._gsparams = GSParams.check(gsparams)

    @staticmethod
    def from_name(name, tol=None, gsparams=None):
        """Interpolant.from_name (interpolant.py:64-110): 'delta', 'nearest', 'sinc',
        'linear', 'cubic', 'quintic' or 'lanczosN' with optional 'F' / 'T' (conserve_dc)."""
        if tol is not None:
            gsparams = GSParams(kvalue_accuracy=tol)
        gsparams = GSParams.check(gsparams)
        name_l = name.lower()
        if name_l.startswith('lanczos'):
            conserve_dc = True
            body = name_l[7:]
            if body.endswith('f'):
                conserve_dc = False
                body = body[:-1]
            elif body.endswith('t'):
                body = body[:-1]
            try:
                n = int(body)
            except ValueError:
                raise GalSimValueError("Invalid Lanczos specification %s.  Should look like "
                                       "lanczosN, where N is an integer" % name, name) from None
            return Lanczos(n, conserve_dc, gsparams=gsparams)
        cls = {'linear': Linear, 'cubic': Cubic, 'quintic': Quintic, 'sinc': SincInterpolant,
               'nearest': Nearest, 'delta': Delta}.get(name_l)
        if cls is None:
            raise GalSimValueError("Invalid Interpolant name %s." % name, name,
                                   ('linear', 'cubic', 'quintic', 'lanczosN', 'nearest', 'delta',
                                    'sinc'))
        return cls(gsparams=gsparams)

    @property
    def gsparams(self):
        return self._gsparams

    def withGSParams(self, gsparams=None, **kwargs):
        if gsparams == self.gsparams and not kwargs:
            return self
        import copy
        ret = copy.copy(self)
        ret._gsparams = GSParams.check(gsparams, self.gsparams, **kwargs)
        return ret

    @property
    def urange(self):
        """The extent of the kernel's Fourier transform in cycles per sample (krange / 2 pi)."""
        return self.krange / (2. * math.pi)

    def _args(self):
        return ()

    def __eq__(self, other):
        return (self is other or
                (type(self) is type(other) and self._args() == other._args() and
                 self.gsparams == other.gsparams))

    def __ne__(self, other):
        return not self.__eq__(other)

    def __hash__(self):
        return hash(('galsim.' + type(self).__name__,) + self._args() + (self.gsparams,))

    def __repr__(self):
        args = ''.join('%r, ' % a for a in self._args())
        return 'galsim.%s(%sgsparams=%r)' % (type(self).__name__, args, self.gsparams)

    def __str__(self):
        return 'galsim.%s(%s)' % (type(self).__name__, ', '.join(str(a) for a in self._args()[:1]))


class Delta(Interpolant):
    """Delta-function interpolation (interpolant.py:222-283); x interpolant only."""
    _code = _lib.INTERP_DELTA
    xrange = property(lambda self: 0.)
    ixrange = property(lambda self: 0)
    krange = property(lambda self: 2. * math.pi / self._gsparams.kvalue_accuracy)


class Nearest(Interpolant):
    """Nearest-neighbour (boxcar) interpolation (interpolant.py:285-347)."""
    _code = _lib.INTERP_NEAREST
    xrange = property(lambda self: 0.5)
    ixrange = property(lambda self: 1)
    krange = property(lambda self: 2. / self._gsparams.kvalue_accuracy)


class SincInterpolant(Interpolant):
    """Sinc interpolation (interpolant.py:349-417); not built on the GPU (infinite support)."""
    xrange = property(lambda self: 1. / (math.pi * self._gsparams.kvalue_accuracy))
    ixrange = property(lambda self: 2 * int(math.ceil(self.xrange)))
    krange = property(lambda self: math.pi)


class Linear(Interpolant):
    """Linear interpolation (interpolant.py:419-485)."""
    _code = _lib.INTERP_LINEAR
    xrange = property(lambda self: 1.)
    ixrange = property(lambda self: 2)
    krange = property(lambda self: 2. / self._gsparams.kvalue_accuracy ** 0.5)


class Cubic(Interpolant):
    """Cubic interpolation (interpolant.py:487-554)."""
    _code = _lib.INTERP_CUBIC
    xrange = property(lambda self: 2.)
    ixrange = property(lambda self: 4)
    # kmax = 2 (3 sqrt(3) / 8 tol)^(1/3)
    krange = property(lambda self: 1.7320508075688774 / self._gsparams.kvalue_accuracy ** (1. / 3.))


class Quintic(Interpolant):
    """Quintic interpolation (interpolant.py:556-602), the default of InterpolatedImage."""
    _code = _lib.INTERP_QUINTIC
    xrange = property(lambda self: 3.)
    ixrange = property(lambda self: 6)
    # kmax = 2 (25 sqrt(5) / 108 tol)^(1/3)
    krange = property(lambda self: 1.6058208066649935 / self._gsparams.kvalue_accuracy ** (1. / 3.))


class Lanczos(Interpolant):
    """Lanczos filter sinc(x) sinc(x / n) (interpolant.py:604-670); not built on the GPU."""

    def __init__(self, n, conserve_dc=True, tol=None, gsparams=None):
        if tol is not None:
            gsparams = GSParams(kvalue_accuracy=tol)
        self._n = int(n)
        self._conserve_dc = bool(conserve_dc)
        self._gsparams = GSParams.check(gsparams)

    n = property(lambda self: self._n)
    conserve_dc = property(lambda self: self._conserve_dc)
    xrange = property(lambda self: self._n)
    ixrange = property(lambda self: 2 * self._n)

    @property
    def krange(self):
        from .errors import GalSimNotImplementedError
        raise GalSimNotImplementedError("Lanczos interpolants are not built on the GPU")

    def _args(self):
        return (self._n, self._conserve_dc)


def convert_interpolant(interpolant):
    """An Interpolant, or one made from its name (interpolant.py:672-685)."""
    if isinstance(interpolant, Interpolant):
        return interpolant
    return Interpolant.from_name(interpolant)


__all__ = ['Interpolant', 'Delta', 'Nearest', 'SincInterpolant', 'Linear', 'Cubic', 'Quintic',
           'Lanczos', 'convert_interpolant']

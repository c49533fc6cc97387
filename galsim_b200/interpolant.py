"""Interpolants for InterpolatedImage (galsim/interpolant.py).

The classes carry what InterpolatedImage needs on the host: the kernel's support (xrange,
ixrange), its Fourier extent (urange, krange), GSParams handling, equality and names.  Their
kernels run on the GPU (galsim_b200/csrc/gsb_interp.cuh): Delta (as x interpolant only),
Nearest, Linear, Cubic and Quintic, Lanczos as the x interpolant (its transform tabulated
on the host exactly as the reference tabulates it, then read from a device table) and as the
k interpolant for n <= 3, and SincInterpolant as the x interpolant.  Sinc and larger Lanczos
k interpolants can be constructed, but an InterpolatedImage using them raises
GalSimNotImplementedError when it is sized or drawn.
"""
import math

import numpy as np

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
    """Sinc interpolation (interpolant.py:349-417): as the x interpolant its transform is the
    box |u| < 1/2 (SincInterpolant::uval); as the k interpolant (infinite support) it is not
    built."""
    _code = _lib.INTERP_SINC
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


def _si(x):
    """The sine integral Si(x) = int_0^x sin(t) / t dt (FP64)."""
    from scipy.special import sici
    return sici(x)[0]


class _LanczosTable(object):
    """The Fourier transform of the Lanczos kernel tabulated as the reference tabulates it
    (Lanczos::Lanczos, uCalc, uCalcRaw; src/Interpolant.cpp:719-895): the kernel's transform
        F(u) = [(vm - 1) Si(pi (vm - 1)) - (vm + 1) Si(pi (vm + 1))
                - (vp - 1) Si(pi (vp - 1)) + (vp + 1) Si(pi (vp + 1))] / 2 pi,
        vp = n (2u + 1),  vm = n (2u - 1),
    with conserve_dc the convolution by the transform of the DC-correcting factor
    sum_j C_j (F(u - j) + F(u + j)) built from K_j = F(j), j = 1..5.  The table's abscissae are
    u = 0, du, 2 du, ... (accumulated by repeated addition, du = table_spacing
    (kvalue_accuracy / 200)^(1/4) / n) until u - uMax >= 1/n and u >= 1.1, where uMax is the
    last u with |F| > kvalue_accuracy; F is interpolated by a natural cubic spline.  The
    device reads the nodes as (u, F, F'') in one buffer (device())."""
    _cache = {}

    def __init__(self, n, conserve_dc, table_spacing, kvalue_accuracy):
        nd = float(n)
        self.n = n

        def raw(u):
            u = np.asarray(u, dtype=float)
            vp = nd * (2. * u + 1.)
            vm = nd * (2. * u - 1.)
            r = ((vm - 1.) * _si(math.pi * (vm - 1.)) - (vm + 1.) * _si(math.pi * (vm + 1.)) -
                 (vp - 1.) * _si(math.pi * (vp - 1.)) + (vp + 1.) * _si(math.pi * (vp + 1.)))
            return r / (2. * math.pi)

        K = [0.] + [float(raw(float(j))) for j in range(1, 6)]
        C = [1. + 2. * (K[1] * (1. + 3. * K[1] + K[2] + K[3]) + K[2] + K[3] + K[4] + K[5]),
             -K[1] * (1. + 4. * K[1] + K[2] + 2. * K[3]),
             K[1] * (K[1] - 2. * K[2] + K[3]) - K[2],
             K[1] * (K[1] - 2. * K[3]) - K[3],
             K[1] * K[3] - K[4],
             -K[5]]
        self.K, self.C = K, C

        def ucalc(u):
            r = raw(u)
            if conserve_dc:
                r = r * C[0]
                for j in range(1, 6):
                    r = r + C[j] * (raw(u + j) + raw(u - j))
            return r

        ustep = table_spacing * (kvalue_accuracy / 200.) ** 0.25 / nd
        # the reference's loop: for (u = 0; u - uMax < 1/n || u < 1.1; u += du) { add u;
        # uMax = u where |F(u)| > kvalue_accuracy }; the abscissae are accumulated in its
        # order, the values evaluated a chunk at a time and the loop condition walked in order
        us, vals = [], np.empty(0)
        u = 0.
        umax = 0.
        k = 0
        while True:
            if k == len(us):
                chunk = []
                for _ in range(1024):
                    chunk.append(u)
                    u += ustep
                us.extend(chunk)
                vals = np.concatenate([vals, ucalc(np.array(chunk))])
            uk = us[k]
            if not (uk - umax < 1. / nd or uk < 1.1):
                break
            if abs(vals[k]) > kvalue_accuracy:
                umax = uk
            k += 1
        us, vals = us[:k], vals[:k]
        from .table import _LookupTable
        self.umax = umax
        self.table = _LookupTable(np.array(us), np.array(vals), 'spline')
        self.conserve_dc = conserve_dc

    @classmethod
    def get(cls, n, conserve_dc, gsparams):
        key = (n, conserve_dc, gsparams.table_spacing, gsparams.kvalue_accuracy)
        t = cls._cache.get(key)
        if t is None:
            t = cls(n, conserve_dc, gsparams.table_spacing, gsparams.kvalue_accuracy)
            cls._cache[key] = t
        return t

    def uval(self, u):
        """F(|u|), 0 beyond uMax (Lanczos::uval)."""
        u = np.abs(np.asarray(u, dtype=float))
        v = self.table(np.minimum(u, self.table.x_max))
        return np.where(u > self.umax, 0., v)

    def kdevice(self):
        """The kernel's coefficients for its use as the k interpolant (Lanczos::xCalc): one FP64
        device buffer {n, conserve_dc, K_1 .. K_5, 0}."""
        import torch
        dev = _lib.Device.torch_device()
        key = ('kdev', dev.index)
        t = self.__dict__.get(key)
        if t is None:
            a = np.array([self.n, 1. if self.conserve_dc else 0.] + list(self.K[1:6]) + [0.])
            t = torch.from_numpy(a).to(dev)
            self.__dict__[key] = t
        return t

    def device(self):
        """The table as one FP64 device buffer of 4 (n + 1) doubles: a header (node count,
        mean spacing, u of the first node, uMax), then per node (u, F(u), F''(u), 0)."""
        import torch
        dev = _lib.Device.torch_device()
        key = ('dev', dev.index)
        t = self.__dict__.get(key)
        if t is None:
            tb = self.table
            n = len(tb.x)
            a = np.zeros((n + 1, 4))
            a[0] = (n, (tb.x[-1] - tb.x[0]) / (n - 1), tb.x[0], self.umax)
            a[1:, 0] = tb.x
            a[1:, 1] = tb.f
            a[1:, 2] = tb._y2
            t = torch.from_numpy(a.reshape(-1)).to(dev)
            self.__dict__[key] = t
        return t


class Lanczos(Interpolant):
    """Lanczos filter sinc(x) sinc(x / n) with the DC-conserving correction
    (interpolant.py:604-670, src/Interpolant.cpp:560-930).  On the GPU it serves as an
    InterpolatedImage's x interpolant (its transform from the reference's spline table,
    _LanczosTable) and, for n <= 3 (at most 7 taps per axis), as its k interpolant (the kernel
    itself, with the DC correction's coefficients K_1..K_5 from the same table object)."""
    _code = _lib.INTERP_LANCZOS

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
    def _table(self):
        return _LanczosTable.get(self._n, self._conserve_dc, self._gsparams)

    @property
    def urange(self):
        return self._table.umax

    @property
    def krange(self):
        return 2. * math.pi * self._table.umax

    def uval(self, u):
        return self._table.uval(u)

    def _args(self):
        return (self._n, self._conserve_dc)


def convert_interpolant(interpolant):
    """An Interpolant, or one made from its name (interpolant.py:672-685)."""
    if isinstance(interpolant, Interpolant):
        return interpolant
    return Interpolant.from_name(interpolant)


__all__ = ['Interpolant', 'Delta', 'Nearest', 'SincInterpolant', 'Linear', 'Cubic', 'Quintic',
           'Lanczos', 'convert_interpolant']

"""LookupTable: 1-d tabulated functions (galsim/table.py:33-420, src/Table.cpp).

Host-side FP64 arithmetic for the chromatic drawing path (SED and Bandpass tables, the
wavelength weights of the integrators).  Interpolants 'linear', 'spline' (natural cubic),
'floor', 'ceil' and 'nearest' for evaluation; integration (integrate, integrate_product) for
'linear' tables, the form every SED / Bandpass product and integrator weight table takes.
The argument lookup follows the reference's ArgVec (Table.cpp:64-130): tables whose
arguments are equally spaced to 1 % of a step use the direct index ceil((a - x0) / da),
others the first argument above a; both are clipped to the interior intervals.
"""
import numpy as np

from .errors import (GalSimValueError, GalSimRangeError, GalSimIncompatibleValuesError,
                     GalSimNotImplementedError)

__all__ = ['LookupTable', '_LookupTable', 'trapz']

_INTERPOLANTS = ('linear', 'spline', 'floor', 'ceil', 'nearest')


def _natural_spline_y2(x, f):
    """Second derivatives of the natural cubic spline through (x, f) (Table.cpp:634-686)."""
    n = len(x)
    y2 = np.zeros(n)
    if n == 3:
        y2[1] = 3. * ((f[2] - f[1]) / (x[2] - x[1]) - (f[1] - f[0]) / (x[1] - x[0])) / (x[2] - x[0])
    elif n > 3:
        c = np.zeros(n)
        for i in range(1, n - 1):
            y2[i] = 6. * ((f[i + 1] - f[i]) / (x[i + 1] - x[i]) - (f[i] - f[i - 1]) / (x[i] - x[i - 1]))
        bb = 2. * (x[2] - x[0])
        for i in range(1, n - 1):
            y2[i] /= bb
            if i == n - 2:
                break
            aa = x[i + 1] - x[i]
            cc = aa / bb
            c[i - 1] = cc
            bb = 2. * (x[i + 2] - x[i]) - aa * cc
            y2[i + 1] -= aa * y2[i]
        for i in range(n - 3, 0, -1):
            y2[i] -= c[i - 1] * y2[i + 1]
    return y2


class LookupTable(object):
    """f(x) tabulated at x, interpolated between the points (table.py:33-420)."""

    def __init__(self, x, f, interpolant='spline', x_log=False, f_log=False):
        if x_log or f_log:
            raise GalSimNotImplementedError("LookupTable with x_log or f_log is not built")
        if interpolant not in _INTERPOLANTS:
            raise GalSimNotImplementedError("LookupTable interpolant %r is not built" % (interpolant,))
        self.interpolant = interpolant
        self.x_log = self.f_log = False
        if len(x) != len(f):
            raise GalSimIncompatibleValuesError("Input array lengths don't match", x=x, f=f)
        if len(x) < 2:
            raise GalSimValueError("Input arrays too small to interpolate", x)
        x = np.asarray(x, dtype=float)
        f = np.asarray(f, dtype=float)
        if not np.all(x[1:] >= x[:-1]):
            s = np.argsort(x)
            x, f = x[s], f[s]
        self.x = np.ascontiguousarray(x)
        self.f = np.ascontiguousarray(f)
        if self.x[0] == self.x[-1]:
            raise GalSimValueError("All x values are equal", x)
        if self.x[-1] == np.inf:
            self.x[-1] = 1.e300
        self._setup()

    def _setup(self):
        x = self.x
        n = len(x)
        self._x_min = float(x[0])
        self._x_max = float(x[-1])
        self._da = (x[-1] - x[0]) / (n - 1)
        self._equal = bool(np.all(np.abs((x - x[0]) / self._da - np.arange(n)) <= 0.01))
        self._y2 = _natural_spline_y2(x, self.f) if self.interpolant == 'spline' else None

    x_min = property(lambda self: self._x_min)
    x_max = property(lambda self: self._x_max)

    def __len__(self):
        return len(self.x)

    def getArgs(self):
        return self.x

    def getVals(self):
        return self.f

    def _index(self, a):
        """ArgVec::upperIndex for each a (Table.cpp:78-130)."""
        x = self.x
        n = len(x)
        a = np.asarray(a, dtype=float)
        if self._equal:
            i = np.ceil((a - x[0]) / self._da)
            i = np.where(np.isfinite(i), i, 1).astype(np.int64)
        else:
            i = np.searchsorted(x, a, side='right')
        i = np.clip(i, 1, n - 1)
        return np.where(a < x[0], 1, np.where(a > x[-1], n - 1, i))

    def _interp(self, a, i):
        x, f = self.x, self.f
        a = np.asarray(a, dtype=float)
        if self.interpolant == 'linear':
            ax = (x[i] - a) / (x[i] - x[i - 1])
            bx = 1.0 - ax
            return f[i] * bx + f[i - 1] * ax
        if self.interpolant == 'spline':
            y2 = self._y2
            h = x[i] - x[i - 1]
            aa = (x[i] - a) / h
            bb = 1. - aa
            return (aa * f[i - 1] + bb * f[i] +
                    ((aa * aa * aa - aa) * y2[i - 1] + (bb * bb * bb - bb) * y2[i]) * (h * h) / 6.0)
        if self.interpolant == 'floor':
            j = np.where(a == x[i], i + 1, i)
            return f[np.minimum(j, len(x)) - 1]
        if self.interpolant == 'ceil':
            j = np.where(a == x[i - 1], i - 1, i)
            return f[j]
        return np.where((a - x[i - 1]) < (x[i] - a), f[i - 1], f[i])

    def _check_range(self, a):
        slop = (self._x_max - self._x_min) * 1.e-6
        a = np.asarray(a, dtype=float)
        if a.size and np.min(a) < self._x_min - slop:
            raise GalSimRangeError("x value(s) below the range of the LookupTable.",
                                   a[a < self._x_min], self._x_min, self._x_max)
        if a.size and np.max(a) > self._x_max + slop:
            raise GalSimRangeError("x value(s) above the range of the LookupTable.",
                                   a[a > self._x_max], self._x_min, self._x_max)

    def __call__(self, x):
        a = np.asarray(x, dtype=float)
        self._check_range(a)
        v = self._interp(a, self._index(a))
        return float(v) if np.ndim(v) == 0 else np.asarray(v)

    # -- integration (linear tables; Table.cpp:280-421, TLinear :532-550) --------------------
    def _need_linear(self, what):
        if self.interpolant != 'linear':
            raise GalSimNotImplementedError("%s of a LookupTable with interpolant=%r is not built"
                                            % (what, self.interpolant))

    def _integrate(self, xmin, xmax):
        x, f = self.x, self.f
        n = len(x)
        i = int(self._index(xmin))
        x1 = xmin
        x2, f2 = x[i], f[i]
        if x2 > xmax:
            x2 = xmax
            f1 = float(self._interp(x1, i))
            f2 = float(self._interp(x2, i))
            return 0.5 * (f1 + f2) * (x2 - x1)
        ans = 0.
        if x2 > x1:
            f1 = float(self._interp(x1, i))
            ans += 0.5 * (f1 + f2) * (x2 - x1)
        x1, f1 = x2, f2
        i += 1
        x2 = x[i] if i < n else np.inf
        f2 = f[i] if i < n else 0.
        while x2 <= xmax and i < n:
            ans += 0.5 * (f1 + f2) * (x2 - x1)
            x1, f1 = x2, f2
            i += 1
            x2 = x[i] if i < n else np.inf
            f2 = f[i] if i < n else 0.
        if x1 < xmax:
            x2 = xmax
            f2 = float(self._interp(xmax, min(i, n - 1)))
            ans += 0.5 * (f1 + f2) * (x2 - x1)
        return ans

    def integrate(self, x_min=None, x_max=None):
        """Integral of the tabulated function over [x_min, x_max], zero outside the table
        (table.py:256-313, Table.cpp:280-341)."""
        self._need_linear('integrate')
        x_min = self._x_min if x_min is None else max(x_min, self._x_min)
        x_max = self._x_max if x_max is None else min(x_max, self._x_max)
        if x_min < x_max:
            return self._integrate(float(x_min), float(x_max))
        elif x_min == x_max:
            return 0.
        return -self.integrate(x_max, x_min)

    def integrate_product(self, g, x_min=None, x_max=None, x_factor=1.):
        """Integral of f(x x_factor) g(x) over [x_min, x_max] with g linear between the
        abscissae of both (table.py:315-383, Table.cpp:344-405)."""
        self._need_linear('integrate_product')
        if x_min is None:
            x_min = self._x_min / x_factor
        else:
            x_min = max(x_min, self._x_min / x_factor)
        if x_max is None:
            x_max = self._x_max / x_factor
        else:
            x_max = min(x_max, self._x_max / x_factor)
        if x_min > x_max:
            return -self.integrate_product(g, x_max, x_min, x_factor)
        elif x_min == x_max:
            return 0.
        if isinstance(g, LookupTable):
            x_min = max(x_min, g.x_min)
            x_max = min(x_max, g.x_max)
            if x_min >= x_max:
                return 0.
        else:
            gx = self.x / x_factor
            gx = gx[(gx >= x_min) & (gx <= x_max)]
            gx = np.unique(np.concatenate([gx, [x_min, x_max]]))
            gf = g(gx)
            if np.ndim(gf) == 0:
                gf = np.full(gx.shape, float(gf))
            g = _LookupTable(gx, gf, 'linear')
        return self._integrate_product(g, float(x_min), float(x_max), float(x_factor))

    def _integrate_product(self, g, xmin, xmax, xfact):
        xs, gs = self.x, g.x

        def fi(a, i):
            return float(self._interp(a, i))

        def gi(a, j):
            return float(g._interp(a, j))

        x1 = xmin
        xx1 = x1 * xfact
        i = int(self._index(xx1))
        j = int(g._index(x1))
        f1 = fi(xx1, i)
        g1 = gi(x1, j)
        x2 = gs[j]
        xx2 = x2 * xfact
        if xs[i] < xx2:
            xx2 = xs[i]
            x2 = xx2 / xfact
        f2 = fi(xx2, i)
        g2 = gi(x2, j)
        ans = 0.
        while x2 < xmax:
            ans += (1. / 6.) * (x2 - x1) * (f1 * (2. * g1 + g2) + f2 * (g1 + 2. * g2))
            x1, f1, g1 = x2, f2, g2
            if xx2 == xs[i]:
                i += 1
            if x2 == gs[j]:
                j += 1
            x2 = gs[j]
            xx2 = x2 * xfact
            if xs[i] < xx2:
                xx2 = xs[i]
                x2 = xx2 / xfact
            f2 = fi(xx2, i)
            g2 = gi(x2, j)
        x2 = xmax
        xx2 = x2 * xfact
        f2 = fi(xx2, i)
        g2 = gi(x2, j)
        ans += (1. / 6.) * (x2 - x1) * (f1 * (2. * g1 + g2) + f2 * (g1 + 2. * g2))
        return ans

    def __eq__(self, other):
        return self is other or (isinstance(other, LookupTable) and
                                 np.array_equal(self.x, other.x) and np.array_equal(self.f, other.f) and
                                 self.interpolant == other.interpolant)

    def __hash__(self):
        return hash(("galsim.LookupTable", tuple(self.x), tuple(self.f), self.interpolant))

    def __repr__(self):
        return 'galsim.LookupTable(x=array(%r), f=array(%r), interpolant=%r)' % (
            self.x.tolist(), self.f.tolist(), self.interpolant)


def _LookupTable(x, f, interpolant='spline', x_log=False, f_log=False):
    """A LookupTable from already sorted arguments, without the input checks (table.py:524-560)."""
    if x_log or f_log:
        raise GalSimNotImplementedError("LookupTable with x_log or f_log is not built")
    ret = LookupTable.__new__(LookupTable)
    ret.interpolant = interpolant
    ret.x_log = ret.f_log = False
    ret.x = np.ascontiguousarray(x, dtype=float)
    ret.f = np.ascontiguousarray(f, dtype=float)
    ret._setup()
    return ret


def trapz(f, x, interpolant='linear'):
    """Integral of f(x) tabulated at x by the trapezoidal rule (table.py:1389-1415)."""
    if len(x) >= 2:
        return _LookupTable(x, f, interpolant=interpolant).integrate()
    return 0.

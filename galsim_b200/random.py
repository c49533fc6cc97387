"""Random deviates: Uniform, Gaussian, Poisson, Weibull, Gamma, Chi-square and Binomial
(galsim/random.py:309-696, src/Random.cpp).

Each deviate is a BaseDeviate stream (seed + raw 32-bit draws taken) with the distribution of
the reference on top.  Uniform, Gaussian and Poisson deviates are drawn on the GPU by the
noise kernels (galsim_b200/csrc/gsb_noise.cu, `gsb_add_noise` applied to a zero FP64 buffer):
uniform_01 as one word / 2^32, the Box-Muller pairs of boost 1.48's normal_distribution, and
its poisson_distribution (inversion below mean 10, PTRD above).  The Weibull, Gamma,
Chi-square and Binomial deviates run boost 1.48's algorithms on the host over the stream's
words, which are read from the GPU in blocks and consumed in order.  What the reference keeps
inside a deviate object between calls is kept here on the host: a GaussianDeviate's second
Box-Muller value (the pair cache, used by the next call, cleared by generate and clearCache),
and a PoissonDeviate's normal branch (means above 2^30 or 0) with its own pair cache.  Single
GPU draws are one small launch each; generate() fills an array in one launch.
"""
import math

import numpy as np

from . import _lib
from .errors import GalSimRangeError, GalSimValueError
from .noise import BaseDeviate, NoiseParamsC, _apply, GAUSSIAN, POISSON, UNIFORM

__all__ = ['UniformDeviate', 'GaussianDeviate', 'PoissonDeviate', 'WeibullDeviate', 'GammaDeviate',
           'Chi2Deviate', 'BinomialDeviate', 'DistDeviate']

_MAX_POISSON = float(1 << 30)


def _draw(stream, kind, n, params=None, values=None):
    """n deviates of `kind` from `stream` (advanced past them) as a host FP64 array: the noise
    kernel applied to a zero buffer (or to `values`, the per-element expectations of Poisson
    draws)."""
    import torch
    if n == 0:
        return np.zeros(0)
    dev = _lib.Device.torch_device()
    if values is None:
        flat = torch.zeros(n, dtype=torch.float64, device=dev)
    else:
        flat = torch.from_numpy(np.ascontiguousarray(values, dtype=np.float64).reshape(-1)).to(dev)
    used = _apply(kind, params if params is not None else NoiseParamsC(), flat, [0], [n],
                  [stream.seed], [stream.used])
    stream.used = int(used[0])
    return flat.cpu().numpy()


def _fill(array, vals, add=False):
    """Write (or add) vals into a numpy array of any shape, as the reference's generate /
    add_generate do (through an FP64 copy, cast back with casting='unsafe')."""
    vals = np.asarray(vals).reshape(array.shape)
    if add:
        vals = np.asarray(array, dtype=float) + vals
    np.copyto(array, vals, casting='unsafe')


class UniformDeviate(BaseDeviate):
    """Uniform deviates in [0, 1) (random.py:309-343): one raw word each, divided by 2^32."""

    def __init__(self, seed=None):
        BaseDeviate.__init__(self, seed)

    def __call__(self):
        return float(_draw(self._stream, UNIFORM, 1)[0])

    def raw(self):
        """The next raw 32-bit word of the stream."""
        return int(_draw(self._stream, UNIFORM, 1)[0] * 4294967296.)

    def clearCache(self):
        pass

    def generate(self, array):
        _fill(array, _draw(self._stream, UNIFORM, int(np.size(array))))

    def add_generate(self, array):
        _fill(array, _draw(self._stream, UNIFORM, int(np.size(array))), add=True)

    def duplicate(self):
        ret = UniformDeviate.__new__(UniformDeviate)
        ret._stream = BaseDeviate.duplicate(self)._stream
        return ret

    def __repr__(self):
        return 'galsim.UniformDeviate(seed=%r)' % self._stream.seed


class GaussianDeviate(BaseDeviate):
    """Gaussian deviates of a mean and sigma (random.py:345-413): Box-Muller pairs, the cosine
    value first; the sine value of the last pair is kept for the next call (boost 1.48
    normal_distribution), and each value is (unit deviate * sigma) + mean."""

    def __init__(self, seed=None, mean=0., sigma=1.):
        if sigma < 0.:
            raise GalSimRangeError("GaussianDeviate sigma must be > 0.", sigma, 0.)
        BaseDeviate.__init__(self, seed)
        self._mean = float(mean)
        self._sigma = float(sigma)
        self._cache = None

    mean = property(lambda self: self._mean)
    sigma = property(lambda self: self._sigma)
    generates_in_pairs = property(lambda self: True)

    def clearCache(self):
        self._cache = None

    def reset(self, seed=None):
        BaseDeviate.reset(self, seed)
        self._cache = None

    def _units(self, n):
        """n unit deviates continuing the pair sequence (the cache first); an odd tail leaves
        its pair's second value in the cache."""
        out = []
        if n and self._cache is not None:
            out.append(self._cache)
            self._cache = None
            n -= 1
        if n:
            m = n + (n & 1)
            p = NoiseParamsC()
            p.sigma = 1.
            z = _draw(self._stream, GAUSSIAN, m, p)
            out.extend(z[:n])
            if m > n:
                self._cache = float(z[n])
        return np.array(out, dtype=float)

    def __call__(self):
        return float(self._units(1)[0] * self._sigma + self._mean)

    def generate(self, array):
        self._cache = None
        _fill(array, self._units(int(np.size(array))) * self._sigma + self._mean)

    def add_generate(self, array):
        self._cache = None
        _fill(array, self._units(int(np.size(array))) * self._sigma + self._mean, add=True)

    def generate_from_variance(self, array):
        """Unit deviates times sqrt(array) (GaussianDeviate::generateFromVariance,
        Random.cpp:402-450); the pair cache is cleared before and after."""
        self._cache = None
        var = np.asarray(array, dtype=float).reshape(-1)
        z = self._units(var.size)
        self._cache = None
        _fill(array, z * np.sqrt(var))

    def duplicate(self):
        ret = GaussianDeviate.__new__(GaussianDeviate)
        ret._stream = BaseDeviate.duplicate(self)._stream
        ret._mean, ret._sigma, ret._cache = self._mean, self._sigma, self._cache
        return ret

    def __repr__(self):
        return 'galsim.GaussianDeviate(seed=%r, mean=%r, sigma=%r)' % (
            self._stream.seed, self._mean, self._sigma)


class PoissonDeviate(BaseDeviate):
    """Poisson deviates of a mean (random.py:468-531, PoissonDeviateImpl in Random.cpp:499-606):
    boost 1.48's poisson_distribution for 0 < mean <= 2^30; for mean 0 and above 2^30 the
    normal approximation N(mean, sqrt(mean)) with its own pair cache (kept while the deviate
    stays on that branch)."""

    def __init__(self, seed=None, mean=1.):
        if mean < 0:
            raise GalSimValueError("PoissonDeviate is only defined for mean >= 0.", mean)
        BaseDeviate.__init__(self, seed)
        self._mean = float(mean)
        self._cache = None

    mean = property(lambda self: self._mean)
    has_reliable_discard = property(lambda self: False)

    def _normal_branch(self):
        return self._mean > _MAX_POISSON or self._mean == 0.

    def clearCache(self):
        self._cache = None

    def reset(self, seed=None):
        BaseDeviate.reset(self, seed)
        self._cache = None

    def _values(self, n):
        if not self._normal_branch():
            p = NoiseParamsC()
            return _draw(self._stream, POISSON, n, p, values=np.full(n, self._mean))
        # the normal branch: Gaussian pairs with the deviate's cache
        out = []
        if n and self._cache is not None:
            out.append(self._cache)
            self._cache = None
            n -= 1
        if n:
            m = n + (n & 1)
            p = NoiseParamsC()
            p.sigma = 1.
            z = _draw(self._stream, GAUSSIAN, m, p)
            out.extend(z[:n])
            if m > n:
                self._cache = float(z[n])
        return np.array(out, dtype=float) * np.sqrt(self._mean) + self._mean

    def __call__(self):
        return float(self._values(1)[0])

    def generate(self, array):
        self._cache = None
        _fill(array, self._values(int(np.size(array))))

    def add_generate(self, array):
        self._cache = None
        _fill(array, self._values(int(np.size(array))), add=True)

    def generate_from_expectation(self, array):
        """Each element replaced by a draw with that element as the mean (elements equal to 0
        stay 0 and take no draws; PoissonDeviate::generateFromExpectation, Random.cpp:594-606),
        in one launch of the Poisson kernel; the normal branch's pair cache starts empty."""
        a = np.asarray(array, dtype=float)
        if np.any(a < 0):
            raise GalSimValueError("Expectation array may not have values < 0.", array)
        self._cache = None
        _fill(array, _draw(self._stream, POISSON, int(a.size), NoiseParamsC(), values=a.reshape(-1)))

    def duplicate(self):
        ret = PoissonDeviate.__new__(PoissonDeviate)
        ret._stream = BaseDeviate.duplicate(self)._stream
        ret._mean, ret._cache = self._mean, self._cache
        return ret

    def __repr__(self):
        return 'galsim.PoissonDeviate(seed=%r, mean=%r)' % (self._stream.seed, self._mean)


class _Words(object):
    """Sequential access to a stream's raw 32-bit words for the deviates drawn on the host (a
    data-dependent number of words each): the words come from the GPU in blocks (the uniform
    kind, word / 2^32), are consumed in order, and commit() moves the stream past the words
    used."""

    def __init__(self, stream, block=1024):
        self.stream = stream
        self.start = stream.used
        self.block = block
        self.buf = np.zeros(0)
        self.pos = 0

    def uniform01(self):
        if self.pos == len(self.buf):
            probe = type(self.stream).__new__(type(self.stream))
            probe.seed, probe.used = self.stream.seed, self.start + self.pos
            nxt = _draw(probe, UNIFORM, self.block)
            self.buf = np.concatenate([self.buf, nxt])
        u = float(self.buf[self.pos])
        self.pos += 1
        return u

    def commit(self):
        self.stream.used = self.start + self.pos


def _host_generate(dev, array, add=False):
    w = _Words(dev._stream, block=max(64, min(1 << 16, 2 * int(np.size(array)))))
    vals = np.array([dev._sample(w) for _ in range(int(np.size(array)))], dtype=float)
    w.commit()
    _fill(array, vals, add=add)


class WeibullDeviate(BaseDeviate):
    """Weibull deviates of shape a and scale b (random.py:534-588): b (-ln(1 - u))^(1/a), one
    uniform each (boost 1.48 weibull_distribution), in the host's FP64 math."""

    def __init__(self, seed=None, a=1., b=1.):
        BaseDeviate.__init__(self, seed)
        self._a, self._b = float(a), float(b)

    a = property(lambda self: self._a)
    b = property(lambda self: self._b)

    def _sample(self, w):
        return self._b * math.pow(-math.log(1. - w.uniform01()), 1. / self._a)

    def __call__(self):
        w = _Words(self._stream, block=64)
        v = self._sample(w)
        w.commit()
        return v

    def generate(self, array):
        _host_generate(self, array)

    def add_generate(self, array):
        _host_generate(self, array, add=True)

    def clearCache(self):
        pass

    def __repr__(self):
        return 'galsim.WeibullDeviate(seed=%r, a=%r, b=%r)' % (self._stream.seed, self._a, self._b)


def _gamma_sample(w, alpha, beta):
    """boost 1.48 gamma_distribution (alpha, beta): an exponential for alpha = 1, the tangent
    rejection method for alpha > 1, and the exponential-mixture rejection for alpha < 1, each
    uniform from the stream in order."""
    if alpha == 1.:
        return -math.log(1. - w.uniform01()) * beta
    if alpha > 1.:
        s = math.sqrt(2. * alpha - 1.)
        while True:
            y = math.tan(math.pi * w.uniform01())
            x = s * y + alpha - 1.
            if x <= 0.:
                continue
            if w.uniform01() > (1. + y * y) * math.exp((alpha - 1.) * math.log(x / (alpha - 1.)) - s * y):
                continue
            return x * beta
    p = math.exp(1.) / (alpha + math.exp(1.))
    while True:
        u = w.uniform01()
        y = -math.log(1. - w.uniform01())
        if u < p:
            x = math.exp(-y / alpha)
            q = p * math.exp(-x)
        else:
            x = 1. + y
            q = p + (1. - p) * math.pow(x, alpha - 1.)
        if u >= q:
            continue
        return x * beta


class GammaDeviate(BaseDeviate):
    """Gamma deviates of shape k and scale theta (random.py:590-645, boost 1.48
    gamma_distribution; a data-dependent number of uniforms each)."""

    def __init__(self, seed=None, k=1., theta=1.):
        BaseDeviate.__init__(self, seed)
        self._k, self._theta = float(k), float(theta)

    k = property(lambda self: self._k)
    theta = property(lambda self: self._theta)
    has_reliable_discard = property(lambda self: False)

    def _sample(self, w):
        return _gamma_sample(w, self._k, self._theta)

    __call__ = WeibullDeviate.__call__
    generate = WeibullDeviate.generate
    add_generate = WeibullDeviate.add_generate
    clearCache = WeibullDeviate.clearCache

    def __repr__(self):
        return 'galsim.GammaDeviate(seed=%r, k=%r, theta=%r)' % (self._stream.seed, self._k, self._theta)


class Chi2Deviate(BaseDeviate):
    """Chi-square deviates with n degrees of freedom (random.py:647-696): 2 Gamma(n / 2, 1)
    (boost 1.48 chi_squared_distribution)."""

    def __init__(self, seed=None, n=1.):
        BaseDeviate.__init__(self, seed)
        self._n = float(n)

    n = property(lambda self: self._n)
    has_reliable_discard = property(lambda self: False)

    def _sample(self, w):
        return 2. * _gamma_sample(w, self._n / 2., 1.)

    __call__ = WeibullDeviate.__call__
    generate = WeibullDeviate.generate
    add_generate = WeibullDeviate.add_generate
    clearCache = WeibullDeviate.clearCache

    def __repr__(self):
        return 'galsim.Chi2Deviate(seed=%r, n=%r)' % (self._stream.seed, self._n)


def _stirling_fc(k):
    """The correction of Stirling's formula, ln k! = (k + 1/2) ln(k + 1) - (k + 1) + ln sqrt(2 pi)
    + fc(k): from ln Gamma below 10, its series 1/12 - (1/360 - (1/1260) z^2) z^2) z with
    z = 1 / (k + 1) above (the form boost 1.48's binomial_distribution uses)."""
    if k < 10:
        return math.lgamma(k + 1.) - ((k + 0.5) * math.log(k + 1.) - (k + 1.) + 0.5 * math.log(2. * math.pi))
    z = 1. / (k + 1)
    return (1. / 12 - (1. / 360 - (1. / 1260) * (z * z)) * (z * z)) * z


class BinomialDeviate(BaseDeviate):
    """Binomial deviates of N trials with probability p (random.py:415-466): boost 1.48's
    binomial_distribution -- inversion while (N + 1) min(p, 1 - p) < 11, else the BTRD
    transformed rejection of Hoermann (1993) -- on the host over the stream's words."""

    def __init__(self, seed=None, N=1, p=0.5):
        BaseDeviate.__init__(self, seed)
        self._N, self._p = int(N), float(p)
        pp = 1. - self._p if 0.5 < self._p else self._p
        t = self._N
        self._m = int((t + 1) * pp)
        if self._m < 11:
            self._q_n = math.pow(1. - pp, float(t))
        else:
            r = pp / (1. - pp)
            npq = t * pp * (1. - pp)
            b = 1.15 + 2.53 * math.sqrt(npq)
            self._btrd = dict(r=r, nr=(t + 1) * r, npq=npq, b=b, a=-0.0873 + 0.0248 * b + 0.01 * pp,
                              c=t * pp + 0.5, alpha=(2.83 + 5.1 / b) * math.sqrt(npq), v_r=0.92 - 4.2 / b)
            self._btrd['u_rv_r'] = 0.86 * self._btrd['v_r']

    n = property(lambda self: self._N)
    p = property(lambda self: self._p)
    has_reliable_discard = property(lambda self: False)

    def _invert(self, w, t, p):
        q = 1. - p
        s = p / q
        a = (t + 1) * s
        r = self._q_n
        u = w.uniform01()
        x = 0
        while u > r:
            u = u - r
            x += 1
            r = ((a / x) - s) * r
        return x

    def _btrd_draw(self, w):
        B = self._btrd
        t, m = self._N, self._m
        while True:
            v = w.uniform01()
            if v <= B['u_rv_r']:
                u = v / B['v_r'] - 0.43
                return int(math.floor((2 * B['a'] / (0.5 - abs(u)) + B['b']) * u + B['c']))
            if v >= B['v_r']:
                u = w.uniform01() - 0.5
            else:
                u = v / B['v_r'] - 0.93
                u = (-0.5 if u < 0 else 0.5) - u
                v = w.uniform01() * B['v_r']
            us = 0.5 - abs(u)
            k = int(math.floor((2 * B['a'] / us + B['b']) * u + B['c']))
            if k < 0 or k > t:
                continue
            v = v * B['alpha'] / (B['a'] / (us * us) + B['b'])
            km = float(abs(k - m))
            if km <= 15:
                f = 1.
                if m < k:
                    i = m
                    while True:
                        i += 1
                        f = f * (B['nr'] / i - B['r'])
                        if i == k:
                            break
                elif m > k:
                    i = k
                    while True:
                        i += 1
                        v = v * (B['nr'] / i - B['r'])
                        if i == m:
                            break
                if v <= f:
                    return k
                continue
            v = math.log(v)
            rho = (km / B['npq']) * (((km / 3. + 0.625) * km + 1. / 6) / B['npq'] + 0.5)
            tt = -km * km / (2 * B['npq'])
            if v < tt - rho:
                return k
            if v > tt + rho:
                continue
            nm = t - m + 1
            h = (m + 0.5) * math.log((m + 1) / (B['r'] * nm)) + _stirling_fc(m) + _stirling_fc(t - m)
            nk = t - k + 1
            if v <= (h + (t + 1) * math.log(float(nm) / nk) + (k + 0.5) * math.log(nk * B['r'] / (k + 1))
                     - _stirling_fc(k) - _stirling_fc(t - k)):
                return k

    def _sample(self, w):
        t = self._N
        if self._m < 11:
            if 0.5 < self._p:
                return float(t - self._invert(w, t, 1. - self._p))
            return float(self._invert(w, t, self._p))
        if 0.5 < self._p:
            return float(t - self._btrd_draw(w))
        return float(self._btrd_draw(w))

    __call__ = WeibullDeviate.__call__
    generate = WeibullDeviate.generate
    add_generate = WeibullDeviate.add_generate
    clearCache = WeibullDeviate.clearCache

    def __repr__(self):
        return 'galsim.BinomialDeviate(seed=%r, N=%r, p=%r)' % (self._stream.seed, self._N, self._p)


class DistDeviate(BaseDeviate):
    """Deviates drawn from a tabulated probability density (random.py:698-930): the density's
    LookupTable gives a CDF by the trapezoid rule on its abscissae, inverted by a linear
    LookupTable of (CDF, x); each draw is one uniform from the stream (on the GPU) mapped through
    it.  Densities given as Python callables, expressions or files need the reference's adaptive
    Gauss-Kronrod integrator over npoints intervals and are not built."""

    def __init__(self, seed=None, function=None, x_min=None, x_max=None, interpolant=None, npoints=None,
                 clip_neg=False):
        from .table import LookupTable
        from .errors import GalSimIncompatibleValuesError, GalSimNotImplementedError
        BaseDeviate.__init__(self, seed)
        if function is None:
            raise TypeError('You must pass a function to DistDeviate!')
        if isinstance(function, str) or not isinstance(function, LookupTable) or npoints is not None:
            if not isinstance(function, str) and not hasattr(function, '__call__'):
                raise TypeError('function must be a callable function or a string')
            raise GalSimNotImplementedError("DistDeviate from a callable, an expression or a file (the "
                                            "adaptive integration of the density) is not built")
        if interpolant:
            raise GalSimIncompatibleValuesError(
                "Cannot provide an interpolant with a callable function argument",
                interpolant=interpolant, function=function)
        if (x_min not in (None, function.x_min)) or (x_max not in (None, function.x_max)):
            raise GalSimIncompatibleValuesError(
                "Cannot provide x_min or x_max with a LookupTable function",
                function=function, x_min=x_min, x_max=x_max)
        xarray = np.array(function.x, dtype=float)
        pdf = np.array(function.f, dtype=float)
        pdf[1:] = pdf[1:] + pdf[:-1]
        pdf[1:] *= np.diff(xarray)
        pdf[0] = 0.
        if clip_neg:
            pdf[~(pdf >= 0)] = 0.
        elif not np.all(pdf >= 0.):
            raise GalSimValueError('Negative probability found in DistDeviate.', function)
        cdf = np.cumsum(pdf)
        cdf /= cdf[-1]
        self._function = function
        self._inverse_cdf = LookupTable(cdf, xarray, interpolant='linear')
        self.x_min = function.x_min
        self.x_max = function.x_max

    def val(self, p):
        if p < 0 or p > 1:
            raise GalSimRangeError('Invalid cumulative probability for DistDeviate', p, 0., 1.)
        return self._inverse_cdf(p)

    def __call__(self):
        return self._inverse_cdf(float(_draw(self._stream, UNIFORM, 1)[0]))

    def generate(self, array):
        p = _draw(self._stream, UNIFORM, int(np.size(array)))
        np.copyto(array, np.asarray(self._inverse_cdf(p)).reshape(np.shape(array)))

    def clearCache(self):
        pass

    def __repr__(self):
        return 'galsim.DistDeviate(seed=%r, function=%r)' % (self._stream.seed, self._function)

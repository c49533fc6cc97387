"""Random streams and noise: BaseDeviate, GaussianNoise, PoissonNoise, CCDNoise,
VariableGaussianNoise
(galsim/random.py, galsim/noise.py).

A BaseDeviate is the reference's random stream, named by its seed and the number of raw
32-bit draws already taken from it; the draws themselves happen on the GPU
(galsim_b200/csrc/gsb_noise.cu, `gsb_add_noise`), where the Mersenne Twister, its seeding and the
Boost.Random 1.48 deviates the reference uses are restated, so a stamp gets the same noise as
`image.addNoise(noise)` in the reference for the same seed.  Noise is applied to host Images
(copied through the device) and, without leaving the device, to every stamp of a StampBatch
with a seed per stamp (`StampBatch.addNoise`), as the reference's config layer seeds each
object.
"""
import ctypes
import math
import os

import numpy as np

from . import _lib
from .errors import GalSimError, GalSimNotImplementedError, GalSimRangeError, GalSimValueError


class _Stream(object):
    def __init__(self, seed):
        self.seed = int(seed)
        self.used = 0


def _random_seed():
    while True:
        s = int.from_bytes(os.urandom(4), 'little')
        if s:
            return s


class BaseDeviate(object):
    """The reference's random-number stream (random.py BaseDeviate).  BaseDeviate(seed) with a
    nonzero int is reproducible; None or 0 draws a seed from the operating system; another
    BaseDeviate shares that stream (as the reference does)."""

    def __init__(self, seed=None):
        if isinstance(seed, BaseDeviate):
            self._stream = seed._stream
        elif seed is None or (not isinstance(seed, str) and int(seed) == 0):
            self._stream = _Stream(_random_seed())
        elif isinstance(seed, str):
            raise GalSimNotImplementedError("BaseDeviate from a serialized state is not built")
        else:
            if int(seed) != seed:
                raise TypeError("BaseDeviate must be initialized with an int or another BaseDeviate")
            self._stream = _Stream(int(seed))

    def seed(self, seed=0):
        """Reseed this stream (seen by every object sharing it)."""
        self._stream.seed = int(seed) if seed else _random_seed()
        self._stream.used = 0

    def reset(self, seed=None):
        """Start an independent stream from seed."""
        self._stream = BaseDeviate(seed)._stream

    def duplicate(self):
        """An independent copy at the same position."""
        ret = BaseDeviate.__new__(BaseDeviate)
        ret._stream = _Stream(self._stream.seed)
        ret._stream.used = self._stream.used
        return ret

    def discard(self, n):
        """Skip n raw draws."""
        self._stream.used += int(n)

    def __eq__(self, other):
        return (isinstance(other, BaseDeviate) and self._stream.seed == other._stream.seed and
                self._stream.used == other._stream.used)

    def __ne__(self, other):
        return not self.__eq__(other)

    __hash__ = None

    def __repr__(self):
        return 'galsim.BaseDeviate(%r)' % self._stream.seed


class NoiseParamsC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ('sigma', 'sky_level', 'gain', 'read_noise',
                                               'frac_sky', 'int_sky')] + \
               [('int_sky_same_dtype', ctypes.c_int32), ('pad', ctypes.c_int32)]


NOISE_STAMP_DTYPE = np.dtype({'names': ['offset', 'npix', 'pad', 'seed', 'skip'],
                              'formats': ['i8', 'i4', 'i4', 'i8', 'i8'],
                              'offsets': [0, 8, 12, 16, 24], 'itemsize': 32})

GAUSSIAN, POISSON, CCD, VARIABLE_GAUSSIAN, UNIFORM = 0, 1, 2, 3, 4


def _sky_split(sky_level, dtype):
    """frac_sky / int_sky of PoissonNoise / CCDNoise._applyTo with numpy's scalar rules
    (noise.py:337-339): for float images frac_sky is 0 and int_sky is sky_level in the image
    type."""
    frac_sky = sky_level - np.dtype(dtype).type(sky_level)
    int_sky = sky_level - frac_sky
    same = np.dtype(type(int_sky)) == np.dtype(dtype)
    return float(frac_sky), float(int_sky), bool(same)


def _torch_codes():
    import torch
    return {torch.float32: _lib.F32, torch.float64: _lib.F64, torch.int16: _lib.I16,
            torch.int32: _lib.I32, torch.uint16: _lib.U16, torch.uint32: _lib.U32}


class _Codes(dict):
    def get(self, k, default=None):
        if not self:
            self.update(_torch_codes())
        return dict.get(self, k, default)


_TORCH_CODES = _Codes()
_IMAGE_TYPES = (np.float32, np.float64, np.int16, np.int32, np.uint16, np.uint32)


def _apply(kind, params, flat, offsets, npix, seeds, skips, scratch=None):
    """Run gsb_add_noise on a device tensor `flat` (float32 / float64) with per-stamp records;
    returns the per-stamp draw counts after the call.  `scratch` (FP64, laid out like `flat`)
    carries the per-pixel variances of variable Gaussian noise."""
    import torch
    dev = _lib.Device.torch_device()
    B = len(offsets)
    # the largest stamps first: each stamp's Poisson stream is one sequential chain, so the
    # longest chains should start before all warps are busy
    order = np.argsort(-np.asarray(npix, np.int64), kind='stable')
    rec = np.zeros(B, dtype=NOISE_STAMP_DTYPE)
    rec['offset'] = np.asarray(offsets, np.int64)[order]
    rec['npix'] = np.asarray(npix)[order]
    rec['seed'] = np.broadcast_to(np.asarray(seeds, np.int64), (B,))[order]
    rec['skip'] = np.broadcast_to(np.asarray(skips, np.int64), (B,))[order]
    d_rec = _lib.to_device(rec)
    dt = _TORCH_CODES.get(flat.dtype)
    if dt is None:
        raise GalSimNotImplementedError("noise is applied to float32 / float64 / int16 / int32 / "
                                        "uint16 / uint32 images")
    if scratch is None:
        scratch = torch.empty(flat.numel() if kind in (POISSON, CCD) else 1, dtype=torch.float64, device=dev)
    used = torch.empty(B, dtype=torch.int64, device=dev)
    _lib.check(_lib.lib().gsb_add_noise(kind, ctypes.byref(params), _lib.ptr(d_rec), B,
                                        int(np.max(npix)) if B else 0, _lib.ptr(flat), dt,
                                        _lib.ptr(scratch), _lib.ptr(used), _lib.Device.stream()))
    out = np.empty(B, np.int64)
    out[order] = used.cpu().numpy()
    return out


class BaseNoise(object):
    """noise.py BaseNoise: a noise model with its random stream."""

    def __init__(self, rng=None):
        if rng is None:
            self._rng = BaseDeviate()
        elif isinstance(rng, BaseDeviate):
            self._rng = rng
        else:
            raise TypeError("rng must be a galsim.BaseDeviate")

    @property
    def rng(self):
        return self._rng

    def getVariance(self):
        return self._getVariance()

    def withVariance(self, variance):
        if variance < 0.:
            raise GalSimRangeError("variance must be >= 0", variance, 0.)
        return self._withVariance(variance)

    def withScaledVariance(self, variance_ratio):
        if variance_ratio < 0.:
            raise GalSimRangeError("variance_ratio must be >= 0", variance_ratio, 0.)
        return self._withScaledVariance(variance_ratio)

    def __mul__(self, variance_ratio):
        return self.withScaledVariance(variance_ratio)

    __rmul__ = __mul__

    def __div__(self, variance_ratio):
        return self.withScaledVariance(1. / variance_ratio)

    __truediv__ = __div__

    def __eq__(self, other):
        return self is other or repr(self) == repr(other)

    def __ne__(self, other):
        return not self.__eq__(other)

    __hash__ = None

    def applyTo(self, image):
        """Add this noise to an Image (on the GPU; the stream advances as in the reference)."""
        from .image import Image
        if not isinstance(image, Image):
            raise TypeError("Provided image must be a galsim.Image")
        self._applyTo(image)

    def _applyTo(self, image):
        import torch
        arr = image.array
        if arr.dtype not in _IMAGE_TYPES:
            raise GalSimNotImplementedError("noise is applied to float32 / float64 / int16 / int32 / "
                                            "uint16 / uint32 images")
        kind, params = self._params(arr.dtype)
        host = np.ascontiguousarray(arr)
        flat = torch.from_numpy(host.reshape(-1).copy()).to(_lib.Device.torch_device())
        st = self._rng._stream
        used = _apply(kind, params, flat, [0], [host.size], [st.seed], [st.used])
        arr[...] = flat.cpu().numpy().reshape(arr.shape)
        st.used = int(used[0])

    def _apply_batch(self, sb, seeds, skips=None):
        B = len(sb.offsets)
        seeds = np.broadcast_to(np.asarray(seeds, dtype=np.int64), (B,))
        if np.any(seeds == 0):
            raise GalSimValueError("stamp seeds must be nonzero", seeds)
        skips = np.zeros(B, np.int64) if skips is None else np.broadcast_to(np.asarray(skips, np.int64), (B,))
        kind, params = self._params(np.float32 if sb.dtype == np.float32 else np.float64)
        npix = (np.asarray(sb.nx) * np.asarray(sb.ny)).astype(np.int32)
        return _apply(kind, params, sb.flat, np.asarray(sb.offsets, np.int64), npix, seeds, skips)


class GaussianNoise(BaseNoise):
    """Gaussian noise of standard deviation sigma (noise.py:227-291)."""

    def __init__(self, rng=None, sigma=1.):
        BaseNoise.__init__(self, rng)
        self._sigma = sigma

    sigma = property(lambda self: self._sigma)

    def _params(self, dtype):
        p = NoiseParamsC()
        p.sigma = float(self._sigma)
        return GAUSSIAN, p

    def _getVariance(self):
        return self.sigma ** 2

    def _withVariance(self, variance):
        return GaussianNoise(self.rng, math.sqrt(variance))

    def _withScaledVariance(self, variance_ratio):
        return GaussianNoise(self.rng, self.sigma * math.sqrt(variance_ratio))

    def copy(self, rng=None):
        return GaussianNoise(self.rng if rng is None else rng, self.sigma)

    def __repr__(self):
        return 'galsim.GaussianNoise(rng=%r, sigma=%r)' % (self.rng, self.sigma)


class PoissonNoise(BaseNoise):
    """Poisson noise of the image plus sky_level counts (noise.py:292-383)."""

    def __init__(self, rng=None, sky_level=0.):
        BaseNoise.__init__(self, rng)
        self._sky_level = sky_level

    sky_level = property(lambda self: self._sky_level)

    def _params(self, dtype):
        p = NoiseParamsC()
        p.sky_level = float(self._sky_level)
        p.frac_sky, p.int_sky, p.int_sky_same_dtype = _sky_split(self._sky_level, dtype)
        return POISSON, p

    def _getVariance(self):
        return self.sky_level

    def _withVariance(self, variance):
        return PoissonNoise(self.rng, variance)

    def _withScaledVariance(self, variance_ratio):
        return PoissonNoise(self.rng, self.sky_level * variance_ratio)

    def copy(self, rng=None):
        return PoissonNoise(self.rng if rng is None else rng, self.sky_level)

    def __repr__(self):
        return 'galsim.PoissonNoise(rng=%r, sky_level=%r)' % (self.rng, self.sky_level)


class CCDNoise(BaseNoise):
    """Poisson noise in electrons (gain e- / ADU) plus Gaussian read noise (noise.py:384-550)."""

    def __init__(self, rng=None, sky_level=0., gain=1., read_noise=0.):
        BaseNoise.__init__(self, rng)
        self._sky_level = float(sky_level)
        self._gain = float(gain)
        self._read_noise = float(read_noise)

    sky_level = property(lambda self: self._sky_level)
    gain = property(lambda self: self._gain)
    read_noise = property(lambda self: self._read_noise)

    def _params(self, dtype):
        p = NoiseParamsC()
        p.sky_level = self._sky_level
        p.gain = self._gain
        p.read_noise = self._read_noise
        p.frac_sky, p.int_sky, p.int_sky_same_dtype = _sky_split(self._sky_level, dtype)
        return CCD, p

    def _getVariance(self):
        if self.gain > 0.:
            return self.sky_level / self.gain + (self.read_noise / self.gain) ** 2
        return self.read_noise ** 2

    def _withVariance(self, variance):
        current = self._getVariance()
        if current > 0.:
            return self._withScaledVariance(variance / current)
        return CCDNoise(self.rng, sky_level=variance)

    def _withScaledVariance(self, variance_ratio):
        return CCDNoise(self.rng, gain=self.gain, sky_level=self.sky_level * variance_ratio,
                        read_noise=self.read_noise * math.sqrt(variance_ratio))

    def copy(self, rng=None):
        return CCDNoise(self.rng if rng is None else rng, self.sky_level, self.gain, self.read_noise)

    def __repr__(self):
        return 'galsim.CCDNoise(rng=%r, sky_level=%r, gain=%r, read_noise=%r)' % (
            self.rng, self.sky_level, self.gain, self.read_noise)


class VariableGaussianNoise(BaseNoise):
    """Gaussian noise with its own variance in every pixel (noise.py:590-664): pixel i gets the
    i-th unit deviate of the stream times sqrt(var_image[i]) (GaussianDeviate.generateFromVariance,
    Random.cpp:402-450), added in the image's type."""

    def __init__(self, rng, var_image):
        from .image import ImageD
        BaseNoise.__init__(self, rng)
        self._var_image = ImageD(var_image)

    var_image = property(lambda self: self._var_image)

    def applyTo(self, image):
        from .image import Image
        from .errors import GalSimIncompatibleValuesError
        if not isinstance(image, Image):
            raise TypeError("Provided image must be a galsim.Image")
        if image.array.shape != self.var_image.array.shape:
            raise GalSimIncompatibleValuesError(
                "Provided image shape does not match the shape of var_image",
                image=image, var_image=self.var_image)
        self._applyTo(image)

    def _params(self, dtype):
        return VARIABLE_GAUSSIAN, NoiseParamsC()

    def _variances(self, n_rep):
        """The variances as an FP64 device buffer laid out like n_rep stamps of the image."""
        import torch
        var = np.ascontiguousarray(self._var_image.array, dtype=np.float64).reshape(-1)
        t = torch.from_numpy(var).to(_lib.Device.torch_device())
        return t.repeat(n_rep) if n_rep > 1 else t

    def _applyTo(self, image):
        import torch
        arr = image.array
        if arr.dtype not in _IMAGE_TYPES:
            raise GalSimNotImplementedError("noise is applied to float32 / float64 / int16 / int32 / "
                                            "uint16 / uint32 images")
        host = np.ascontiguousarray(arr)
        flat = torch.from_numpy(host.reshape(-1).copy()).to(_lib.Device.torch_device())
        st = self._rng._stream
        used = _apply(VARIABLE_GAUSSIAN, NoiseParamsC(), flat, [0], [host.size], [st.seed], [st.used],
                      scratch=self._variances(1))
        arr[...] = flat.cpu().numpy().reshape(arr.shape)
        st.used = int(used[0])

    def _apply_batch(self, sb, seeds, skips=None):
        from .errors import GalSimIncompatibleValuesError
        B = len(sb.offsets)
        shape = self._var_image.array.shape
        if (np.any(np.asarray(sb.ny) != shape[0]) or np.any(np.asarray(sb.nx) != shape[1]) or
                np.any(np.asarray(sb.offsets, np.int64) != np.arange(B, dtype=np.int64) * shape[0] * shape[1])):
            raise GalSimIncompatibleValuesError(
                "every stamp must have the shape of var_image", var_image=self.var_image)
        seeds = np.broadcast_to(np.asarray(seeds, dtype=np.int64), (B,))
        if np.any(seeds == 0):
            raise GalSimValueError("stamp seeds must be nonzero", seeds)
        skips = np.zeros(B, np.int64) if skips is None else np.broadcast_to(np.asarray(skips, np.int64), (B,))
        npix = np.full(B, shape[0] * shape[1], np.int32)
        return _apply(VARIABLE_GAUSSIAN, NoiseParamsC(), sb.flat, np.asarray(sb.offsets, np.int64), npix,
                      seeds, skips, scratch=self._variances(B))

    def copy(self, rng=None):
        return VariableGaussianNoise(self.rng if rng is None else rng, self.var_image)

    def _getVariance(self):
        raise GalSimError("No single variance value for VariableGaussianNoise")

    def _withVariance(self, variance):
        raise GalSimError("Changing the variance is not allowed for VariableGaussianNoise")

    def _withScaledVariance(self, variance):
        raise GalSimError("Changing the variance is not allowed for VariableGaussianNoise")

    def __repr__(self):
        return 'galsim.VariableGaussianNoise(rng=%r, var_image%r)' % (self.rng, self.var_image)


class DeviateNoise(BaseNoise):
    """Noise drawn from a deviate (noise.py:532-588): dev.generate fills one value per pixel in
    row-major order (on the GPU, galsim_b200.random), added to the image in its type."""

    def __init__(self, dev):
        BaseNoise.__init__(self, dev)

    def _applyTo(self, image):
        arr = image.array
        noise = np.empty(arr.size, dtype=float)
        self._rng.generate(noise)
        arr[...] += noise.reshape(arr.shape).astype(arr.dtype)

    def _apply_batch(self, sb, seeds, skips=None):
        raise GalSimNotImplementedError("DeviateNoise on a stamp batch is not built")

    def _getVariance(self):
        raise GalSimError("No single variance value for DeviateNoise")

    def _withVariance(self, variance):
        raise GalSimError("Changing the variance is not allowed for DeviateNoise")

    def _withScaledVariance(self, variance):
        raise GalSimError("Changing the variance is not allowed for DeviateNoise")

    def copy(self, rng=None):
        if rng is None:
            dev = self.rng
        else:
            dev = self.rng.duplicate()
            dev.reset(rng)
        return DeviateNoise(dev)

    def __repr__(self):
        return 'galsim.DeviateNoise(dev=%r)' % self.rng


__all__ = ['BaseDeviate', 'BaseNoise', 'GaussianNoise', 'PoissonNoise', 'CCDNoise', 'VariableGaussianNoise',
           'DeviateNoise']

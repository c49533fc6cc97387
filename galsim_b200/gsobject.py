"""GSObject: the base class of every surface-brightness profile (galsim/gsobject.py).

Drawing goes through the GPU: ``drawImage(method='fft')`` (also 'auto'), 'no_pixel' / 'sb'
(by FFT for profiles that are not analytic in real space, by real-space evaluation --
``drawReal`` -- for sums and transformations of analytic leaves, as the reference chooses) and
``drawKImage``.  Real-space convolution and photon shooting are not part of this package and
raise GalSimNotImplementedError.  Multiplying by an SED makes a chromatic object
(galsim_b200.chromatic).

Parameters of the leaf profiles may be numpy arrays: such an object stands for a batch of
profiles (one per array element) with the same tree structure, and is drawn with
``galsim_b200.draw_batch``.  Scalar objects behave like the reference's.
"""
import math

import numpy as np

from . import _lib
from .bounds import BoundsI, _BoundsI
from .errors import (GalSimError, GalSimIncompatibleValuesError, GalSimNotImplementedError,
                     GalSimRangeError, GalSimValueError, galsim_warn)
from .gsparams import GSParams
from .image import Image, ImageCD, ImageCF
from .position import Position, PositionD, _PositionD, _PositionI, parse_pos_args
from .shear import Shear
from .wcs import BaseWCS, PixelScale


def _as_param(v):
    """A scalar as float, an array as a 1-d float64 array."""
    if np.ndim(v) == 0:
        return float(v)
    return np.asarray(v, dtype=np.float64).reshape(-1)


def _plen(*vals):
    n = 1
    for v in vals:
        if np.ndim(v):
            m = np.size(v)
            if n != 1 and m != 1 and m != n:
                raise GalSimIncompatibleValuesError("batched parameters have different lengths")
            n = max(n, m)
    return n


class GSObject(object):
    _has_hard_edges = False
    _is_axisymmetric = False
    _is_analytic_x = False
    _is_analytic_k = True
    _batch = 1

    # -- basic properties -------------------------------------------------------------------
    @property
    def flux(self):
        return self._flux

    @property
    def gsparams(self):
        return self._gsparams

    @property
    def has_hard_edges(self):
        return self._has_hard_edges

    @property
    def is_axisymmetric(self):
        return self._is_axisymmetric

    @property
    def is_analytic_x(self):
        return self._is_analytic_x

    @property
    def is_analytic_k(self):
        return self._is_analytic_k

    def _sizes(self):
        if not hasattr(self, '_cached_sizes'):
            from .program import Program
            self._cached_sizes = Program(self).stepk_maxk()
        return self._cached_sizes

    @property
    def maxk(self):
        """The k beyond which aliasing can be neglected (gsobject.py:267-271)."""
        mk = self._sizes()[1]
        return float(mk[0]) if self._batch == 1 else mk

    @property
    def stepk(self):
        """The k-space sampling that avoids folding (gsobject.py:273-277)."""
        sk = self._sizes()[0]
        return float(sk[0]) if self._batch == 1 else sk

    @property
    def nyquist_scale(self):
        return math.pi / self.maxk

    # -- sizing composition (overridden by composites) ---------------------------------------
    def _size(self, prog, it):
        return prog.leaf_size(next(it))

    # -- operators (gsobject.py:459-505, 781-1092) -------------------------------------------
    def __add__(self, other):
        from .compound import Add
        return Add([self, other])

    def __sub__(self, other):
        from .compound import Add
        return Add([self, (-1. * other)])

    def __mul__(self, other):
        return self.withScaledFlux(other)

    def __rmul__(self, other):
        return self.__mul__(other)

    def __div__(self, other):
        return self * (1. / other)

    __truediv__ = __div__

    def __neg__(self):
        return -1. * self

    def withGSParams(self, gsparams=None, **kwargs):
        if gsparams == self.gsparams and not kwargs:
            return self
        import copy
        ret = copy.copy(self)
        ret._gsparams = GSParams.check(gsparams, self.gsparams, **kwargs)
        ret.__dict__.pop('_cached_sizes', None)
        return ret

    def withFlux(self, flux):
        return self.withScaledFlux(flux / self.flux)

    def withScaledFlux(self, flux_ratio):
        from .compound import Transform
        from .sed import SED
        if isinstance(flux_ratio, SED):
            # obj * SED: a separable chromatic object (gsobject.py:799-838, transform.py:76-83)
            from .chromatic import SimpleChromaticTransformation
            return SimpleChromaticTransformation(self, flux_ratio)
        if hasattr(flux_ratio, '__call__'):
            raise TypeError('callable flux_ratio must be an SED.')
        if np.ndim(flux_ratio) == 0 and flux_ratio == 1:
            return self
        return Transform(self, flux_ratio=flux_ratio)

    # -- duck typing as a ChromaticObject (gsobject.py:427-454) --------------------------------
    separable = property(lambda self: True)
    interpolated = property(lambda self: False)
    deinterpolated = property(lambda self: self)
    spectral = property(lambda self: False)
    dimensionless = property(lambda self: True)
    wave_list = property(lambda self: np.array([], dtype=float))

    @property
    def sed(self):
        from .sed import SED
        return SED(float(self.flux), 'nm', '1')

    def _fiducial_profile(self, bandpass):
        return bandpass.effective_wavelength, self

    def evaluateAtWavelength(self, wave):
        return self

    def _approxWavelength(self, wave):
        return wave, self

    def expand(self, scale):
        from .compound import Transform
        return Transform(self, jac=_diag_jac(scale))

    def dilate(self, scale):
        from .compound import Transform
        return Transform(self, jac=_diag_jac(scale), flux_ratio=np.asarray(scale, float) ** -2
                         if np.ndim(scale) else scale ** -2)

    def magnify(self, mu):
        return self.expand(np.sqrt(mu) if np.ndim(mu) else math.sqrt(mu))

    def shear(self, *args, **kwargs):
        from .compound import Transform
        if len(args) == 1:
            if kwargs:
                raise TypeError("Error, gave both unnamed and named arguments to GSObject.shear!")
            if not isinstance(args[0], Shear):
                raise TypeError("Error, unnamed argument to GSObject.shear is not a Shear!")
            shear = args[0]
        elif len(args) > 1:
            raise TypeError("Error, too many unnamed arguments to GSObject.shear!")
        elif len(kwargs) == 0:
            raise TypeError("Error, shear argument is required")
        else:
            shear = Shear(**kwargs)
        return Transform(self, shear.getMatrix())

    def _shear(self, shear):
        from .compound import _Transform
        return _Transform(self, shear.getMatrix())

    def lens(self, g1, g2, mu):
        from .compound import Transform
        m = Shear(g1=g1, g2=g2).getMatrix()
        return Transform(self, m * (np.sqrt(mu)[..., None, None] if np.ndim(mu) else math.sqrt(mu)))

    def rotate(self, theta):
        from .angle import Angle
        from .compound import Transform
        if not isinstance(theta, Angle):
            raise TypeError("Input theta should be an Angle")
        s, c = theta.sincos()
        return Transform(self, jac=[c, -s, s, c])

    def transform(self, dudx, dudy, dvdx, dvdy):
        from .compound import Transform
        return Transform(self, jac=[dudx, dudy, dvdx, dvdy])

    def shift(self, *args, **kwargs):
        from .compound import Transform
        if len(args) == 2 and not kwargs and (np.ndim(args[0]) or np.ndim(args[1])):
            return Transform(self, offset=(args[0], args[1]))
        offset = parse_pos_args(args, kwargs, 'dx', 'dy')
        return Transform(self, offset=offset)

    def _shift(self, dx, dy):
        from .compound import _Transform
        return _Transform(self, offset=(dx, dy))

    # -- image set-up (gsobject.py:1115-1281) ------------------------------------------------
    def _setup_image(self, image, nx, ny, bounds, add_to_image, dtype, center, odd=False):
        if image is not None:
            if bounds is not None:
                raise GalSimIncompatibleValuesError(
                    "Cannot provide bounds if image is provided", bounds=bounds, image=image)
            if nx is not None or ny is not None:
                raise GalSimIncompatibleValuesError(
                    "Cannot provide nx,ny if image is provided", nx=nx, ny=ny, image=image)
            if dtype is not None and image.array.dtype != dtype:
                raise GalSimIncompatibleValuesError(
                    "Cannot specify dtype != image.array.dtype if image is provided",
                    dtype=dtype, image=image)
            if not image.bounds.isDefined():
                if add_to_image:
                    raise GalSimIncompatibleValuesError(
                        "Cannot add_to_image if image bounds are not defined",
                        add_to_image=add_to_image, image=image)
                N = self.getGoodImageSize(1.0)
                if odd:
                    N += 1
                image.resize(_BoundsI(1, N, 1, N))
        else:
            if add_to_image:
                raise GalSimIncompatibleValuesError(
                    "Cannot add_to_image if image is None", add_to_image=add_to_image, image=image)
            if bounds is not None:
                if nx is not None or ny is not None:
                    raise GalSimIncompatibleValuesError(
                        "Cannot set both bounds and (nx, ny)", nx=nx, ny=ny, bounds=bounds)
                if not bounds.isDefined():
                    raise GalSimValueError("Cannot use undefined bounds", bounds)
                image = Image(bounds=bounds, dtype=dtype)
            elif nx is not None or ny is not None:
                if nx is None or ny is None:
                    raise GalSimIncompatibleValuesError(
                        "Must set either both or neither of nx, ny", nx=nx, ny=ny)
                image = Image(nx, ny, dtype=dtype)
                if center is not None:
                    image.shift(_PositionI(np.floor(center.x + 0.5 - image.true_center.x),
                                           np.floor(center.y + 0.5 - image.true_center.y)))
            else:
                N = self.getGoodImageSize(1.0)
                if odd:
                    N += 1
                image = Image(N, N, dtype=dtype)
                if center is not None:
                    image.setCenter(_PositionI(np.ceil(center.x), np.ceil(center.y)))
        return image

    def _local_wcs(self, wcs, image, offset, center, use_true_center, new_bounds):
        return wcs.local()

    def _parse_offset(self, offset):
        if offset is None:
            return _PositionD(0, 0)
        elif isinstance(offset, Position):
            return _PositionD(offset.x, offset.y)
        return _PositionD(offset[0], offset[1])

    def _parse_center(self, center):
        if center is None:
            return None
        elif isinstance(center, Position):
            return _PositionD(center.x, center.y)
        return _PositionD(center[0], center[1])

    def _get_new_bounds(self, image, nx, ny, bounds, center):
        if image is not None and image.bounds.isDefined():
            return image.bounds
        elif nx is not None and ny is not None:
            b = BoundsI(1, nx, 1, ny)
            if center is not None:
                b = b.shift(_PositionI(np.floor(center.x + 0.5 - b.true_center.x),
                                       np.floor(center.y + 0.5 - b.true_center.y)))
            return b
        elif bounds is not None and bounds.isDefined():
            return bounds
        return BoundsI()

    def _adjust_offset(self, new_bounds, offset, center, use_true_center):
        if center is not None:
            if new_bounds.isDefined():
                offset += center - new_bounds.center
            else:
                offset += _PositionD(center.x - np.ceil(center.x), center.y - np.ceil(center.y))
        elif use_true_center:
            dx = offset.x
            dy = offset.y
            shape = new_bounds.numpyShape()
            if shape[1] % 2 == 0:
                dx -= 0.5
            if shape[0] % 2 == 0:
                dy -= 0.5
            offset = _PositionD(dx, dy)
        return offset

    def _determine_wcs(self, scale, wcs, image, default_wcs=None):
        if wcs is not None:
            if scale is not None:
                raise GalSimIncompatibleValuesError(
                    "Cannot provide both wcs and scale", wcs=wcs, scale=scale)
            if not isinstance(wcs, BaseWCS):
                raise TypeError("wcs must be a BaseWCS instance")
            if image is not None:
                image.wcs = None
        elif scale is not None:
            wcs = PixelScale(scale)
            if image is not None:
                image.wcs = None
        elif image is not None and image.wcs is not None:
            wcs = image.wcs
        if wcs is None or (wcs._isPixelScale and not wcs.scale > 0):
            wcs = PixelScale(self.nyquist_scale) if default_wcs is None else default_wcs
        if not wcs._isPixelScale:
            raise GalSimNotImplementedError("only PixelScale WCS is supported by the FFT path")
        return wcs

    def getGoodImageSize(self, pixel_scale):
        """gsobject.py:1900-1925."""
        Nd = 2. * math.pi / (pixel_scale * self.stepk)
        N = int(math.ceil(Nd * (1. - 1.e-12)))
        return 2 * ((N + 1) // 2)

    # -- drawing ----------------------------------------------------------------------------
    def drawImage(self, image=None, nx=None, ny=None, bounds=None, scale=None, wcs=None, dtype=None,
                  method='auto', area=1., exptime=1., gain=1., add_to_image=False,
                  center=None, use_true_center=True, offset=None,
                  n_photons=0., rng=None, max_extra_noise=0.,
                  poisson_flux=None, sensor=None, photon_ops=None, n_subsample=3, maxN=None,
                  save_photons=False, bandpass=None, setup_only=False, surface_ops=None,
                  precision='fp32'):
        """Draw the profile into an Image (gsobject.py:1283-1844) through the GPU FFT path.

        ``precision`` ('fp32' default, or 'fp64') selects the arithmetic of the k-space
        evaluation and the FFT; it is the only argument the reference does not have."""
        from . import box, compound
        if self._batch != 1:
            raise GalSimIncompatibleValuesError(
                "drawImage draws one profile; use galsim_b200.draw_batch for batched parameters")
        if image is not None and not isinstance(image, Image):
            raise TypeError("image is not an Image instance", image)
        if not gain > 0.:
            raise GalSimRangeError("Invalid gain <= 0.", gain, 0., None)
        if not area > 0.:
            raise GalSimRangeError("Invalid area <= 0.", area, 0., None)
        if not exptime > 0.:
            raise GalSimRangeError("Invalid exptime <= 0.", exptime, 0., None)
        if method not in ('auto', 'fft', 'real_space', 'phot', 'no_pixel', 'sb'):
            raise GalSimValueError("Invalid method name", method,
                                   ('auto', 'fft', 'real_space', 'phot', 'no_pixel', 'sb'))
        if method == 'auto' and isinstance(self, compound.Convolution):
            if any(isinstance(obj, box.Pixel) for obj in self.obj_list):
                galsim_warn(
                    "You called drawImage with ``method='auto'`` for an object that includes "
                    "convolution by a Pixel.  This is probably an error.  Normally, you should "
                    "let GalSim handle the Pixel convolution for you.  If you want to handle the "
                    "Pixel convolution yourself, you can use method=no_pixel.  Or if you really "
                    "meant for your profile to include the Pixel and also have GalSim convolve by "
                    "an _additional_ Pixel, you can suppress this warning by using method=fft.")
        if method in ('phot', 'real_space'):
            raise GalSimNotImplementedError("method=%r is not part of the FFT drawing path" % method)
        if method != 'phot':
            if n_photons != 0.:
                raise GalSimIncompatibleValuesError(
                    "n_photons is only relevant for method='phot'", method=method, n_photons=n_photons)
            if max_extra_noise != 0.:
                raise GalSimIncompatibleValuesError(
                    "max_extra_noise is only relevant for method='phot'", method=method,
                    max_extra_noise=max_extra_noise)
            if poisson_flux is not None:
                raise GalSimIncompatibleValuesError(
                    "poisson_flux is only relevant for method='phot'", method=method,
                    poisson_flux=poisson_flux)
        if sensor is not None or photon_ops or surface_ops is not None:
            raise GalSimNotImplementedError("sensors and photon operators are not part of the FFT path")
        if rng is not None:
            raise GalSimIncompatibleValuesError(
                "rng is only relevant for method='phot' or when using a sensor", method=method, rng=rng)
        if maxN is not None:
            raise GalSimIncompatibleValuesError(
                "maxN is only relevant for method='phot' or when using a sensor", method=method, maxN=maxN)
        if save_photons:
            raise GalSimIncompatibleValuesError(
                "save_photons is only valid for method='phot' or when using a sensor",
                method=method, save_photons=save_photons)

        wcs = self._determine_wcs(scale, wcs, image)
        offset = self._parse_offset(offset)
        center = self._parse_center(center)
        new_bounds = self._get_new_bounds(image, nx, ny, bounds, center)
        local_wcs = self._local_wcs(wcs, image, offset, center, use_true_center, new_bounds)
        flux_scale = area * exptime
        if method == 'sb':
            flux_scale /= local_wcs.pixelArea()
        if gain != 1:
            flux_scale /= gain
        offset = self._adjust_offset(new_bounds, offset, center, use_true_center)
        prof = local_wcs.profileToImage(self, flux_ratio=flux_scale, offset=offset)
        if method in ('auto', 'fft'):
            real_space = None if method == 'auto' else False
            prof = compound.Convolve(prof, box.Pixel(scale=1.0, gsparams=self.gsparams),
                                     real_space=real_space, gsparams=self.gsparams)
            if prof.real_space:
                raise GalSimNotImplementedError("real-space convolution is not part of the FFT path")
        image = prof._setup_image(image, nx, ny, bounds, add_to_image, dtype, center)
        image.wcs = wcs
        if setup_only:
            image.added_flux = 0.
            return image
        imview = image._view()
        imview._shift(-image.center)
        imview.wcs = PixelScale(1.0)
        if prof.is_analytic_x:
            # method 'no_pixel' / 'sb' on a profile analytic in real space (gsobject.py:1810-1811)
            added_photons = prof.drawReal(imview, add_to_image)
        else:
            added_photons = prof.drawFFT(imview, add_to_image, precision=precision)
        image.added_flux = added_photons / flux_scale
        return image

    def drawReal(self, image, add_to_image=False):
        """The profile sampled at the pixel centres of an image with a PixelScale wcs, times the
        pixel area (gsobject.py:1846-1889), drawn on the GPU (gsb_draw_real).  Returns the total
        flux drawn."""
        import torch
        from .compound import _Transform
        from .realspace import draw_real_stamps
        if image.wcs is None or not image.wcs._isPixelScale:
            raise GalSimValueError("drawReal requires an image with a PixelScale wcs", image)
        if self._batch != 1:
            raise GalSimIncompatibleValuesError(
                "drawReal draws one profile; use galsim_b200.draw_batch for batched parameters")
        if image.dtype not in (np.float32, np.float64):
            raise GalSimNotImplementedError("drawReal into an image of dtype %s" % image.dtype)
        scale = image.scale
        prof = self if scale == 1. else _Transform(self, jac=np.array([[1. / scale, 0.], [0., 1. / scale]]),
                                                    flux_ratio=scale ** 2)
        b = image.bounds
        nx, ny = b.xmax - b.xmin + 1, b.ymax - b.ymin + 1
        init = None
        if add_to_image:
            init = torch.from_numpy(np.ascontiguousarray(image.array).reshape(-1).copy()).to(
                _lib.Device.torch_device())
        out, _, flux = draw_real_stamps(prof, 1, self.gsparams, [b.xmin], [b.ymin], [nx], [ny], image.dtype,
                                        init=init)
        image.array[...] = out.cpu().numpy().reshape(image.array.shape)
        return float(flux[0].item())

    def drawFFT(self, image, add_to_image=False, precision='fp32'):
        """Draw by k-space evaluation and FFT into an image with a PixelScale wcs, centred on
        (0,0) of its bounds (gsobject.py:2014-2045).  Returns the drawn flux."""
        from .program import Program, fft_sizes
        if image.wcs is None or not image.wcs._isPixelScale:
            raise GalSimValueError("drawPhot requires an image with a PixelScale wcs", image)
        prog = Program(self)
        stepk, maxk = prog.stepk_maxk()
        b = image.bounds
        N, Nk = fft_sizes(stepk, maxk, b.xmin, b.xmax, b.ymin, b.ymax, self.gsparams,
                          scale=image.scale)
        if image.scale != 1.0:
            raise GalSimNotImplementedError("drawFFT draws in image coordinates (scale 1)")
        out_f64 = image.dtype != np.float32
        dtype = _lib.F64 if out_f64 else _lib.F32
        prec = _lib.F64 if precision == 'fp64' else _lib.F32
        out, _, flux = prog.draw_stamps(N, Nk, [b.xmin], [b.ymin], [b.xmax - b.xmin + 1],
                                        [b.ymax - b.ymin + 1], dtype, precision=prec)
        arr = out[:image.array.size].cpu().numpy().reshape(image.array.shape)
        if add_to_image:
            image.array[...] += arr.astype(image.dtype, copy=False)
        else:
            image.array[...] = arr
        return float(flux[0].item())

    def drawKImage(self, image=None, nx=None, ny=None, bounds=None, scale=None,
                   add_to_image=False, recenter=True, bandpass=None, setup_only=False,
                   precision=None):
        """The k-space image of the profile (gsobject.py:2464-2582)."""
        if self._batch != 1:
            raise GalSimIncompatibleValuesError("drawKImage draws one profile")
        if image is not None:
            if not isinstance(image, Image):
                raise TypeError("Provided image must be galsim.Image", image)
            if not image.iscomplex:
                raise GalSimValueError("Provided image must be complex", image)
        if image is not None and scale is None:
            scale = image.scale
        if scale is None or not scale > 0:
            dk = self.stepk
        else:
            dk = float(scale)
        if image is not None and image.bounds.isDefined():
            dx = np.pi / (max(image.array.shape) // 2 * dk)
        elif scale is None or not scale > 0:
            dx = self.nyquist_scale
        else:
            dx = self.nyquist_scale * dk / self.stepk
        if image is None or not image.bounds.isDefined():
            real_prof = PixelScale(dx).profileToImage(self)
            dtype = np.complex128 if image is None else image.dtype
            image = real_prof._setup_image(image, nx, ny, bounds, add_to_image, dtype,
                                           center=None, odd=True)
        else:
            if bounds is not None:
                raise GalSimIncompatibleValuesError(
                    "Cannot provide bounds if image is provided", bounds=bounds, image=image)
            if nx is not None or ny is not None:
                raise GalSimIncompatibleValuesError(
                    "Cannot provide nx,ny if image is provided", nx=nx, ny=ny, image=image)
        if recenter and image.center != _PositionI(0, 0) and add_to_image:
            raise GalSimIncompatibleValuesError(
                "Cannot use add_to_image=True unless image is centered at (0,0) or recenter=False",
                recenter=recenter, image=image, add_to_image=add_to_image)
        if recenter and image.center != _PositionI(0, 0):
            image._shift(-image.center)
        image.scale = dk
        if setup_only:
            return image
        self._drawKImage_into(image, add_to_image, precision)
        return image

    def _drawKImage(self, image, jac=None):
        """Draw into a complex image with its own bounds and scale = dk (no checks)."""
        if jac is not None:
            from .compound import _Transform
            return _Transform(self, jac)._drawKImage_into(image, False, None)
        self._drawKImage_into(image, False, None)

    def _drawKImage_into(self, image, add, precision):
        from .program import Program
        prog = Program(self)
        b = image.bounds
        f64 = image.dtype == np.complex128 if precision is None else precision == 'fp64'
        arr = prog.draw_kimage(image.scale, b.xmin, b.ymin, b.xmax - b.xmin + 1,
                               b.ymax - b.ymin + 1, _lib.F64 if f64 else _lib.F32)[0]
        if add:
            image.array[...] += arr
        else:
            image.array[...] = arr


def _diag_jac(scale):
    if np.ndim(scale):
        s = np.asarray(scale, float)
        j = np.zeros(s.shape + (2, 2))
        j[..., 0, 0] = s
        j[..., 1, 1] = s
        return j
    return [scale, 0., 0., scale]


__all__ = ['GSObject']

"""Chromatic objects and their drawing through a bandpass (galsim/chromatic.py).

A ChromaticObject is a surface brightness profile that depends on wavelength: a GSObject
times an SED (separable), a PSF whose size and position change with wavelength
(ChromaticAtmosphere, or any transformation by functions of wavelength), and convolutions and
sums of those.  drawImage(bandpass) integrates the profile times the throughput over
wavelength with the reference's algorithm and numbers (chromatic.py:409-525, 2852-3055):

  * separable profiles are drawn once, at the fiducial wavelength, scaled by the integral of
    SED x throughput (ChromaticObject.drawImage :483-487);
  * otherwise the integrand is drawn at the integration wavelengths and summed with the
    rule's weights.  Here all wavelengths are drawn in ONE batched pass (each with its own
    FFT size as the reference sizes each of its per-wavelength drawImage calls, or in real
    space where the reference draws in real space), and the weighted sum is taken on the
    device (gsb_weighted_stamp_sum);
  * a convolution of separable galaxies with inseparable PSFs is drawn as the reference does:
    sums are distributed over the convolution, the inseparable factors times the galaxy's SED
    are integrated into an "effective PSF" image at half the Nyquist scale (drawn as above,
    without a pixel -- in real space for analytic PSFs) and turned into an InterpolatedImage,
    and the galaxy's spatial profile is convolved with it and drawn once
    (chromatic.py:2752-2779, 2999-3030).

Not built: photon shooting, InterpolatedChromaticObject (interpolate()), chromatic
deconvolution / autoconvolution / Fourier square root, ChromaticOpticalPSF / ChromaticAiry,
drawKImage of chromatic objects, celestial-coordinate DCR angles.
"""
import copy

import numpy as np

from .gsobject import GSObject
from .sed import SED, combine_wave_list
from .bandpass import Bandpass
from .table import _LookupTable
from .gsparams import GSParams
from .angle import arcsec, AngleUnit
from .position import PositionD
from .shear import Shear
from . import integ, dcr
from .errors import (GalSimError, GalSimSEDError, GalSimValueError, GalSimIncompatibleValuesError,
                     GalSimNotImplementedError)

__all__ = ['ChromaticObject', 'ChromaticTransformation', 'SimpleChromaticTransformation',
           'ChromaticAtmosphere', 'ChromaticAiry', 'ChromaticSum', 'ChromaticConvolution', 'draw_batch_chromatic']


def _remove_setup_kwargs(kwargs):
    """chromatic.py:3912-3920."""
    for k in ('dtype', 'scale', 'wcs', 'nx', 'ny', 'bounds'):
        kwargs.pop(k, None)


def _get_multiplier(sed, bandpass, wave_list):
    """Integral of SED x throughput (chromatic.py:214-224)."""
    wave_list = np.asarray(wave_list, dtype=float)
    if len(wave_list) > 0:
        bp = _LookupTable(wave_list, bandpass(wave_list), 'linear')
        return bp.integrate_product(sed)
    raise GalSimNotImplementedError("the SED x throughput integral of analytic functions is not built")


def _get_integrator(integrator, wave_list):
    """chromatic.py:1095-1117."""
    if isinstance(integrator, str):
        rule = {'quadratic': integ.quadRule, 'trapezoidal': integ.trapzRule,
                'midpoint': integ.midptRule}.get(integrator)
        if rule is None:
            raise GalSimValueError("Unrecognized integration rule", integrator,
                                   ('trapezoidal', 'midpoint', 'quadratic'))
        if len(wave_list) > 0:
            return integ.SampleIntegrator(rule)
        return integ.ContinuousIntegrator(rule)
    if not isinstance(integrator, integ.ImageIntegrator):
        raise TypeError("Invalid type passed in for integrator!")
    return integrator


def _integrate_images(chrom, waves, weights, image, kwargs):
    """The integrand of ChromaticObject.drawImage drawn at all `waves` in one batched pass
    (one stamp per wavelength, image's bounds and scale) and summed on the device with
    `weights` into a new Image like `image` (integ.py:257-271 and :134-146)."""
    import torch
    from . import _lib
    from .batch import draw_batch
    from .image import Image
    kw = dict(kwargs)
    method = kw.pop('method', 'auto')
    for k in ('center', 'n_photons', 'rng', 'sensor', 'photon_ops', 'save_photons'):
        if kw.get(k) not in (None, False, 0, 0., []):
            raise GalSimNotImplementedError("chromatic drawing with %s is not built" % k)
        kw.pop(k, None)
    precision = kw.pop('precision', 'fp32')
    offset = kw.pop('offset', None)
    if offset is not None:
        offset = (offset.x, offset.y) if hasattr(offset, 'x') else tuple(offset)
    use_true_center = kw.pop('use_true_center', True)
    area, exptime, gain = kw.pop('area', 1.), kw.pop('exptime', 1.), kw.pop('gain', 1.)
    if kw:
        raise GalSimNotImplementedError("chromatic drawImage arguments not built: %s" % sorted(kw))
    profs = chrom._evaluate_batch(waves)
    nx, ny = image.array.shape[1], image.array.shape[0]
    st = draw_batch(profs, nx=nx, ny=ny, scale=image.scale, dtype=np.dtype(image.dtype).type, method=method,
                    area=area, exptime=exptime, gain=gain, offset=offset, use_true_center=use_true_center,
                    precision=precision)
    if len(st) != len(waves):
        raise GalSimError("internal: the chromatic integrand batch has %d stamps for %d wavelengths"
                          % (len(st), len(waves)))
    dev = st.flat.device
    d_off = torch.as_tensor(np.asarray(st.offsets, dtype=np.int64), device=dev)
    d_w = torch.as_tensor(np.asarray(weights, dtype=np.float64), device=dev)
    f64 = np.dtype(image.dtype) == np.float64
    out = torch.empty(nx * ny, dtype=torch.float64 if f64 else torch.float32, device=dev)
    in_dt = _lib.F64 if st.flat.dtype == torch.float64 else _lib.F32
    _lib.check(_lib.lib().gsb_weighted_stamp_sum(
        _lib.ptr(st.flat), in_dt, _lib.ptr(d_off), _lib.ptr(d_w), len(waves), nx * ny, _lib.ptr(out),
        _lib.F64 if f64 else _lib.F32, _lib.Device.stream()))
    ret = Image(out.cpu().numpy().reshape(ny, nx).astype(image.dtype, copy=False), xmin=image.xmin,
                ymin=image.ymin, wcs=image.wcs)
    ret.added_flux = float(np.dot(np.asarray(weights, float), st.added_flux))
    return ret


def _is_chromatic_callable(x):
    return hasattr(x, '__call__')


class ChromaticObject(object):
    """Base of the wavelength-dependent profiles (chromatic.py:55-1190).  Made from a GSObject
    it is that profile with a dimensionless flat SED, on which the transformation methods
    accept functions of wavelength in nm."""

    def __init__(self, obj):
        if not isinstance(obj, (GSObject, ChromaticObject)):
            raise TypeError("Can only directly instantiate ChromaticObject with a GSObject "
                            "or ChromaticObject argument.")
        self._obj = obj
        self.separable = obj.separable
        self.interpolated = False
        self.deinterpolated = self

    sed = property(lambda self: self._obj.sed)
    wave_list = property(lambda self: self.sed.wave_list)
    gsparams = property(lambda self: self._obj.gsparams)
    redshift = property(lambda self: self.sed.redshift)
    spectral = property(lambda self: self.sed.spectral)
    dimensionless = property(lambda self: self.sed.dimensionless)

    def withGSParams(self, gsparams=None, **kwargs):
        if gsparams == self.gsparams and not kwargs:
            return self
        ret = copy.copy(self)
        ret._obj = self._obj.withGSParams(gsparams, **kwargs)
        return ret

    # -- monochromatic profiles -----------------------------------------------------------
    def evaluateAtWavelength(self, wave):
        """The monochromatic GSObject at wavelength `wave` (nm)."""
        return self._obj.evaluateAtWavelength(wave)

    def _evaluate_batch(self, waves):
        """The monochromatic profiles at all `waves` as one batched GSObject (batch axis =
        wavelength; achromatic parts broadcast)."""
        return _evaluate_batch(self._obj, waves)

    def _approxWavelength(self, wave):
        return wave, self.evaluateAtWavelength(wave)

    def _fiducial_profile(self, bandpass):
        """chromatic.py:226-259."""
        bpwave = bandpass.effective_wavelength
        bpwave, prof0 = self._approxWavelength(bpwave)
        if np.all(np.asarray(prof0.flux) != 0):
            return bpwave, prof0
        candidate_waves = np.concatenate([np.array([0.5 * (bandpass.blue_limit + bandpass.red_limit)]),
                                          bandpass.wave_list, self.wave_list])
        candidate_waves = candidate_waves[np.argsort(np.abs(candidate_waves - bpwave))]
        for w in candidate_waves:
            if bandpass.blue_limit <= w <= bandpass.red_limit:
                prof0 = self.evaluateAtWavelength(w)
                if np.all(np.asarray(prof0.flux) != 0):
                    return w, prof0
        raise GalSimError("Could not locate fiducial wavelength where SED * Bandpass is nonzero.")

    # -- flux --------------------------------------------------------------------------------
    def calculateFlux(self, bandpass):
        if self.sed.dimensionless:
            raise GalSimSEDError("Cannot calculate flux of dimensionless ChromaticObject.", self.sed)
        return self.sed.calculateFlux(bandpass)

    def withFlux(self, target_flux, bandpass):
        return self * (target_flux / self.calculateFlux(bandpass))

    def withScaledFlux(self, flux_ratio):
        return _Transform(self, flux_ratio=flux_ratio)

    def __mul__(self, flux_ratio):
        return self.withScaledFlux(flux_ratio)

    __rmul__ = __mul__

    def __truediv__(self, other):
        return self.__mul__(1. / other)

    __div__ = __truediv__

    def __add__(self, other):
        return ChromaticSum([self, other])

    def __neg__(self):
        return -1. * self

    # -- transformations (chromatic.py:856-1185) ----------------------------------------------
    def expand(self, scale):
        if _is_chromatic_callable(scale):
            def jac(w):
                s = scale(w)
                return np.array([[s, np.zeros_like(s)], [np.zeros_like(s), s]])
        else:
            jac = None if scale == 1 else np.diag([scale, scale])
        return _Transform(self, jac=jac)

    def dilate(self, scale):
        if _is_chromatic_callable(scale):
            return self.expand(scale).withScaledFlux(lambda w: 1. / scale(w) ** 2)
        return self.expand(scale).withScaledFlux(1. / scale ** 2)

    def magnify(self, mu):
        if _is_chromatic_callable(mu):
            return self.expand(lambda w: np.sqrt(mu(w)))
        return self.expand(np.sqrt(mu))

    def shear(self, *args, **kwargs):
        if len(args) == 1:
            if kwargs:
                raise TypeError("Gave both unnamed and named arguments!")
            shear = args[0]
            if not _is_chromatic_callable(shear) and not isinstance(shear, Shear):
                raise TypeError("Unnamed argument is not a Shear or function returning Shear!")
        elif len(args) > 1:
            raise TypeError("Too many unnamed arguments!")
        elif 'shear' in kwargs:
            shear = kwargs.pop('shear')
            if kwargs:
                raise TypeError("Too many kwargs provided!")
        else:
            shear = Shear(**kwargs)
        if _is_chromatic_callable(shear):
            return _Transform(self, jac=lambda w: shear(w).getMatrix())
        return _Transform(self, jac=shear.getMatrix())

    def _shear(self, shear):
        return _Transform(self, jac=shear.getMatrix())

    def rotate(self, theta):
        if _is_chromatic_callable(theta):
            def jac(w):
                s, c = theta(w).sincos()
                return np.array([[c, -s], [s, c]])
            return _Transform(self, jac=jac)
        s, c = theta.sincos()
        return _Transform(self, jac=np.array([[c, -s], [s, c]]))

    def transform(self, dudx, dudy, dvdx, dvdy):
        if any(_is_chromatic_callable(v) for v in (dudx, dudy, dvdx, dvdy)):
            f = [v if _is_chromatic_callable(v) else (lambda w, v=v: v) for v in (dudx, dudy, dvdx, dvdy)]
            return _Transform(self, jac=lambda w: np.array([[f[0](w), f[1](w)], [f[2](w), f[3](w)]]))
        return _Transform(self, jac=np.array([[dudx, dudy], [dvdx, dvdy]]))

    def shift(self, *args, **kwargs):
        if len(args) == 0:
            dx, dy = kwargs.pop('dx'), kwargs.pop('dy')
        elif len(args) == 1:
            a = args[0]
            if _is_chromatic_callable(a):
                def off(w):
                    v = a(w)
                    return (v.x, v.y) if hasattr(v, 'x') else (v[0], v[1])
                return _Transform(self, offset=off)
            dx, dy = (a.x, a.y) if hasattr(a, 'x') else (a[0], a[1])
        elif len(args) == 2:
            dx, dy = args
        else:
            raise TypeError("Too many arguments supplied!")
        if kwargs:
            raise TypeError("Got unexpected keyword arguments: %s" % kwargs.keys())
        if _is_chromatic_callable(dx) or _is_chromatic_callable(dy):
            fx = dx if _is_chromatic_callable(dx) else (lambda w: dx)
            fy = dy if _is_chromatic_callable(dy) else (lambda w: dy)
            return _Transform(self, offset=lambda w: (fx(w), fy(w)))
        return _Transform(self, offset=(dx, dy))

    def _shift(self, dx, dy):
        return _Transform(self, offset=(dx, dy))

    # -- drawing -----------------------------------------------------------------------------
    def drawImage(self, bandpass, image=None, integrator='quadratic', **kwargs):
        """Image of the profile integrated over the bandpass (chromatic.py:409-525); the
        keyword arguments are GSObject.drawImage's, plus precision."""
        if self.sed.dimensionless:
            raise GalSimSEDError("Can only draw ChromaticObjects with spectral SEDs.", self.sed)
        wave0, prof0 = self._fiducial_profile(bandpass)
        precision = kwargs.pop('precision', 'fp32')
        image = prof0.drawImage(image=image, setup_only=True, **kwargs)
        _remove_setup_kwargs(kwargs)
        wave_list, _, _ = combine_wave_list(self, bandpass)
        if self.separable:
            multiplier = _get_multiplier(self.sed, bandpass, tuple(wave_list))
            prof0 *= multiplier / self.sed(wave0)
            return prof0.drawImage(image=image, precision=precision, **kwargs)
        if kwargs.get('method', None) == 'phot':
            raise GalSimNotImplementedError("photon shooting is not built")
        integrator = _get_integrator(integrator, wave_list)
        if isinstance(integrator, integ.SampleIntegrator):
            if len(wave_list) < 2:
                raise GalSimIncompatibleValuesError(
                    "Cannot use SampleIntegrator when Bandpass and SED are both analytic.",
                    integrator=integrator, bandpass=bandpass, sed=self.sed)
            bandpass = Bandpass(_LookupTable(wave_list, bandpass(wave_list), 'linear'), 'nm')
        add_to_image = kwargs.pop('add_to_image', False)
        kwargs['precision'] = precision
        integral = integrator(self, bandpass, image, kwargs)
        self._last_n_eval = integrator.last_n_eval
        if not add_to_image:
            image.setZero()
        image += integral
        # (image.added_flux stays what the set-up draw left, as in the reference)
        return image

    def drawKImage(self, bandpass, image=None, integrator='quadratic', **kwargs):
        """The Fourier transform of the profile integrated over the bandpass (chromatic.py:
        526-594): the monochromatic k-images at the integrator's wavelengths, as one batch on
        the GPU, summed with the rule's weights in the rule's order; the keyword arguments are
        GSObject.drawKImage's."""
        if self.sed.dimensionless:
            raise GalSimSEDError("Can only drawK ChromaticObjects with spectral SEDs.", self.sed)
        prof0 = self.evaluateAtWavelength(bandpass.effective_wavelength)
        image = prof0.drawKImage(image=image, setup_only=True, **kwargs)
        _remove_setup_kwargs(kwargs)
        wave_list, _, _ = combine_wave_list(self, bandpass)
        if self.separable:
            multiplier = _get_multiplier(self.sed, bandpass, tuple(wave_list))
            prof0 *= multiplier / self.sed(bandpass.effective_wavelength)
            return prof0.drawKImage(image=image, **kwargs)
        integrator = _get_integrator(integrator, wave_list)
        if isinstance(integrator, integ.SampleIntegrator):
            bandpass = Bandpass(_LookupTable(wave_list, bandpass(wave_list), 'linear'), 'nm')
        add_to_image = kwargs.pop('add_to_image', False)
        image_int = integrator(self, bandpass, image, kwargs, doK=True)
        self._last_n_eval = integrator.last_n_eval
        if add_to_image:
            image.array[...] += image_int.array
        else:
            image.array[...] = image_int.array
        return image


def _integrate_kimages(chrom, waves, weights, image, kwargs):
    """The integrand of ChromaticObject.drawKImage at all `waves` in one batched k-space pass on
    the image's grid (its bounds, scale = dk), summed as the rule sums it (integ.py:134-146:
    0 + g_0 K_0 + g_1 K_1 + ..., complex, in the image's precision)."""
    from . import _lib
    from .image import Image
    from .program import Program
    kw = dict(kwargs)
    kw.pop('recenter', None)
    precision = kw.pop('precision', None)
    if kw:
        raise GalSimNotImplementedError("chromatic drawKImage arguments not built: %s" % sorted(kw))
    profs = chrom._evaluate_batch(np.asarray(waves, dtype=float))
    b = image.bounds
    f64 = image.dtype == np.complex128 if precision is None else precision == 'fp64'
    prog = Program(profs)
    arrs = prog.draw_kimage(image.scale, b.xmin, b.ymin, b.xmax - b.xmin + 1, b.ymax - b.ymin + 1,
                            _lib.F64 if f64 else _lib.F32)
    if prog.B != len(waves):
        arrs = np.broadcast_to(arrs, (len(waves),) + arrs.shape[1:])
    acc = 0
    for g, a in zip(weights, arrs):
        acc = acc + g * a.astype(image.dtype)
    return Image(np.asarray(acc, dtype=image.dtype), xmin=b.xmin, ymin=b.ymin, scale=image.scale)


def _evaluate_batch(obj, waves):
    """Batched evaluateAtWavelength of a GSObject or ChromaticObject."""
    if isinstance(obj, GSObject):
        return obj
    return obj._evaluate_batch(waves)


def _stack_jac(jacs):
    return np.stack([np.asarray(j, dtype=float).reshape(2, 2) for j in jacs])


class ChromaticTransformation(ChromaticObject):
    """An affine transformation whose Jacobian, offset and flux ratio may be functions of
    wavelength (chromatic.py:1788-2205); flux_ratio may be an SED."""

    def __init__(self, obj, jac=None, offset=(0., 0.), flux_ratio=1., redshift=None, gsparams=None,
                 propagate_gsparams=True):
        if isinstance(offset, PositionD):
            offset = (offset.x, offset.y)
        self.chromatic = _is_chromatic_callable(jac) or _is_chromatic_callable(offset)
        self.separable = obj.separable and not self.chromatic
        self.interpolated = False
        self.deinterpolated = self
        self._redshift = redshift
        self._gsparams = GSParams.check(gsparams, obj.gsparams)
        self._propagate_gsparams = propagate_gsparams
        if jac is not None and not _is_chromatic_callable(jac):
            jac = np.asarray(jac, dtype=float).reshape(2, 2)
        if not _is_chromatic_callable(offset):
            offset = np.asarray(offset, dtype=float)
        if (isinstance(obj, ChromaticTransformation) and not self.chromatic and not obj.chromatic
                and self._redshift is None and obj._redshift is None):
            self._original = obj._original
            if jac is None:
                self._jac = obj._jac
                self._offset = obj._offset + offset
            else:
                self._jac = jac if obj._jac is None else jac.dot(obj._jac)
                self._offset = jac.dot(obj._offset) + offset
            if (not isinstance(flux_ratio, SED) and
                    (_is_chromatic_callable(flux_ratio) or _is_chromatic_callable(obj._flux_ratio))):
                self._flux_ratio = SED(flux_ratio, 'nm', '1') * obj._flux_ratio
            else:
                self._flux_ratio = obj._flux_ratio * flux_ratio
        else:
            self._original = obj
            self._jac = jac
            self._offset = offset
            self._flux_ratio = flux_ratio
        if self._propagate_gsparams:
            self._original = self._original.withGSParams(self._gsparams)

    original = property(lambda self: self._original)
    gsparams = property(lambda self: self._gsparams)

    @property
    def sed(self):
        fr = self._flux_ratio
        sed = self._original.sed * (fr if isinstance(fr, SED) or _is_chromatic_callable(fr) else float(fr))
        if self._redshift is not None:
            sed = sed.atRedshift(self._redshift)
        if _is_chromatic_callable(self._jac):
            jacf = self._jac

            def detjac(w):
                w = np.asarray(w, dtype=float)
                return np.vectorize(lambda x: np.abs(np.linalg.det(np.asarray(jacf(x)).reshape(2, 2))))(w)
            sed = sed * detjac
        elif self._jac is not None:
            sed = sed * float(np.abs(np.linalg.det(np.asarray(self._jac).reshape(2, 2))))
        return sed

    def withGSParams(self, gsparams=None, **kwargs):
        if gsparams == self.gsparams and not kwargs:
            return self
        ret = copy.copy(self)
        ret._gsparams = GSParams.check(gsparams, self.gsparams, **kwargs)
        if self._propagate_gsparams:
            ret._original = self._original.withGSParams(ret._gsparams)
        return ret

    def _getTransformations(self, wave):
        jac = self._jac(wave) if _is_chromatic_callable(self._jac) else self._jac
        offset = self._offset(wave) if _is_chromatic_callable(self._offset) else self._offset
        fr = self._flux_ratio(wave) if _is_chromatic_callable(self._flux_ratio) else self._flux_ratio
        return jac, offset, fr

    def _approxWavelength(self, wave):
        from .compound import Transformation
        wave1 = wave / (1. + self._redshift) if self._redshift is not None else wave
        wave2, ret = self._original._approxWavelength(wave1)
        wave = wave2 * (1. + self.redshift) if self._redshift is not None else wave2
        jac, offset, fr = self._getTransformations(wave)
        return wave, Transformation(ret, jac=jac, offset=(offset[0], offset[1]), flux_ratio=fr,
                                    gsparams=self._gsparams, propagate_gsparams=self._propagate_gsparams)

    def evaluateAtWavelength(self, wave):
        from .compound import Transformation
        wave1 = wave / (1. + self._redshift) if self._redshift is not None else wave
        ret = self._original.evaluateAtWavelength(wave1)
        jac, offset, fr = self._getTransformations(wave)
        return Transformation(ret, jac=jac, offset=(offset[0], offset[1]), flux_ratio=fr,
                              gsparams=self._gsparams, propagate_gsparams=self._propagate_gsparams)

    def _evaluate_batch(self, waves):
        from .compound import Transformation
        waves = np.asarray(waves, dtype=float)
        w1 = waves / (1. + self._redshift) if self._redshift is not None else waves
        ret = _evaluate_batch(self._original, w1)
        if _is_chromatic_callable(self._jac):
            jac = _stack_jac([self._jac(float(w)) for w in waves])
        else:
            jac = self._jac
        if _is_chromatic_callable(self._offset):
            offs = [self._offset(float(w)) for w in waves]
            offset = (np.array([float(o[0]) for o in offs]), np.array([float(o[1]) for o in offs]))
        else:
            offset = (float(self._offset[0]), float(self._offset[1]))
        fr = self._flux_ratio
        if isinstance(fr, SED):
            fr = np.asarray(fr(waves), dtype=float)
        elif _is_chromatic_callable(fr):
            fr = np.array([float(fr(float(w))) for w in waves])
        return Transformation(ret, jac=jac, offset=offset, flux_ratio=fr, gsparams=self._gsparams,
                              propagate_gsparams=self._propagate_gsparams)

    def __repr__(self):
        return 'galsim.ChromaticTransformation(%r, jac=%r, offset=%r, flux_ratio=%r)' % (
            self._original, self._jac, self._offset, self._flux_ratio)


class SimpleChromaticTransformation(ChromaticTransformation):
    """GSObject * SED: a separable profile (chromatic.py:2208-2312)."""

    def __init__(self, obj, sed=1., gsparams=None, propagate_gsparams=True):
        self.chromatic = False
        self.separable = True
        self.interpolated = False
        self.deinterpolated = self
        self._redshift = None
        self._gsparams = GSParams.check(gsparams, obj.gsparams)
        self._propagate_gsparams = propagate_gsparams
        self._original = obj
        self._jac = None
        self._offset = np.array([0., 0.])
        self._flux_ratio = sed
        if self._propagate_gsparams:
            self._original = self._original.withGSParams(self._gsparams)

    @property
    def sed(self):
        flux = self._original.flux
        if np.ndim(flux) > 0:
            # a batch of galaxies sharing the SED: the flux stays with the batched profile
            return self._flux_ratio
        return self._flux_ratio * float(flux)

    def _getTransformations(self, wave):
        return self._jac, self._offset, self._flux_ratio(wave)

    def __repr__(self):
        return 'galsim.SimpleChromaticTransformation(%r, sed=%r)' % (self._original, self._flux_ratio)


def _Transform(obj, jac=None, offset=(0., 0.), flux_ratio=1., gsparams=None, propagate_gsparams=True):
    """transform.Transform for chromatic arguments (transform.py:40-110)."""
    from .compound import Transformation
    off_callable = _is_chromatic_callable(offset)
    if (isinstance(obj, (GSObject, SimpleChromaticTransformation)) and not _is_chromatic_callable(jac)
            and not off_callable):
        if isinstance(obj, GSObject):
            if not _is_chromatic_callable(flux_ratio):
                return Transformation(obj, jac, offset, flux_ratio, gsparams, propagate_gsparams)
            if jac is None and tuple(np.asarray(offset, float)) == (0., 0.):
                if not isinstance(flux_ratio, SED):
                    flux_ratio = SED(flux_ratio, 'nm', '1')
                return SimpleChromaticTransformation(obj, flux_ratio, gsparams=gsparams,
                                                     propagate_gsparams=propagate_gsparams)
            return ChromaticTransformation(obj, jac, offset, flux_ratio, gsparams=gsparams,
                                           propagate_gsparams=propagate_gsparams)
        if not _is_chromatic_callable(flux_ratio):
            new_obj = Transformation(obj.original, jac, offset, flux_ratio, gsparams, propagate_gsparams)
            return SimpleChromaticTransformation(new_obj, obj._flux_ratio, gsparams=gsparams,
                                                 propagate_gsparams=propagate_gsparams)
    return ChromaticTransformation(obj, jac, offset, flux_ratio, gsparams=gsparams,
                                   propagate_gsparams=propagate_gsparams)


class ChromaticAtmosphere(ChromaticObject):
    """Atmospheric PSF with differential chromatic refraction and seeing proportional to
    wavelength^alpha (chromatic.py:1602-1785): base_obj at base_wavelength, dilated by
    (wave / base_wavelength)^alpha and shifted along the parallactic angle by the refraction
    relative to base_wavelength (in scale_unit, arcsec by default)."""

    def __init__(self, base_obj, base_wavelength, scale_unit=None, **kwargs):
        self.base_obj = base_obj
        self.base_wavelength = base_wavelength
        self._gsparams = base_obj.gsparams
        if scale_unit is None:
            scale_unit = arcsec
        elif isinstance(scale_unit, str):
            scale_unit = AngleUnit.from_name(scale_unit)
        self.scale_unit = scale_unit
        self.alpha = kwargs.pop('alpha', -0.2)
        self.zenith_angle, self.parallactic_angle, self.kw = dcr.parse_dcr_angles(**kwargs)
        for kw in self.kw:
            if kw not in ('temperature', 'pressure', 'H2O_pressure'):
                raise TypeError("Got unexpected keyword: {0}".format(kw))
        self.base_refraction = dcr.get_refraction(self.base_wavelength, self.zenith_angle, **self.kw)
        self.separable = False
        self.interpolated = False
        self.deinterpolated = self

    sed = property(lambda self: self.base_obj.sed)
    gsparams = property(lambda self: self.base_obj.gsparams)

    def withGSParams(self, gsparams=None, **kwargs):
        if gsparams == self.gsparams and not kwargs:
            return self
        ret = copy.copy(self)
        ret.base_obj = self.base_obj.withGSParams(gsparams, **kwargs)
        return ret

    def build_obj(self):
        """The ChromaticTransformation of base_obj (chromatic.py:1734-1757)."""
        def shift_fn(w):
            shift_magnitude = dcr.get_refraction(w, self.zenith_angle, **self.kw)
            shift_magnitude -= self.base_refraction
            # (x radians) / scale_unit in the reference's Angle arithmetic
            shift_magnitude = shift_magnitude * 1.0 / self.scale_unit.value
            sinp, cosp = self.parallactic_angle.sincos()
            return (-shift_magnitude * sinp, shift_magnitude * cosp)

        def jac_fn(w):
            scale = (w / self.base_wavelength) ** self.alpha
            return np.diag([scale, scale])

        flux_ratio = lambda w: (w / self.base_wavelength) ** (-2. * self.alpha)
        return ChromaticTransformation(self.base_obj, jac=jac_fn, offset=shift_fn, flux_ratio=flux_ratio)

    def evaluateAtWavelength(self, wave):
        return self.build_obj().evaluateAtWavelength(wave)

    def _evaluate_batch(self, waves):
        return self.build_obj()._evaluate_batch(waves)

    def __repr__(self):
        return 'galsim.ChromaticAtmosphere(%r, base_wavelength=%r, alpha=%r)' % (
            self.base_obj, self.base_wavelength, self.alpha)


class ChromaticAiry(ChromaticObject):
    """An Airy PSF whose diffraction limit scales with wavelength (chromatic.py:3765-3885): at
    wavelength w, Airy(lam_over_diam * w / lam) with the other Airy arguments (flux, obscuration)
    unchanged; the fiducial lam_over_diam is given, or (1e-9 lam / diam) radians in scale_unit."""

    def __init__(self, lam, diam=None, lam_over_diam=None, scale_unit=None, gsparams=None, **kwargs):
        from .angle import radians
        if scale_unit is None:
            scale_unit = arcsec
        elif isinstance(scale_unit, str):
            scale_unit = AngleUnit.from_name(scale_unit)
        self.scale_unit = scale_unit
        self._gsparams = GSParams.check(gsparams)
        if (diam is None) == (lam_over_diam is None):
            raise GalSimIncompatibleValuesError(
                "Need to specify telescope diameter OR wavelength/diam ratio",
                diam=diam, lam_over_diam=lam_over_diam)
        if diam is not None:
            self.lam_over_diam = (1.e-9 * lam / diam) * (radians / self.scale_unit)
        else:
            self.lam_over_diam = float(lam_over_diam)
        self.lam = float(lam)
        self.kwargs = kwargs
        self.separable = False
        self.interpolated = False
        self.deinterpolated = self

    @property
    def sed(self):
        return SED(1, 'nm', '1')

    gsparams = property(lambda self: self._gsparams)

    def withGSParams(self, gsparams=None, **kwargs):
        if gsparams == self.gsparams and not kwargs:
            return self
        ret = copy.copy(self)
        ret._gsparams = GSParams.check(gsparams, self.gsparams, **kwargs)
        return ret

    def _airy(self, lod):
        from .profiles import Airy
        return Airy(lam_over_diam=lod, scale_unit=self.scale_unit, gsparams=self.gsparams, **self.kwargs)

    def evaluateAtWavelength(self, wave):
        return self._airy(self.lam_over_diam * (wave / self.lam))

    def _evaluate_batch(self, waves):
        return self._airy(self.lam_over_diam * (np.asarray(waves, dtype=float) / self.lam))

    def __eq__(self, other):
        return (self is other or
                (isinstance(other, ChromaticAiry) and self.lam == other.lam and
                 self.lam_over_diam == other.lam_over_diam and self.scale_unit == other.scale_unit and
                 self.gsparams == other.gsparams and self.kwargs == other.kwargs))

    def __hash__(self):
        return hash(("galsim.ChromaticAiry", self.lam, self.lam_over_diam, self.scale_unit,
                     self.gsparams, frozenset(self.kwargs.items())))

    def __repr__(self):
        return 'galsim.ChromaticAiry(lam=%r, lam_over_diam=%r)' % (self.lam, self.lam_over_diam)


class ChromaticSum(ChromaticObject):
    """Sum of chromatic (and achromatic) profiles (chromatic.py:2315-2613)."""

    def __init__(self, *args, **kwargs):
        gsparams = kwargs.pop("gsparams", None)
        self._propagate_gsparams = kwargs.pop("propagate_gsparams", True)
        if kwargs:
            raise TypeError("Got unexpected keyword argument(s): %s" % kwargs.keys())
        if len(args) == 0:
            raise TypeError("Must provide at least one GSObject or ChromaticObject.")
        if len(args) == 1:
            if isinstance(args[0], (GSObject, ChromaticObject)):
                args = [args[0]]
            elif isinstance(args[0], list):
                args = args[0]
            else:
                raise TypeError("Single input argument must be a GSObject, a ChromaticObject, or list of them.")
        self._gsparams = (GSParams.combine([obj.gsparams for obj in args]) if gsparams is None
                          else GSParams.check(gsparams))
        dimensionless = all(a.dimensionless for a in args)
        spectral = all(a.spectral for a in args)
        if not (dimensionless or spectral):
            raise GalSimIncompatibleValuesError("Cannot add dimensionless and spectral ChromaticObjects.",
                                                args=args)
        self.separable = False
        self.interpolated = False
        self.deinterpolated = self
        self._obj_list = []
        for obj in args:
            if self._propagate_gsparams:
                obj = obj.withGSParams(self._gsparams)
            self._obj_list.append(obj)

    obj_list = property(lambda self: self._obj_list)
    gsparams = property(lambda self: self._gsparams)

    @property
    def sed(self):
        sed = self._obj_list[0].sed
        for obj in self._obj_list[1:]:
            sed = sed + obj.sed
        return sed

    def withGSParams(self, gsparams=None, **kwargs):
        if gsparams == self.gsparams and not kwargs:
            return self
        ret = copy.copy(self)
        ret._gsparams = GSParams.check(gsparams, self.gsparams, **kwargs)
        if self._propagate_gsparams:
            ret._obj_list = [obj.withGSParams(ret._gsparams) for obj in self._obj_list]
        return ret

    def evaluateAtWavelength(self, wave):
        from .compound import Add
        return Add([obj.evaluateAtWavelength(wave) for obj in self._obj_list], gsparams=self._gsparams,
                   propagate_gsparams=self._propagate_gsparams)

    def _evaluate_batch(self, waves):
        from .compound import Add
        return Add([_evaluate_batch(obj, waves) for obj in self._obj_list], gsparams=self._gsparams,
                   propagate_gsparams=self._propagate_gsparams)

    def drawImage(self, bandpass, image=None, integrator='quadratic', **kwargs):
        """Each summand drawn in turn onto the image (chromatic.py:2504-2560)."""
        if self.sed.dimensionless:
            raise GalSimSEDError("Can only draw ChromaticObjects with spectral SEDs.", self.sed)
        add_to_image = kwargs.pop('add_to_image', False)
        image = self._obj_list[0].drawImage(bandpass, image=image, integrator=integrator,
                                            add_to_image=add_to_image, **kwargs)
        _remove_setup_kwargs(kwargs)
        added_flux = image.added_flux
        for obj in self._obj_list[1:]:
            image = obj.drawImage(bandpass, image=image, integrator=integrator, add_to_image=True, **kwargs)
            added_flux += image.added_flux
        image.added_flux = added_flux
        return image


class ChromaticConvolution(ChromaticObject):
    """Convolution of chromatic (and achromatic) profiles (chromatic.py:2616-3055)."""

    def __init__(self, *args, **kwargs):
        if len(args) == 0:
            raise TypeError("Must provide at least one GSObject or ChromaticObject")
        if len(args) == 1:
            if isinstance(args[0], (GSObject, ChromaticObject)):
                args = [args[0]]
            elif isinstance(args[0], list):
                args = args[0]
            else:
                raise TypeError("Single input argument must be a GSObject, or a ChromaticObject, or list of them.")
        if kwargs.pop("real_space", None):
            raise GalSimNotImplementedError("Real space convolution of chromatic objects not implemented.")
        gsparams = kwargs.pop("gsparams", None)
        self._propagate_gsparams = kwargs.pop("propagate_gsparams", True)
        self._gsparams = (GSParams.combine([obj.gsparams for obj in args]) if gsparams is None
                          else GSParams.check(gsparams))
        if kwargs:
            raise TypeError("Got unexpected keyword argument(s): %s" % kwargs.keys())
        if sum(arg.spectral for arg in args) > 1:
            raise GalSimIncompatibleValuesError("Cannot convolve more than one spectral ChromaticObject.",
                                                args=args)
        self._obj_list = []
        for obj in args:
            if self._propagate_gsparams:
                obj = obj.withGSParams(self._gsparams)
            if isinstance(obj, ChromaticConvolution):
                self._obj_list.extend(obj.obj_list)
            else:
                self._obj_list.append(obj)
        self.separable = all(obj.separable for obj in self._obj_list)
        self.interpolated = False
        self.deinterpolated = self

    obj_list = property(lambda self: self._obj_list)
    gsparams = property(lambda self: self._gsparams)

    @property
    def sed(self):
        sed = self._obj_list[0].sed
        for obj in self._obj_list[1:]:
            sed = sed * obj.sed
        return sed

    def withGSParams(self, gsparams=None, **kwargs):
        if gsparams == self.gsparams and not kwargs:
            return self
        ret = copy.copy(self)
        ret._gsparams = GSParams.check(gsparams, self.gsparams, **kwargs)
        if self._propagate_gsparams:
            ret._obj_list = [obj.withGSParams(ret._gsparams) for obj in self._obj_list]
        return ret

    def evaluateAtWavelength(self, wave):
        from .compound import Convolve
        return Convolve([obj.evaluateAtWavelength(wave) for obj in self._obj_list], gsparams=self._gsparams,
                        propagate_gsparams=self._propagate_gsparams)

    def _approxWavelength(self, wave):
        from .compound import Convolve
        achrom = []
        for k, obj in enumerate(self._obj_list):
            new_wave, aobj = obj._approxWavelength(wave)
            if new_wave != wave:
                achrom = ([o.evaluateAtWavelength(new_wave) for o in self._obj_list[:k]] + [aobj] +
                          [o.evaluateAtWavelength(new_wave) for o in self._obj_list[k + 1:]])
                wave = new_wave
                break
            achrom.append(aobj)
        return wave, Convolve(achrom, gsparams=self._gsparams, propagate_gsparams=self._propagate_gsparams)

    def _evaluate_batch(self, waves):
        from .compound import Convolve
        return Convolve([_evaluate_batch(obj, waves) for obj in self._obj_list], gsparams=self._gsparams,
                        propagate_gsparams=self._propagate_gsparams)

    @staticmethod
    def _get_effective_prof(insep_obj, bandpass, iimult, integrator, gsparams, precision='fp32'):
        """The inseparable factors (times the galaxy SED) integrated over the bandpass, as an
        InterpolatedImage of their image at half the Nyquist scale (chromatic.py:2752-2779)."""
        from .interpolatedimage import InterpolatedImage
        _, prof0 = insep_obj._fiducial_profile(bandpass)
        prof1 = insep_obj.evaluateAtWavelength(bandpass.red_limit)
        prof2 = insep_obj.evaluateAtWavelength(bandpass.blue_limit)
        iiscale = min(prof0.nyquist_scale, prof1.nyquist_scale, prof2.nyquist_scale)
        iiscale /= 2
        if iimult is not None:
            iiscale /= iimult
        if isinstance(insep_obj, ChromaticConvolution):
            img = ChromaticObject.drawImage(insep_obj, bandpass, scale=iiscale, integrator=integrator,
                                            method='no_pixel', precision=precision)
        else:
            img = insep_obj.drawImage(bandpass, scale=iiscale, integrator=integrator, method='no_pixel',
                                      precision=precision)
        return InterpolatedImage(img, gsparams=gsparams)

    def drawImage(self, bandpass, image=None, integrator='quadratic', iimult=None, **kwargs):
        """chromatic.py:2852-3030 (the drawImage path without photon shooting)."""
        from .compound import Convolve
        if self.sed.dimensionless:
            raise GalSimSEDError("Can only draw ChromaticObjects with spectral SEDs.", self.sed)
        if self.separable:
            return ChromaticObject.drawImage(self, bandpass, image=image, integrator=integrator, **kwargs)
        if kwargs.get('method', 'auto') == 'phot':
            raise GalSimNotImplementedError("photon shooting is not built")
        # distribute sums: int((g1 h1 + g2 h2) * f3) -> g1 * int(h1 f3) + g2 * int(h2 f3)
        for i, obj in enumerate(self._obj_list):
            if isinstance(obj, ChromaticSum):
                tmplist = list(self._obj_list)
                del tmplist[i]
                tmplist.append(obj.obj_list[0])
                add_to_image = kwargs.pop('add_to_image', False)
                image = ChromaticConvolution(tmplist).drawImage(bandpass, image=image, integrator=integrator,
                                                                iimult=iimult, add_to_image=add_to_image,
                                                                **kwargs)
                for summand in obj.obj_list[1:]:
                    tmplist = list(self._obj_list)
                    del tmplist[i]
                    tmplist.append(summand)
                    _remove_setup_kwargs(kwargs)
                    image = ChromaticConvolution(tmplist).drawImage(bandpass, image=image, integrator=integrator,
                                                                    iimult=iimult, add_to_image=True, **kwargs)
                # (image.added_flux is the last summand's, as in the reference)
                return image
        precision = kwargs.pop('precision', 'fp32')
        wave0, prof0 = self._fiducial_profile(bandpass)
        image = prof0.drawImage(image=image, setup_only=True, **kwargs)
        _remove_setup_kwargs(kwargs)
        insep = [obj for obj in self._obj_list if not obj.separable]
        insep_obj = insep[0] if len(insep) == 1 else ChromaticConvolution(
            insep, gsparams=self._gsparams, propagate_gsparams=self._propagate_gsparams)
        sep_profs = []
        for obj in self._obj_list:
            if not obj.separable:
                continue
            wave0, p0 = obj._fiducial_profile(bandpass)
            sep_profs.append(p0 / obj.sed(wave0))
            insep_obj = insep_obj * obj.sed
        effective_prof = ChromaticConvolution._get_effective_prof(insep_obj, bandpass, iimult, integrator,
                                                                  self._gsparams, precision)
        sep_profs.append(effective_prof)
        final_prof = Convolve(sep_profs, gsparams=self._gsparams, propagate_gsparams=self._propagate_gsparams)
        return final_prof.drawImage(image=image, precision=precision, **kwargs)


def _batch_terms(obj):
    """The terms of a chromatic batch: ChromaticSums distributed over the convolution, as
    ChromaticConvolution.drawImage distributes them (chromatic.py:2935-2975)."""
    if isinstance(obj, ChromaticSum):
        out = []
        for o in obj.obj_list:
            out.extend(_batch_terms(o))
        return out
    if isinstance(obj, ChromaticConvolution):
        for i, o in enumerate(obj.obj_list):
            if isinstance(o, ChromaticSum):
                out = []
                for summand in o.obj_list:
                    tmp = list(obj.obj_list)
                    del tmp[i]
                    tmp.append(summand)
                    out.extend(_batch_terms(ChromaticConvolution(tmp)))
                return out
    return [obj]


def _batch_term_profile(term, bandpass, integrator, precision):
    """The achromatic (batched) profile whose draw is the term's chromatic draw: the fiducial
    profile scaled by the SED x throughput integral for a separable term (chromatic.py:483-487),
    the separable factors convolved with the effective PSF for a convolution with inseparable
    factors (chromatic.py:2999-3030).  The effective PSF, which depends only on the PSF, the
    galaxy SED and the bandpass, is integrated once for the whole batch."""
    from .compound import Convolve
    if term.sed.dimensionless:
        raise GalSimSEDError("Can only draw ChromaticObjects with spectral SEDs.", term.sed)
    if term.separable:
        wave0, prof0 = term._fiducial_profile(bandpass)
        wave_list, _, _ = combine_wave_list(term, bandpass)
        return prof0 * (_get_multiplier(term.sed, bandpass, tuple(wave_list)) / term.sed(wave0))
    if not isinstance(term, ChromaticConvolution):
        raise GalSimNotImplementedError("batched drawing of a chromatic %s that is not a convolution with "
                                        "separable galaxy terms is not built" % type(term).__name__)
    insep = [o for o in term.obj_list if not o.separable]
    insep_obj = insep[0] if len(insep) == 1 else ChromaticConvolution(
        insep, gsparams=term._gsparams, propagate_gsparams=term._propagate_gsparams)
    sep = []
    for o in term.obj_list:
        if o.separable:
            wave0, p0 = o._fiducial_profile(bandpass)
            sep.append(p0 / o.sed(wave0))
            insep_obj = insep_obj * o.sed
    eff = ChromaticConvolution._get_effective_prof(insep_obj, bandpass, None, integrator, term._gsparams,
                                                   precision)
    return Convolve(sep + [eff], gsparams=term._gsparams, propagate_gsparams=term._propagate_gsparams)


def draw_batch_chromatic(obj, bandpass, nx, ny, scale, dtype=np.float32, method='auto', area=1., exptime=1.,
                         gain=1., offset=None, use_true_center=True, precision='fp32', integrator='quadratic'):
    """A batch of chromatic objects drawn through a bandpass: galaxies whose spatial profiles
    are batched GSObjects times one SED per term, convolved with chromatic (or achromatic)
    PSFs shared by the batch.  Stamp i is what ``obj_i.drawImage(bandpass, nx=nx, ny=ny,
    scale=scale, ...)`` draws: each term's effective PSF is integrated once (one batched draw
    of its wavelengths) and the terms' batched profiles are drawn with draw_batch, their stamps
    summed on the device.  added_flux is the sum over the terms."""
    from .batch import draw_batch
    if nx is None or ny is None:
        raise GalSimIncompatibleValuesError("batched chromatic drawing needs fixed nx, ny", nx=nx, ny=ny)
    out = None
    flux = None
    for term in _batch_terms(obj):
        prof = _batch_term_profile(term, bandpass, integrator, precision)
        st = draw_batch(prof, nx=nx, ny=ny, scale=scale, dtype=dtype, method=method, area=area,
                        exptime=exptime, gain=gain, offset=offset, use_true_center=use_true_center,
                        precision=precision)
        if out is None:
            out = st
            flux = st._flux_dev.clone()
        else:
            if len(st) != len(out) and len(out) == 1:
                raise GalSimIncompatibleValuesError("the terms of a chromatic batch have different batch sizes")
            out.flat += st.flat
            flux += st._flux_dev
    out._flux_dev = flux
    return out

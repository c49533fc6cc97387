"""Leaf profiles: Gaussian, Exponential, Sersic (+ DeVaucouleurs), Moffat, Kolmogorov, Airy.

Front-ends with the reference's constructors, size conversions and errors
(gaussian.py:60-183, exponential.py:60-164, sersic.py:196-373, moffat.py:76-231,
kolmogorov.py:163-313, airy.py:98-249).  Their Fourier transforms, stepk and maxk are
evaluated on the GPU (galsim_b200/csrc/gsb_profiles.cuh, gsb_tables.cu).  Any size or flux
parameter may be a numpy array, which makes the object a batch of profiles.
"""
import math

import numpy as np

from . import _lib
from .angle import AngleUnit, arcsec, radians
from .errors import GalSimIncompatibleValuesError, GalSimRangeError
from .gsobject import GSObject, _as_param, _plen
from .gsparams import GSParams


class _Leaf(GSObject):
    _is_analytic_x = True
    _is_analytic_k = True

    def _flatten(self, bld, jac):
        bld.add_leaf(self._type, jac, self._flux, self._params(), self._leaf_flags())

    def _leaf_flags(self):
        return 0

    def __getstate__(self):
        d = self.__dict__.copy()
        d.pop('_cached_sizes', None)
        return d

    def __setstate__(self, d):
        self.__dict__ = d

    def __ne__(self, other):
        return not self.__eq__(other)


def _eq(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b))


class Gaussian(_Leaf):
    """exp(-r^2 / 2 sigma^2) (gaussian.py:60-183)."""
    _fwhm_factor = 2.3548200450309493
    _hlr_factor = 1.1774100225154747
    _is_axisymmetric = True
    _type = _lib.GAUSSIAN

    def __init__(self, half_light_radius=None, sigma=None, fwhm=None, flux=1., gsparams=None):
        if fwhm is not None:
            if sigma is not None or half_light_radius is not None:
                raise GalSimIncompatibleValuesError(
                    "Only one of sigma, fwhm, and half_light_radius may be specified",
                    fwhm=fwhm, sigma=sigma, half_light_radius=half_light_radius)
            sigma = _as_param(fwhm) / Gaussian._fwhm_factor
        elif half_light_radius is not None:
            if sigma is not None:
                raise GalSimIncompatibleValuesError(
                    "Only one of sigma, fwhm, and half_light_radius may be specified",
                    fwhm=fwhm, sigma=sigma, half_light_radius=half_light_radius)
            sigma = _as_param(half_light_radius) / Gaussian._hlr_factor
        elif sigma is None:
            raise GalSimIncompatibleValuesError(
                "One of sigma, fwhm, and half_light_radius must be specified",
                fwhm=fwhm, sigma=sigma, half_light_radius=half_light_radius)
        self._sigma = _as_param(sigma)
        self._flux = _as_param(flux)
        self._gsparams = GSParams.check(gsparams)
        self._batch = _plen(self._sigma, self._flux)

    sigma = property(lambda self: self._sigma)
    half_light_radius = property(lambda self: self._sigma * Gaussian._hlr_factor)
    fwhm = property(lambda self: self._sigma * Gaussian._fwhm_factor)

    def _params(self):
        return (self._sigma,)

    def withFlux(self, flux):
        return Gaussian(sigma=self.sigma, flux=flux, gsparams=self.gsparams)

    def __eq__(self, other):
        return self is other or (isinstance(other, Gaussian) and _eq(self.sigma, other.sigma) and
                                 _eq(self.flux, other.flux) and self.gsparams == other.gsparams)

    def __hash__(self):
        return hash(("galsim.Gaussian", str(self.sigma), str(self.flux), self.gsparams))

    def __repr__(self):
        return 'galsim.Gaussian(sigma=%r, flux=%r, gsparams=%r)' % (self.sigma, self.flux, self.gsparams)


class Exponential(_Leaf):
    """exp(-r / r0) (exponential.py:60-164)."""
    _hlr_factor = 1.6783469900166605
    _is_axisymmetric = True
    _type = _lib.EXPONENTIAL

    def __init__(self, half_light_radius=None, scale_radius=None, flux=1., gsparams=None):
        if half_light_radius is not None:
            if scale_radius is not None:
                raise GalSimIncompatibleValuesError(
                    "Only one of scale_radius and half_light_radius may be specified",
                    half_light_radius=half_light_radius, scale_radius=scale_radius)
            scale_radius = _as_param(half_light_radius) / Exponential._hlr_factor
        elif scale_radius is None:
            raise GalSimIncompatibleValuesError(
                "Either scale_radius or half_light_radius must be specified",
                half_light_radius=half_light_radius, scale_radius=scale_radius)
        self._r0 = _as_param(scale_radius)
        self._flux = _as_param(flux)
        self._gsparams = GSParams.check(gsparams)
        self._batch = _plen(self._r0, self._flux)

    scale_radius = property(lambda self: self._r0)
    half_light_radius = property(lambda self: self._r0 * Exponential._hlr_factor)

    def _params(self):
        return (self._r0,)

    def withFlux(self, flux):
        return Exponential(scale_radius=self.scale_radius, flux=flux, gsparams=self.gsparams)

    def __eq__(self, other):
        return self is other or (isinstance(other, Exponential) and
                                 _eq(self.scale_radius, other.scale_radius) and
                                 _eq(self.flux, other.flux) and self.gsparams == other.gsparams)

    def __hash__(self):
        return hash(("galsim.Exponential", str(self.scale_radius), str(self.flux), self.gsparams))

    def __repr__(self):
        return 'galsim.Exponential(scale_radius=%r, flux=%r, gsparams=%r)' % (
            self.scale_radius, self.flux, self.gsparams)


class Sersic(_Leaf):
    """exp(-(r/r0)^(1/n)) (sersic.py:196-373).  The FT is a per-n FP64 Hankel table built on
    the GPU; half_light_radius -> scale_radius uses the same table build (Brent in FP64).
    trunc > 0 truncates the profile there: without flux_untruncated, flux and half_light_radius
    refer to the truncated profile (its scale radius from SersicTruncatedScale), with it to the
    untruncated one (the flux then scaled by the fraction inside trunc), sersic.py:218-247; the
    sizes come from an FP64 root find on the GPU and the table from the truncated Hankel
    transform."""
    _minimum_n = 0.3
    _maximum_n = 6.2
    _is_axisymmetric = True
    _type = _lib.SERSIC

    def __init__(self, n, half_light_radius=None, scale_radius=None,
                 flux=1., trunc=0., flux_untruncated=False, gsparams=None):
        self._n = _as_param(n)
        self._flux = _as_param(flux)
        self._trunc = _as_param(trunc)
        self._flux_untruncated = bool(flux_untruncated)
        self._gsparams = GSParams.check(gsparams)
        if np.any(np.asarray(self._n) < Sersic._minimum_n):
            raise GalSimRangeError("Requested Sersic index is too small",
                                   self._n, Sersic._minimum_n, Sersic._maximum_n)
        if np.any(np.asarray(self._n) > Sersic._maximum_n):
            raise GalSimRangeError("Requested Sersic index is too large",
                                   self._n, Sersic._minimum_n, Sersic._maximum_n)
        if np.any(np.asarray(self._trunc) < 0):
            raise GalSimRangeError("Sersic trunc must be > 0", self._trunc, 0.)
        if half_light_radius is not None:
            if scale_radius is not None:
                raise GalSimIncompatibleValuesError(
                    "Only one of scale_radius or half_light_radius may be specified for Spergel",
                    half_light_radius=half_light_radius, scale_radius=scale_radius)
            self._hlr = _as_param(half_light_radius)
            self._r0 = None
        elif scale_radius is not None:
            self._r0 = _as_param(scale_radius)
            self._hlr = None
        else:
            raise GalSimIncompatibleValuesError(
                "Either scale_radius or half_light_radius must be specified for Spergel",
                half_light_radius=half_light_radius, scale_radius=scale_radius)
        self._flux_fraction = 1.
        truncated = np.any(np.asarray(self._trunc) > 0)
        if truncated:
            if not np.all(np.asarray(self._trunc) > 0):
                raise GalSimIncompatibleValuesError("a batch of Sersic profiles is either truncated "
                                                    "or not", trunc=self._trunc)
            if self._hlr is not None and not self._flux_untruncated and \
                    np.any(np.asarray(self._trunc) <= math.sqrt(2.) * np.asarray(self._hlr)):
                raise GalSimRangeError("Sersic trunc must be > sqrt(2) * half_light_radius",
                                       self._trunc, math.sqrt(2.) * np.asarray(self._hlr))
            size = self._hlr if self._hlr is not None else self._r0
            r0, ff = _lib.sersic_truncation(self._n, size, self._trunc, self._hlr is not None,
                                            self._flux_untruncated)
            scalar = np.ndim(self._n) == 0 and np.ndim(size) == 0 and np.ndim(self._trunc) == 0
            self._r0 = float(r0[0]) if scalar else r0
            self._flux_fraction = float(ff[0]) if scalar else ff
            if self._flux_untruncated:
                self._flux = self._flux * self._flux_fraction
                self._hlr = None          # the truncated profile's, computed when asked for
        self._batch = _plen(self._n, self._flux, self._hlr if self._hlr is not None else self._r0,
                            self._trunc)

    n = property(lambda self: self._n)
    trunc = property(lambda self: self._trunc)
    # a truncated profile has a hard edge (sersic.py:338-340)
    _has_hard_edges = property(lambda self: bool(np.any(np.asarray(self._trunc) > 0.)))

    def calculateHLRFactor(self):
        """Half-light radius in units of the scale radius (SersicHLR, SBSersic.cpp:660-667),
        computed on the GPU (of the truncated profile when truncated)."""
        n = np.atleast_1d(self._n)
        t = np.broadcast_to(np.atleast_1d(np.asarray(self._trunc, float)), n.shape)
        r0 = np.broadcast_to(np.atleast_1d(np.asarray(self._r0, float)), n.shape) if self._r0 is not None else None
        tr = (t / r0) if (r0 is not None and np.any(t > 0)) else np.zeros_like(n)
        uniq, inv = np.unique(np.stack([n, tr], -1), axis=0, return_inverse=True)
        tabs = _lib.Tables()
        tabs.build_sersic(uniq[:, 0], self.gsparams, trunc_over_r0=uniq[:, 1] if np.any(uniq[:, 1] > 0) else None)
        re = tabs.sersic_info()[:, _lib.SH_RE][np.asarray(inv).reshape(-1)]
        return float(re[0]) if np.ndim(self._n) == 0 and re.size == 1 else re

    @property
    def scale_radius(self):
        if self._r0 is None:
            self._r0 = self._hlr / self.calculateHLRFactor()
        return self._r0

    @property
    def half_light_radius(self):
        if self._hlr is None:
            self._hlr = self._r0 * self.calculateHLRFactor()
        return self._hlr

    def _params(self):
        if self._hlr is not None and self._r0 is None:
            return (self._n, self._hlr, 0.)
        return (self._n, self._r0, self._trunc)

    def _leaf_flags(self):
        return _lib.LEAF_SIZE_IS_HLR if (self._hlr is not None and self._r0 is None) else 0

    def withFlux(self, flux):
        if np.any(np.asarray(self._trunc) > 0):
            return Sersic(n=self.n, scale_radius=self._r0, flux=flux, trunc=self._trunc, gsparams=self.gsparams)
        if self._r0 is None:
            return Sersic(n=self.n, half_light_radius=self._hlr, flux=flux, gsparams=self.gsparams)
        return Sersic(n=self.n, scale_radius=self._r0, flux=flux, gsparams=self.gsparams)

    def __eq__(self, other):
        return self is other or (isinstance(other, Sersic) and _eq(self.n, other.n) and
                                 _eq(self.scale_radius, other.scale_radius) and
                                 _eq(self.trunc, other.trunc) and _eq(self.flux, other.flux) and
                                 self.gsparams == other.gsparams)

    def __hash__(self):
        return hash(("galsim.Sersic", str(self.n), str(self._hlr), str(self._r0), str(self.flux),
                     self.gsparams))

    def __repr__(self):
        size = ('half_light_radius=%r' % self._hlr) if self._r0 is None else ('scale_radius=%r' % self._r0)
        return 'galsim.Sersic(n=%r, %s, flux=%r, gsparams=%r)' % (self.n, size, self.flux, self.gsparams)


class DeVaucouleurs(Sersic):
    """Sersic with n = 4 (sersic.py:376-427)."""

    def __init__(self, half_light_radius=None, scale_radius=None, flux=1., trunc=0.,
                 flux_untruncated=False, gsparams=None):
        super(DeVaucouleurs, self).__init__(n=4, half_light_radius=half_light_radius,
                                            scale_radius=scale_radius, flux=flux, trunc=trunc,
                                            flux_untruncated=flux_untruncated, gsparams=gsparams)


class Moffat(_Leaf):
    """(1 + (r/r0)^2)^-beta (moffat.py:76-231).  trunc > 0 truncates the profile there
    (beta <= 1.1 needs it): the FT then comes from an FP64 table of the truncated Hankel
    transform built on the GPU per (beta, trunc / scale_radius), and a half_light_radius of a
    truncated profile gives the scale radius by an FP64 root find on the GPU.  A batch may mix
    truncated and untruncated profiles."""
    _is_axisymmetric = True
    _type = _lib.MOFFAT

    def __init__(self, beta, scale_radius=None, half_light_radius=None, fwhm=None, trunc=0.,
                 flux=1., gsparams=None):
        self._beta = _as_param(beta)
        self._trunc = _as_param(trunc)
        self._flux = _as_param(flux)
        self._gsparams = GSParams.check(gsparams)
        beta = np.asarray(self._beta, float)
        trunc = np.asarray(self._trunc, float)
        bb, tt = np.broadcast_arrays(beta, trunc)
        if np.any((bb <= 1.1) & (tt == 0.)):
            raise GalSimRangeError("Moffat profiles with beta <= 1.1 must be truncated", self._beta, 1.1)
        if np.any(trunc < 0.):
            raise GalSimRangeError("Moffat trunc must be >= 0", self._trunc, 0.)
        if half_light_radius is not None:
            if scale_radius is not None or fwhm is not None:
                raise GalSimIncompatibleValuesError(
                    "Only one of scale_radius, half_light_radius, or fwhm may be specified",
                    half_light_radius=half_light_radius, scale_radius=scale_radius, fwhm=fwhm)
            self._hlr = _as_param(half_light_radius)
            hlr = np.asarray(self._hlr, float)
            if np.any((trunc > 0.) & (trunc <= math.sqrt(2.) * hlr)):
                raise GalSimRangeError("Moffat trunc must be > sqrt(2) * half_light_radius.",
                                       self._trunc, math.sqrt(2.) * hlr)
            if np.any(trunc > 0.):
                # MoffatCalculateScaleRadiusFromHLR with rm = trunc (SBMoffat.cpp:128-160)
                r0 = _lib.moffat_scale_radius(self._beta, self._hlr, self._trunc)
                scalar = np.ndim(self._beta) == 0 and np.ndim(self._hlr) == 0 and np.ndim(self._trunc) == 0
                self._r0 = float(r0[0]) if scalar else r0
            else:
                # the untruncated case is analytic (SBMoffat.cpp:103-127)
                self._r0 = self._hlr / np.sqrt(np.power(0.5, 1. / (1. - self._beta)) - 1.)
                if np.ndim(self._r0) == 0:
                    self._r0 = float(self._r0)
            self._fwhm = 0.
        elif fwhm is not None:
            if scale_radius is not None:
                raise GalSimIncompatibleValuesError(
                    "Only one of scale_radius, half_light_radius, or fwhm may be specified",
                    half_light_radius=half_light_radius, scale_radius=scale_radius, fwhm=fwhm)
            self._fwhm = _as_param(fwhm)
            if np.ndim(self._fwhm) == 0 and np.ndim(self._beta) == 0:
                self._r0 = self._fwhm / (2. * math.sqrt(2. ** (1. / self._beta) - 1.))
            else:
                self._r0 = self._fwhm / (2. * np.sqrt(2. ** (1. / np.asarray(self._beta)) - 1.))
            self._hlr = 0.
        elif scale_radius is not None:
            self._r0 = _as_param(scale_radius)
            self._hlr = 0.
            self._fwhm = 0.
        else:
            raise GalSimIncompatibleValuesError(
                "One of scale_radius, half_light_radius, or fwhm must be specified",
                half_light_radius=half_light_radius, scale_radius=scale_radius, fwhm=fwhm)
        self._batch = _plen(self._beta, self._r0, self._flux, self._trunc)

    beta = property(lambda self: self._beta)
    scale_radius = property(lambda self: self._r0)
    trunc = property(lambda self: self._trunc)
    # a truncated profile has a hard edge (moffat.py:202-204)
    _has_hard_edges = property(lambda self: bool(np.any(np.asarray(self._trunc) > 0.)))

    @property
    def half_light_radius(self):
        """getHalfLightRadius (SBMoffat.cpp:246-249): rD sqrt((1 - F/2)^(1/(1-beta)) - 1) with
        F the flux fraction factor 1 - (1 + (trunc/rD)^2)^(1-beta) (1 untruncated); the given
        value when the profile was made from its half-light radius (moffat.py:144-150)."""
        if not (np.ndim(self._hlr) == 0 and self._hlr == 0.):
            return self._hlr
        beta = np.asarray(self._beta, float)
        rd = np.asarray(self._r0, float)
        t = np.asarray(self._trunc, float)
        with np.errstate(divide='ignore', invalid='ignore'):
            ff = np.where(t > 0., 1. - np.power(1. + (t / rd) ** 2, 1. - beta), 1.)
            hlr = rd * np.sqrt(np.power(1. - 0.5 * ff, 1. / (1. - beta)) - 1.)
        return float(hlr) if np.ndim(hlr) == 0 else hlr

    @property
    def fwhm(self):
        return self._r0 * (2. * np.sqrt(2. ** (1. / np.asarray(self._beta)) - 1.))

    def _params(self):
        return (self._beta, self._r0, self._trunc)

    def withFlux(self, flux):
        return Moffat(beta=self.beta, scale_radius=self.scale_radius, trunc=self.trunc, flux=flux,
                      gsparams=self.gsparams)

    def __eq__(self, other):
        return self is other or (isinstance(other, Moffat) and _eq(self.beta, other.beta) and
                                 _eq(self.scale_radius, other.scale_radius) and
                                 _eq(self.trunc, other.trunc) and _eq(self.flux, other.flux) and
                                 self.gsparams == other.gsparams)

    def __hash__(self):
        return hash(("galsim.Moffat", str(self.beta), str(self.scale_radius), str(self.trunc), str(self.flux),
                     self.gsparams))

    def __repr__(self):
        return 'galsim.Moffat(beta=%r, scale_radius=%r, trunc=%r, flux=%r, gsparams=%r)' % (
            self.beta, self.scale_radius, self.trunc, self.flux, self.gsparams)


class Kolmogorov(_Leaf):
    """Kolmogorov turbulence PSF, FT exp(-(k/k0)^{5/3}) (kolmogorov.py:163-313)."""
    _fwhm_factor = 0.9758634299
    _hlr_factor = 0.5548101137
    _k0_factor = 2.992939911888651
    _is_axisymmetric = True
    _type = _lib.KOLMOGOROV

    def __init__(self, lam_over_r0=None, fwhm=None, half_light_radius=None, lam=None, r0=None,
                 r0_500=None, flux=1., scale_unit=None, gsparams=None):
        self._flux = _as_param(flux)
        self._gsparams = GSParams.check(gsparams)
        if fwhm is not None:
            if any(item is not None for item in (lam_over_r0, lam, r0, r0_500, half_light_radius)):
                raise GalSimIncompatibleValuesError(
                    "Only one of lam_over_r0, fwhm, half_light_radius, or lam (with r0 or r0_500) "
                    "may be specified", fwhm=fwhm, lam_over_r0=lam_over_r0, lam=lam, r0=r0,
                    r0_500=r0_500, half_light_radius=half_light_radius)
            self._lor0 = _as_param(fwhm) / Kolmogorov._fwhm_factor
        elif half_light_radius is not None:
            if any(item is not None for item in (lam_over_r0, lam, r0, r0_500)):
                raise GalSimIncompatibleValuesError(
                    "Only one of lam_over_r0, fwhm, half_light_radius, or lam (with r0 or r0_500) "
                    "may be specified", fwhm=fwhm, lam_over_r0=lam_over_r0, lam=lam, r0=r0,
                    r0_500=r0_500, half_light_radius=half_light_radius)
            self._lor0 = _as_param(half_light_radius) / Kolmogorov._hlr_factor
        elif lam_over_r0 is not None:
            if any(item is not None for item in (lam, r0, r0_500)):
                raise GalSimIncompatibleValuesError(
                    "Cannot specify lam, r0 or r0_500 in conjunction with lam_over_r0.",
                    lam_over_r0=lam_over_r0, lam=lam, r0=r0, r0_500=r0_500)
            self._lor0 = _as_param(lam_over_r0)
        else:
            if lam is None or (r0 is None and r0_500 is None):
                raise GalSimIncompatibleValuesError(
                    "One of lam_over_r0, fwhm, half_light_radius, or lam (with r0 or r0_500) "
                    "must be specified", fwhm=fwhm, lam_over_r0=lam_over_r0, lam=lam, r0=r0,
                    r0_500=r0_500, half_light_radius=half_light_radius)
            if scale_unit is None:
                scale_unit = arcsec
            elif isinstance(scale_unit, str):
                scale_unit = AngleUnit.from_name(scale_unit)
            if r0 is None:
                r0 = r0_500 * (lam / 500.) ** 1.2
            self._lor0 = (1.e-9 * float(lam) / float(r0)) * (radians / scale_unit)
        self._k0 = Kolmogorov._k0_factor / self._lor0
        self._batch = _plen(self._lor0, self._flux)

    lam_over_r0 = property(lambda self: self._lor0)
    fwhm = property(lambda self: self._lor0 * Kolmogorov._fwhm_factor)
    half_light_radius = property(lambda self: self._lor0 * Kolmogorov._hlr_factor)

    def _params(self):
        return (self._lor0,)

    def withFlux(self, flux):
        return Kolmogorov(lam_over_r0=self.lam_over_r0, flux=flux, gsparams=self.gsparams)

    def __eq__(self, other):
        return self is other or (isinstance(other, Kolmogorov) and
                                 _eq(self.lam_over_r0, other.lam_over_r0) and
                                 _eq(self.flux, other.flux) and self.gsparams == other.gsparams)

    def __hash__(self):
        return hash(("galsim.Kolmogorov", str(self.lam_over_r0), str(self.flux), self.gsparams))

    def __repr__(self):
        return 'galsim.Kolmogorov(lam_over_r0=%r, flux=%r, gsparams=%r)' % (
            self.lam_over_r0, self.flux, self.gsparams)


class Airy(_Leaf):
    """Airy pattern of a circular (optionally obscured) aperture (airy.py:98-249)."""
    _hlr_factor = 0.5348321477242647
    _fwhm_factor = 1.028993969962188
    _is_axisymmetric = True
    _type = _lib.AIRY

    def __init__(self, lam_over_diam=None, lam=None, diam=None, obscuration=0., flux=1.,
                 scale_unit=None, gsparams=None):
        self._obscuration = _as_param(obscuration)
        self._flux = _as_param(flux)
        self._gsparams = GSParams.check(gsparams)
        if lam_over_diam is not None:
            if lam is not None or diam is not None:
                raise GalSimIncompatibleValuesError(
                    "If specifying lam_over_diam, then do not specify lam or diam",
                    lam_over_diam=lam_over_diam, lam=lam, diam=diam)
            self._lod = _as_param(lam_over_diam)
        else:
            if lam is None or diam is None:
                raise GalSimIncompatibleValuesError(
                    "If not specifying lam_over_diam, then specify lam AND diam",
                    lam_over_diam=lam_over_diam, lam=lam, diam=diam)
            if isinstance(scale_unit, str):
                scale_unit = AngleUnit.from_name(scale_unit)
            elif scale_unit is None:
                scale_unit = arcsec
            self._lod = (1.e-9 * float(lam) / float(diam)) * (radians / scale_unit)
        self._batch = _plen(self._lod, self._obscuration, self._flux)

    lam_over_diam = property(lambda self: self._lod)
    obscuration = property(lambda self: self._obscuration)

    @property
    def half_light_radius(self):
        if np.all(np.asarray(self._obscuration) == 0.):
            return self._lod * Airy._hlr_factor
        from .errors import GalSimNotImplementedError
        raise GalSimNotImplementedError("Half light radius calculation not implemented for Airy "
                                        "objects with non-zero obscuration.")

    @property
    def fwhm(self):
        if np.all(np.asarray(self._obscuration) == 0.):
            return self._lod * Airy._fwhm_factor
        from .errors import GalSimNotImplementedError
        raise GalSimNotImplementedError("FWHM calculation not implemented for Airy "
                                        "objects with non-zero obscuration.")

    def _params(self):
        return (self._lod, self._obscuration)

    def withFlux(self, flux):
        return Airy(lam_over_diam=self.lam_over_diam, obscuration=self.obscuration, flux=flux,
                    gsparams=self.gsparams)

    def __eq__(self, other):
        return self is other or (isinstance(other, Airy) and
                                 _eq(self.lam_over_diam, other.lam_over_diam) and
                                 _eq(self.obscuration, other.obscuration) and
                                 _eq(self.flux, other.flux) and self.gsparams == other.gsparams)

    def __hash__(self):
        return hash(("galsim.Airy", str(self.lam_over_diam), str(self.obscuration), str(self.flux),
                     self.gsparams))

    def __repr__(self):
        return 'galsim.Airy(lam_over_diam=%r, obscuration=%r, flux=%r, gsparams=%r)' % (
            self.lam_over_diam, self.obscuration, self.flux, self.gsparams)


__all__ = ['Gaussian', 'Exponential', 'Sersic', 'DeVaucouleurs', 'Moffat', 'Kolmogorov', 'Airy']

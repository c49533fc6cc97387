"""SED: spectral energy distributions (galsim/sed.py:33-1000).

Host-side FP64 arithmetic for chromatic drawing.  An SED maps wavelength in nm (observed
frame) to photons/nm/cm^2/s (spectral SEDs) or to a dimensionless factor ('1').  Spectra are
a LookupTable, a callable of wavelength in the SED's own units, or a constant; wave_type 'nm'
or 'Angstrom'; flux_type 'fphotons', 'flambda' (erg/nm/cm^2/s), 'fnu' (erg/Hz/cm^2/s) or '1'.
Unit conversions use the exact SI values of h and c (the reference takes them from
astropy.constants).  The fast evaluation path follows the reference's: a spectrum in nm and
photons is called directly; any other is re-tabulated on its own wavelength list with the
conversion folded in (sed.py:398-417).
"""
import numpy as np

from .table import LookupTable, _LookupTable
from .errors import (GalSimValueError, GalSimRangeError, GalSimSEDError,
                     GalSimIncompatibleValuesError, GalSimNotImplementedError)

__all__ = ['SED']


def _merge_sorted(arrays):
    """utilities.merge_sorted (utilities.py:1153-1177): the sorted union of sorted arrays."""
    arrs = [np.asarray(a, dtype=float).ravel() for a in arrays]
    return np.unique(np.concatenate(arrs)) if arrs else np.array([], dtype=float)


def combine_wave_list(*args):
    """utilities.combine_wave_list (utilities.py:1179-1215): the union of the objects'
    wave_lists inside the intersection of their [blue_limit, red_limit], with both limits."""
    if len(args) == 1:
        if isinstance(args[0], (list, tuple)):
            args = args[0]
        else:
            raise TypeError("Single input argument must be a list or tuple")
    if len(args) == 0:
        return np.array([], dtype=float), 0.0, np.inf
    if len(args) == 1:
        obj = args[0]
        return obj.wave_list, getattr(obj, 'blue_limit', 0.0), getattr(obj, 'red_limit', np.inf)
    blue_limit = np.max([getattr(obj, 'blue_limit', 0.0) for obj in args])
    red_limit = np.min([getattr(obj, 'red_limit', np.inf) for obj in args])
    if blue_limit > red_limit:
        from .errors import GalSimError
        raise GalSimError("Empty wave_list intersection.")
    waves = [np.asarray(obj.wave_list) for obj in args]
    waves = [w[(blue_limit <= w) & (w <= red_limit)] for w in waves]
    if any(len(w) > 0 for w in waves):
        waves.append([blue_limit, red_limit])
    return _merge_sorted(waves), blue_limit, red_limit


class SED(object):
    """Spectral energy distribution (sed.py:33-1000); see the module docstring."""
    _h = 6.62607015e-27          # erg s
    _c = 2.99792458e17           # nm / s

    def __init__(self, spec, wave_type, flux_type, redshift=0., fast=True, interpolant='linear',
                 _blue_limit=0.0, _red_limit=np.inf, _wave_list=None):
        self._flux_type = flux_type
        self.interpolant = interpolant
        self.wave_type, self.wave_factor = self._parse_wave_type(wave_type)
        self.flux_factor = None
        if not isinstance(flux_type, str):
            raise GalSimNotImplementedError("SED flux_type must be one of 'flambda', 'fnu', 'fphotons', '1'")
        ft = flux_type.lower()
        if ft == 'flambda':
            self.flux_type = 'flambda'
            self.spectral = True
            self.flux_factor = 1. / (SED._h * SED._c)
        elif ft == 'fphotons':
            self.flux_type = 'fphotons'
            self.spectral = True
            self.flux_factor = self.wave_factor
        elif ft == 'fnu':
            self.flux_type = 'fnu'
            self.spectral = True
            self.flux_factor = self.wave_factor / SED._h
        elif flux_type == '1':
            self.flux_type = '1'
            self.spectral = False
        else:
            raise GalSimValueError("Unknown flux_type", flux_type, ('flambda', 'fnu', 'fphotons', '1'))
        self.redshift = redshift
        self.fast = fast
        self._orig_spec = spec
        self._initialize_spec()
        if _wave_list is not None:
            self.wave_list = np.asarray(_wave_list, dtype=float)
            self.blue_limit = float(_blue_limit)
            self.red_limit = float(_red_limit)
        elif isinstance(self._spec, LookupTable):
            self.wave_list = np.array(self._spec.getArgs(), dtype=float) * ((1.0 + self.redshift) / self.wave_factor)
            self.blue_limit = float(np.min(self.wave_list))
            self.red_limit = float(np.max(self.wave_list))
        else:
            self.blue_limit = 0.0
            self.red_limit = np.inf
            self.wave_list = np.array([], dtype=float)
        self._fast_spec_cache = None

    @staticmethod
    def _parse_wave_type(wave_type):
        if isinstance(wave_type, str):
            if wave_type.lower() in ('nm', 'nanometer', 'nanometers'):
                return 'nm', 1.
            if wave_type.lower() in ('a', 'ang', 'angstrom', 'angstroms'):
                return 'Angstrom', 10.
        raise GalSimValueError("Unknown wave_type", wave_type, ('nm', 'Angstrom'))

    def _initialize_spec(self):
        self._const = False
        s = self._orig_spec
        if isinstance(s, (int, float)) and not isinstance(s, bool):
            if not self.dimensionless:
                raise GalSimSEDError("Attempt to set spectral SED using float or integer.", self)
            self._const = True
            self._spec = lambda w: float(s)
        elif isinstance(s, str):
            try:
                v = float(s)
            except ValueError:
                raise GalSimNotImplementedError("SED spec strings other than a number (file names, "
                                                "expressions) are not built")
            self._const = True
            self._spec = lambda w: v
        else:
            self._spec = s

    dimensionless = property(lambda self: not self.spectral)

    # -- evaluation ---------------------------------------------------------------------------
    def _flux_to_photons(self, flux_native, wave_native):
        if self.flux_type == 'fphotons':
            return flux_native * self.flux_factor
        if self.flux_type == 'flambda':
            return flux_native * wave_native * self.flux_factor
        return flux_native / wave_native * self.flux_factor

    def _rest_nm_to_photons(self, wave):
        wave_native = np.asarray(wave) * self.wave_factor if self.wave_factor != 1 else wave
        return self._flux_to_photons(self._spec(wave_native), wave_native)

    def _rest_nm_to_dimensionless(self, wave):
        wave_native = np.asarray(wave) * self.wave_factor if self.wave_factor != 1 else wave
        return self._spec(wave_native)

    @property
    def _fast_spec(self):
        """sed.py:398-417: the spectrum as a function of rest-frame nm in photons (or the
        dimensionless factor)."""
        if self._fast_spec_cache is None:
            if self.wave_factor == 1. and self.flux_factor == 1.:
                self._fast_spec_cache = self._spec
            elif len(self.wave_list) == 0:
                self._fast_spec_cache = self._rest_nm_to_photons if self.spectral else self._rest_nm_to_dimensionless
            else:
                x = self.wave_list / (1.0 + self.redshift)
                f = self._rest_nm_to_photons(x) if self.spectral else self._rest_nm_to_dimensionless(x)
                interp = self._spec.interpolant if isinstance(self._spec, LookupTable) else 'linear'
                self._fast_spec_cache = _LookupTable(x, f, interpolant=interp)
        return self._fast_spec_cache

    def _check_bounds(self, wave):
        w = np.asarray(wave, dtype=float)
        wmin = np.min(w) if w.size else 0.
        wmax = np.max(w) if w.size else 0.
        slop = 1.e-6
        if wmin < self.blue_limit - slop:
            raise GalSimRangeError("Requested wavelength is bluer than blue_limit.",
                                   wave, self.blue_limit, self.red_limit)
        if wmax > self.red_limit + slop:
            raise GalSimRangeError("Requested wavelength is redder than red_limit.",
                                   wave, self.blue_limit, self.red_limit)

    def __call__(self, wave):
        """Photons/nm/cm^2/s (or the dimensionless value) at observed wavelength(s) in nm
        (sed.py:443-470, _call_fast)."""
        self._check_bounds(wave)
        v = self._fast_spec(np.asarray(wave, dtype=float) / (1.0 + self.redshift))
        if np.ndim(v) == 0:
            return float(v)
        return np.asarray(v, dtype=float)

    # -- arithmetic (sed.py:495-700) ----------------------------------------------------------
    def _mul_scalar(self, other, spectral):
        if isinstance(self._spec, LookupTable):
            wave_type, flux_type = self.wave_type, self._flux_type
            spec = _LookupTable(self._spec.getArgs(), np.array(self._spec.getVals()) * other,
                                interpolant=self._spec.interpolant)
        elif self._const and not spectral:
            spec = self._spec(42.0) * other
            wave_type, flux_type = 'nm', '1'
        else:
            wave_type = 'nm'
            flux_type = 'fphotons' if spectral else '1'
            fs = self._fast_spec
            spec = lambda w: fs(w) * other
        return SED(spec, wave_type, flux_type, redshift=self.redshift, fast=self.fast,
                   _blue_limit=self.blue_limit, _red_limit=self.red_limit, _wave_list=self.wave_list)

    def _mul_sed(self, other):
        redshift = self.redshift + other.redshift
        wave_list, blue_limit, red_limit = combine_wave_list(self, other)
        a, b = self._fast_spec, other._fast_spec
        if isinstance(a, LookupTable):
            x = wave_list / (1.0 + self.redshift)
            x = _merge_sorted([x, np.linspace(x[0], x[-1], 500)])
            zfactor2 = (1. + redshift) / (1. + other.redshift)
            spec = _LookupTable(x, a(x) * b(x * zfactor2), a.interpolant)
        elif isinstance(b, LookupTable):
            x = wave_list / (1.0 + other.redshift)
            x = _merge_sorted([x, np.linspace(x[0], x[-1], 500)])
            zfactor1 = (1. + redshift) / (1. + other.redshift)
            spec = _LookupTable(x, a(x * zfactor1) * b(x), b.interpolant)
        else:
            zfactor1 = (1. + redshift) / (1. + self.redshift)
            zfactor2 = (1. + redshift) / (1. + other.redshift)
            spec = lambda w: a(w * zfactor1) * b(w * zfactor2)
        spectral = self.spectral or other.spectral
        return SED(spec, 'nm', 'fphotons' if spectral else '1', redshift=redshift, fast=True,
                   _blue_limit=blue_limit, _red_limit=red_limit, _wave_list=wave_list)

    def __mul__(self, other):
        from .gsobject import GSObject
        from .bandpass import Bandpass
        if not self.fast:
            raise GalSimNotImplementedError("SED arithmetic with fast=False is not built")
        if isinstance(other, SED):
            if self.spectral and other.spectral:
                raise GalSimIncompatibleValuesError("Cannot multiply two spectral densities together.",
                                                    self_sed=self, other=other)
            if other._const:
                return self._mul_scalar(other._spec(42.0), self.spectral or other.spectral)
            if self._const:
                return other._mul_scalar(self._spec(42.0), self.spectral or other.spectral)
            return self._mul_sed(other)
        if isinstance(other, GSObject):
            return other * self
        from .chromatic import ChromaticObject
        if isinstance(other, ChromaticObject):
            return other * self
        if isinstance(other, Bandpass):
            raise GalSimNotImplementedError("SED * Bandpass is not built")
        if hasattr(other, '__call__'):
            fs = self._fast_spec
            z = self.redshift
            spec = lambda w: fs(w) * other(w * (1.0 + z))
            return SED(spec, 'nm', 'fphotons' if self.spectral else '1', redshift=self.redshift,
                       fast=True, _blue_limit=self.blue_limit, _red_limit=self.red_limit,
                       _wave_list=self.wave_list)
        if isinstance(other, (int, float, np.floating, np.integer)):
            return self._mul_scalar(float(other), self.spectral)
        raise TypeError("Cannot multiply an SED by %s" % (other,))

    def __rmul__(self, other):
        return self * other

    def __truediv__(self, other):
        if isinstance(other, (int, float, np.floating, np.integer)):
            return self._mul_scalar(1. / float(other), self.spectral)
        raise GalSimNotImplementedError("SED division by a non-scalar is not built")

    __div__ = __truediv__

    def __add__(self, other):
        if self.spectral != other.spectral:
            raise GalSimIncompatibleValuesError("Cannot add SEDs with incompatible dimensions.",
                                                self_sed=self, other=other)
        wave_list, blue_limit, red_limit = combine_wave_list(self, other)
        a, b = self, other
        spec = lambda w: a(w) + b(w)
        return SED(spec, 'nm', 'fphotons' if self.spectral else '1', fast=True,
                   _blue_limit=blue_limit, _red_limit=red_limit, _wave_list=wave_list)

    # -- redshift, flux ------------------------------------------------------------------------
    def atRedshift(self, redshift):
        """sed.py:788-807."""
        if redshift == self.redshift:
            return self
        if redshift <= -1:
            raise GalSimRangeError("Invalid redshift", redshift, -1.)
        zfactor = (1.0 + redshift) / (1.0 + self.redshift)
        return SED(self._spec, self.wave_type, self._flux_type, redshift, self.fast,
                   _wave_list=self.wave_list * zfactor, _blue_limit=self.blue_limit * zfactor,
                   _red_limit=self.red_limit * zfactor)

    def calculateFlux(self, bandpass):
        """Photons/cm^2/s through the bandpass (sed.py:809-852)."""
        if self.dimensionless:
            raise GalSimSEDError("Cannot calculate flux of dimensionless SED.", self)
        if bandpass is None:
            raise GalSimNotImplementedError("bolometric SED flux is not built")
        if len(bandpass.wave_list) > 0 or len(self.wave_list) > 0:
            slop = 1e-6
            if self.blue_limit > bandpass.blue_limit + slop or self.red_limit < bandpass.red_limit - slop:
                raise GalSimRangeError("Bandpass is not completely within defined wavelength range for this SED.",
                                       (bandpass.blue_limit, bandpass.red_limit), self.blue_limit, self.red_limit)
            wmin = max(self.blue_limit, bandpass.blue_limit)
            wmax = min(self.red_limit, bandpass.red_limit)
            fs = self._fast_spec
            if isinstance(fs, LookupTable):
                wf = 1. / (1. + self.redshift) / bandpass.wave_factor
                ff = 1. / bandpass.wave_factor
                wmin *= bandpass.wave_factor
                wmax *= bandpass.wave_factor
                return fs.integrate_product(bandpass._tp, wmin, wmax, wf) * ff
            w, _, _ = combine_wave_list(self, bandpass)
            interpolant = bandpass._tp.interpolant if hasattr(bandpass._tp, 'interpolant') else 'linear'
            return _LookupTable(w, bandpass(w), interpolant).integrate_product(self)
        raise GalSimNotImplementedError("flux of an analytic SED through an analytic Bandpass is not built")

    def withFlux(self, target_flux, bandpass):
        """sed.py:749-764."""
        return self * (target_flux / self.calculateFlux(bandpass))

    def __repr__(self):
        return 'galsim.SED(%r, wave_type=%r, flux_type=%r, redshift=%r)' % (
            self._orig_spec, self.wave_type, self._flux_type, self.redshift)

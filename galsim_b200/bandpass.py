"""Bandpass: filter throughputs (galsim/bandpass.py:33-720).

Host-side FP64 arithmetic for chromatic drawing: the dimensionless throughput as a function
of wavelength in nm, zero outside [blue_limit, red_limit], from a LookupTable or a callable
(with explicit limits) in nm or Angstrom, and the throughput-weighted mean wavelength.
"""
import numpy as np

from .table import LookupTable, _LookupTable
from .errors import (GalSimValueError, GalSimRangeError, GalSimIncompatibleValuesError,
                     GalSimNotImplementedError)

__all__ = ['Bandpass']


class Bandpass(object):
    """Throughput of a filter (bandpass.py:33-720); see the module docstring."""

    def __init__(self, throughput, wave_type, blue_limit=None, red_limit=None, zeropoint=None,
                 interpolant='linear', _wave_list=None, _tp=None):
        self._orig_tp = throughput
        if isinstance(wave_type, str) and wave_type.lower() in ('nm', 'nanometer', 'nanometers'):
            self.wave_type, self.wave_factor = 'nm', 1.
        elif isinstance(wave_type, str) and wave_type.lower() in ('a', 'ang', 'angstrom', 'angstroms'):
            self.wave_type, self.wave_factor = 'Angstrom', 10.
        else:
            raise GalSimValueError("Invalid wave_type.", wave_type, ('nm', 'Angstrom'))
        if blue_limit is not None and red_limit is not None and blue_limit >= red_limit:
            raise GalSimRangeError("blue_limit must be less than red_limit", blue_limit, None, red_limit)
        self.blue_limit = blue_limit
        self.red_limit = red_limit
        self.zeropoint = zeropoint
        self.interpolant = interpolant
        if _tp is not None:
            self._tp = _tp
        elif isinstance(throughput, LookupTable) or hasattr(throughput, '__call__'):
            self._tp = throughput
        elif isinstance(throughput, (int, float, np.floating)) or isinstance(throughput, str):
            try:
                v = float(throughput)
            except ValueError:
                raise GalSimNotImplementedError("Bandpass throughput strings other than a number "
                                                "(file names, expressions) are not built")
            self._tp = lambda w: np.full(np.shape(w), v) if np.ndim(w) else v
        else:
            raise GalSimValueError("Invalid throughput", throughput)
        if _wave_list is not None:
            self.wave_list = np.asarray(_wave_list, dtype=float)
            return
        if self.wave_factor != 1.0:
            if self.blue_limit is not None:
                self.blue_limit /= self.wave_factor
            if self.red_limit is not None:
                self.red_limit /= self.wave_factor
        if isinstance(self._tp, LookupTable):
            if self.blue_limit is None:
                self.blue_limit = float(self._tp.x_min) / self.wave_factor
            if self.red_limit is None:
                self.red_limit = float(self._tp.x_max) / self.wave_factor
        elif self.blue_limit is None or self.red_limit is None:
            raise GalSimIncompatibleValuesError(
                "red_limit and blue_limit are required if throughput is not a LookupTable.",
                blue_limit=blue_limit, red_limit=red_limit, throughput=throughput)
        if isinstance(self._tp, LookupTable):
            wl = np.array(self._tp.getArgs()) / self.wave_factor
            if self.blue_limit < self._tp.x_min / self.wave_factor:
                raise GalSimRangeError("Cannot set blue_limit to be less than throughput x_min",
                                       self.blue_limit, self._tp.x_min, self._tp.x_max)
            if self.red_limit > self._tp.x_max / self.wave_factor:
                raise GalSimRangeError("Cannot set red_limit to be greater than throughput x_max",
                                       self.red_limit, self._tp.x_min, self._tp.x_max)
            # (the reference's np.append / np.insert of the limits here discard their results,
            # bandpass.py:213-216, so the list holds only the table's arguments in range)
            self.wave_list = wl[(wl >= self.blue_limit) & (wl <= self.red_limit)]
        else:
            self.wave_list = np.array([], dtype=float)

    def func(self, wave):
        if self.wave_factor == 1.:
            return self._tp(np.asarray(wave, dtype=float))
        return self._tp(np.asarray(wave) * self.wave_factor)

    def __call__(self, wave):
        """Throughput at wavelength(s) in nm, 0 outside the limits (bandpass.py:334-356)."""
        wave = np.asarray(wave)
        if wave.shape == ():
            if self.blue_limit <= wave <= self.red_limit:
                return float(self.func(float(wave)))
            return 0.0
        wgood = (wave >= self.blue_limit) & (wave <= self.red_limit)
        ret = np.zeros(wave.shape, dtype=float)
        np.place(ret, wgood, self.func(wave[wgood]))
        return ret

    @property
    def effective_wavelength(self):
        return self.calculateEffectiveWavelength()

    def calculateEffectiveWavelength(self, precise=False):
        """Throughput-weighted mean wavelength in nm (bandpass.py:366-390)."""
        if not hasattr(self, '_effective_wavelength') or precise:
            if len(self.wave_list) > 0 and not precise:
                num = self._tp.integrate_product(lambda w: w, self.blue_limit, self.red_limit,
                                                 x_factor=self.wave_factor)
                denom = self._tp.integrate(self.blue_limit * self.wave_factor,
                                           self.red_limit * self.wave_factor) / self.wave_factor
            else:
                raise GalSimNotImplementedError("the effective wavelength of an analytic throughput "
                                                "(adaptive integration) is not built")
            self._effective_wavelength = num / denom
        return self._effective_wavelength

    def __mul__(self, other):
        if isinstance(other, (int, float, np.floating)):
            import copy
            ret = copy.copy(self)
            if isinstance(self._tp, LookupTable):
                ret._tp = _LookupTable(self._tp.getArgs(), np.asarray(self._tp.getVals()) * other,
                                       self._tp.interpolant)
            else:
                f = self._tp
                ret._tp = lambda w: f(w) * other
            ret.__dict__.pop('_effective_wavelength', None)
            return ret
        raise GalSimNotImplementedError("Bandpass products other than with a scalar are not built")

    __rmul__ = __mul__

    def __repr__(self):
        return 'galsim.Bandpass(%r, wave_type=%r, blue_limit=%r, red_limit=%r)' % (
            self._orig_tp, self.wave_type, self.blue_limit, self.red_limit)

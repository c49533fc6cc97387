"""Differential chromatic refraction (galsim/dcr.py:22-148).

The refraction of the atmosphere as a function of wavelength, for ChromaticAtmosphere's
wavelength-dependent shifts: the refractive index of air by the Edlen / Coleman-Bozman-Meggers
formulae as given by Filippenko (1982, PASP 94, 715), and the plane-parallel refraction angle.
"""
from .angle import Angle, degrees

__all__ = ['air_refractive_index_minus_one', 'get_refraction', 'parse_dcr_angles']


def air_refractive_index_minus_one(wave, pressure=69.328, temperature=293.15, H2O_pressure=1.067):
    """n - 1 of air at wavelength(s) `wave` in nm; pressure and water vapour pressure in kPa,
    temperature in K (dcr.py:22-53)."""
    P = pressure * 7.50061683            # kPa -> mmHg
    T = temperature - 273.15             # K -> C
    W = H2O_pressure * 7.50061683
    sigma_squared = 1.0 / (wave * 1.e-3) ** 2.0   # micron^-2
    n_minus_one = (64.328 + (29498.1 / (146.0 - sigma_squared)) + (255.4 / (41.0 - sigma_squared))) * 1.e-6
    n_minus_one *= P * (1.0 + (1.049 - 0.0157 * T) * 1.e-6 * P) / (720.883 * (1.0 + 0.003661 * T))
    n_minus_one -= (0.0624 - 0.000680 * sigma_squared) / (1.0 + 0.003661 * T) * W * 1.e-6
    return n_minus_one


def get_refraction(wave, zenith_angle, **kwargs):
    """Change of zenith angle in radians of light of wavelength `wave` (nm) entering the
    atmosphere at `zenith_angle` (dcr.py:55-77)."""
    nm1 = air_refractive_index_minus_one(wave, **kwargs)
    r0 = nm1 * (nm1 + 2) / 2.0 / (nm1 ** 2 + 2 * nm1 + 1)
    return r0 * zenith_angle.tan()


def parse_dcr_angles(**kwargs):
    """zenith_angle and parallactic_angle (default 0) from the keywords; the others are returned
    for get_refraction (dcr.py:111-148).  Celestial coordinates (obj_coord with zenith_coord or
    HA and latitude) are not built."""
    if 'zenith_angle' in kwargs:
        zenith_angle = kwargs.pop('zenith_angle')
        parallactic_angle = kwargs.pop('parallactic_angle', 0.0 * degrees)
        kwargs.pop('obj_coord', None)
        if not isinstance(zenith_angle, Angle):
            raise TypeError("zenith_angle must be a galsim.Angle.")
        if not isinstance(parallactic_angle, Angle):
            raise TypeError("parallactic_angle must be a galsim.Angles.")
    elif 'obj_coord' in kwargs:
        from .errors import GalSimNotImplementedError
        raise GalSimNotImplementedError("DCR angles from celestial coordinates are not built")
    else:
        raise TypeError("Need to specify zenith_angle and parallactic_angle.")
    return zenith_angle, parallactic_angle, kwargs

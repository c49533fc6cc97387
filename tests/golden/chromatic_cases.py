"""Chromatic drawing cases, built with either galsim module (the reference, to make the
fixtures in reference_chromatic.npz, or galsim_b200, in the tests): the two share this API.

Tables are in nm and photons/nm/cm^2/s with linear interpolation (the reference's SED flux
conversions other than 'fphotons' need astropy, which the fixture run does not have)."""
import numpy as np

SED1 = ([300., 380., 450., 520., 600., 700., 820., 950., 1100.],
        [0.8, 1.1, 1.6, 1.9, 1.7, 1.3, 1.0, 0.7, 0.5])
SED2 = ([320., 400., 440., 480., 530., 580., 650., 760., 900., 1050.],
        [2.4, 2.0, 1.5, 1.4, 1.0, 0.9, 0.8, 0.6, 0.5, 0.45])
BP1 = ([400., 420., 440., 460., 480., 500., 520., 540., 560., 580., 600.],
       [0.0, 0.35, 0.62, 0.71, 0.74, 0.76, 0.75, 0.70, 0.52, 0.2, 0.0])
BP2 = ([540., 570., 600., 630., 660., 690., 720.],
       [0.0, 0.5, 0.8, 0.85, 0.8, 0.45, 0.0])


def seds(galsim):
    s1 = galsim.SED(galsim.LookupTable(*SED1, interpolant='linear'), 'nm', 'fphotons')
    s2 = galsim.SED(galsim.LookupTable(*SED2, interpolant='linear'), 'nm', 'fphotons')
    return s1, s2


def bandpasses(galsim):
    b1 = galsim.Bandpass(galsim.LookupTable(*BP1, interpolant='linear'), 'nm')
    b2 = galsim.Bandpass(galsim.LookupTable(*BP2, interpolant='linear'), 'nm')
    return b1, b2


def case(galsim, name):
    """(object, bandpass, drawImage kwargs) of case `name`."""
    s1, s2 = seds(galsim)
    b1, b2 = bandpasses(galsim)
    deg = galsim.degrees
    if name == 'sep_moffat':
        obj = galsim.Convolve(galsim.Exponential(half_light_radius=0.5, flux=1.) * s1,
                              galsim.Moffat(beta=3., fwhm=0.7))
        return obj, b1, dict(nx=40, ny=40, scale=0.2)
    if name == 'sep_z_kolm_f8':
        obj = galsim.Convolve(galsim.Sersic(n=1.5, half_light_radius=0.4) * s2.atRedshift(0.3),
                              galsim.Kolmogorov(fwhm=0.6))
        return obj, b2, dict(nx=40, ny=40, scale=0.2, dtype=np.float64)
    if name in ('atm_kolm', 'atm_kolm_trapz', 'atm_kolm_midpt', 'atm_kolm_f8'):
        psf = galsim.ChromaticAtmosphere(galsim.Kolmogorov(fwhm=0.7), 500., zenith_angle=30. * deg,
                                         parallactic_angle=20. * deg)
        obj = galsim.Convolve(galsim.Exponential(half_light_radius=0.4) * s1, psf)
        kw = dict(nx=40, ny=40, scale=0.2)
        if name == 'atm_kolm_trapz':
            kw['integrator'] = 'trapezoidal'
        if name == 'atm_kolm_midpt':
            kw['integrator'] = 'midpoint'
        if name == 'atm_kolm_f8':
            kw['dtype'] = np.float64
        return obj, b1, kw
    if name == 'atm_bulge_disk':
        psf = galsim.ChromaticAtmosphere(galsim.Moffat(beta=2.5, fwhm=0.6), 600., zenith_angle=45. * deg,
                                         alpha=-0.3, temperature=280., pressure=75.)
        gal = (galsim.DeVaucouleurs(half_light_radius=0.3) * s1 +
               galsim.Exponential(half_light_radius=0.6).shear(g1=0.2, g2=0.1) * s2)
        return galsim.Convolve(gal, psf), b2, dict(nx=48, ny=48, scale=0.2)
    if name == 'dilate_star':
        obj = galsim.ChromaticObject(galsim.Gaussian(sigma=0.3)).dilate(lambda w: (w / 500.) ** 0.3) * s2
        return obj, b1, dict(nx=32, ny=32, scale=0.2)
    if name == 'shift_gal_psf':
        psf = galsim.ChromaticObject(galsim.Moffat(beta=3.5, fwhm=0.5)).shift(lambda w: ((w - 500.) * 1e-3, 0.))
        obj = galsim.Convolve(galsim.Gaussian(sigma=0.4, flux=2.) * s1, psf)
        return obj, b1, dict(nx=32, ny=32, scale=0.2, offset=(0.3, -0.2))
    if name == 'airy_gal':
        psf = galsim.ChromaticAiry(lam=500., diam=0.5, obscuration=0.3)
        obj = galsim.Convolve(galsim.Exponential(half_light_radius=0.3) * s1, psf)
        return obj, b1, dict(nx=48, ny=48, scale=0.1)
    if name == 'atm_airy_f8':
        psf = galsim.Convolve(galsim.ChromaticAtmosphere(galsim.Kolmogorov(fwhm=0.5), 600., zenith_angle=20. * deg),
                              galsim.ChromaticAiry(lam=600., lam_over_diam=0.15))
        obj = galsim.Convolve(galsim.Sersic(n=2., half_light_radius=0.3) * s2, psf)
        return obj, b2, dict(nx=40, ny=40, scale=0.15, dtype=np.float64)
    raise ValueError(name)


CASES = ['sep_moffat', 'sep_z_kolm_f8', 'atm_kolm', 'atm_kolm_trapz', 'atm_kolm_midpt', 'atm_kolm_f8',
         'atm_bulge_disk', 'dilate_star', 'shift_gal_psf', 'airy_gal', 'atm_airy_f8']
REFRACTION_WAVES = [350., 420.5, 500., 633., 800., 1000.]


# drawKImage through a bandpass: (name, case of `case`, nx, scale = dk)
KCASES = [('k_atm_kolm', 'atm_kolm', 25, 0.6), ('k_atm_bulge_disk', 'atm_bulge_disk', 21, 0.8),
          ('k_shift_gal_psf', 'shift_gal_psf', 23, 0.7), ('k_sep_moffat', 'sep_moffat', 25, 0.6)]


def drawk(galsim, kname):
    _, name, n, dk = [k for k in KCASES if k[0] == kname][0]
    obj, bp, kw = case(galsim, name)
    return obj.drawKImage(bp, nx=n, ny=n, scale=dk)


def draw(galsim, name):
    obj, bp, kw = case(galsim, name)
    kw = dict(kw)
    integrator = kw.pop('integrator', 'quadratic')
    return obj.drawImage(bp, integrator=integrator, **kw)

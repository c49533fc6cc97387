"""Translate the plain-data profile descriptions of make_golden.py into oracle objects
(tests only)."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), 'oracle'))
import galsim_oracle as O  # noqa: E402


def oracle_profile(spec):
    kind = spec[0]
    if kind == 'gauss':
        return O.OGaussian(spec[1], spec[2])
    if kind == 'exp':
        return O.OExponential(spec[1] / 1.6783469900166605, spec[2])
    if kind == 'sersic':
        return O.OSersic(spec[1], hlr=spec[2], flux=spec[3])
    if kind == 'sersict':
        size = dict(hlr=spec[2]) if spec[6] == 'hlr' else dict(r0=spec[2])
        return O.OSersic(spec[1], flux=spec[3], trunc=spec[4], flux_untruncated=spec[5], **size)
    if kind == 'moffat':
        return O.OMoffat(spec[1], fwhm=spec[2], flux=spec[3])
    if kind == 'moffatt':
        key = {'fwhm': 'fwhm', 'hlr': 'hlr', 'r0': 'r0'}[spec[5]]
        return O.OMoffat(spec[1], flux=spec[3], trunc=spec[4], **{key: spec[2]})
    if kind == 'kolmogorov':
        return O.OKolmogorov(fwhm=spec[1], flux=spec[2])
    if kind == 'airy':
        return O.OAiry(spec[1], spec[2], spec[3])
    if kind == 'box':
        return O.OBox(spec[1], spec[2], spec[3])
    if kind == 'pixel':
        return O.OBox(spec[1], spec[1], 1.)
    if kind == 'shear':
        return oracle_profile(spec[3]).shear(spec[1], spec[2])
    if kind == 'shift':
        return oracle_profile(spec[3]).shift(spec[1], spec[2])
    if kind == 'dilate':
        s = spec[1]
        return O.OTransform(oracle_profile(spec[2]), jac=[[s, 0.], [0., s]], flux_ratio=s ** -2)
    if kind == 'rotate':
        import math
        t = math.radians(spec[1])
        s, c = math.sin(t), math.cos(t)
        return O.OTransform(oracle_profile(spec[2]), jac=[[c, -s], [s, c]])
    if kind == 'scaleflux':
        return O.OTransform(oracle_profile(spec[2]), flux_ratio=spec[1])
    if kind == 'conv':
        return O.OConvolve(*[oracle_profile(s) for s in spec[1]])
    if kind == 'sum':
        return O.OSum(*[oracle_profile(s) for s in spec[1]])
    if kind == 'ii':
        from make_golden import IMAGES
        kw = dict(spec[3])
        names = {'x_interpolant': 'x_interp', 'k_interpolant': 'k_interp',
                 '_force_stepk': 'force_stepk', '_force_maxk': 'force_maxk'}
        kw = {names.get(k, k): v for k, v in kw.items()}
        if 'pad_image' in kw:
            kw['pad_image'] = IMAGES[kw['pad_image']]
        return O.OInterpolatedImage(IMAGES[spec[1]], spec[2], **kw)
    raise ValueError(kind)


def load_interp_images(npz):
    """Register the InterpolatedImage source images stored in a fixture for the 'ii' specs."""
    import make_golden
    for k in npz.files:
        if k.startswith('img_'):
            make_golden.IMAGES[k[4:]] = npz[k]
    return make_golden.IMAGES


def product_profile(galsim, spec):
    """The same description built with a GalSim-like API module (galsim_b200)."""
    from make_golden import profile
    return profile(galsim, spec)

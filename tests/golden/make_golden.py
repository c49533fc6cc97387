"""Make the golden fixtures in tests/golden/ by running the reference GalSim itself.

    make -C oracle ref REF=/path/to/reference    # build the reference C++ into oracle/_ref
    python tests/golden/make_golden.py /path/to/reference [--configs-only | --grad-only | ...]

The reference Python package is imported from its checkout with the extension built from
its own C++ sources (oracle/ref_import.py).  Everything drawn here goes through the
reference's drawImage / drawKImage / wrap / irfft / stepk / maxk; the fixtures record the
inputs next to the outputs.  These files are the pin for both the numpy oracle and the GPU
kernels; the GPU tests read only these .npz files, never the reference checkout.
(reference_fits.npz, from main_fits, holds the reference's FITS test files as bytes.)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))


def profile(galsim, spec):
    """Build a reference object from a plain-data description (shared with the tests)."""
    kind = spec[0]
    if kind == 'gauss':
        return galsim.Gaussian(sigma=spec[1], flux=spec[2])
    if kind == 'exp':
        return galsim.Exponential(half_light_radius=spec[1], flux=spec[2])
    if kind == 'sersic':
        return galsim.Sersic(n=spec[1], half_light_radius=spec[2], flux=spec[3])
    if kind == 'sersict':
        # ('sersict', n, size, flux, trunc, flux_untruncated, 'hlr' | 'r0')
        size = dict(half_light_radius=spec[2]) if spec[6] == 'hlr' else dict(scale_radius=spec[2])
        return galsim.Sersic(n=spec[1], flux=spec[3], trunc=spec[4], flux_untruncated=spec[5], **size)
    if kind == 'moffat':
        return galsim.Moffat(beta=spec[1], fwhm=spec[2], flux=spec[3])
    if kind == 'moffatt':
        # ('moffatt', beta, size, flux, trunc, 'fwhm' | 'hlr' | 'r0')
        key = {'fwhm': 'fwhm', 'hlr': 'half_light_radius', 'r0': 'scale_radius'}[spec[5]]
        return galsim.Moffat(beta=spec[1], flux=spec[3], trunc=spec[4], **{key: spec[2]})
    if kind == 'kolmogorov':
        return galsim.Kolmogorov(fwhm=spec[1], flux=spec[2])
    if kind == 'airy':
        return galsim.Airy(lam_over_diam=spec[1], obscuration=spec[2], flux=spec[3])
    if kind == 'box':
        return galsim.Box(spec[1], spec[2], flux=spec[3])
    if kind == 'pixel':
        return galsim.Pixel(spec[1])
    if kind == 'shear':
        return profile(galsim, spec[3]).shear(g1=spec[1], g2=spec[2])
    if kind == 'shift':
        return profile(galsim, spec[3]).shift(spec[1], spec[2])
    if kind == 'dilate':
        return profile(galsim, spec[2]).dilate(spec[1])
    if kind == 'rotate':
        return profile(galsim, spec[2]).rotate(spec[1] * galsim.degrees)
    if kind == 'scaleflux':
        return profile(galsim, spec[2]) * spec[1]
    if kind == 'conv':
        return galsim.Convolve([profile(galsim, s) for s in spec[1]])
    if kind == 'sum':
        return galsim.Add([profile(galsim, s) for s in spec[1]])
    if kind == 'ii':
        # ('ii', image name, scale, keyword arguments); pad_image given by image name
        kw = dict(spec[3])
        if 'pad_image' in kw:
            kw['pad_image'] = galsim.Image(IMAGES[kw['pad_image']])
        if 'rng_seed' in kw:
            kw['rng'] = galsim.BaseDeviate(kw.pop('rng_seed'))
        return galsim.InterpolatedImage(galsim.Image(IMAGES[spec[1]], scale=spec[2]), **kw)
    raise ValueError(kind)


# ---- InterpolatedImage sources ---------------------------------------------------------------
# Seeded synthetic images: sums of elliptical Gaussians sampled at pixel centres plus a little
# Gaussian noise (a PSF-like and a galaxy-like shape, odd and even sizes), and a low-level
# noise field used as a pad image.  The arrays are stored in the fixture; the tests use them
# from there.
IMAGES = {}


def _blob(nx, ny, comps, noise, seed):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:ny, 0:nx].astype(float)
    x -= (nx - 1) / 2.
    y -= (ny - 1) / 2.
    im = np.zeros((ny, nx))
    for amp, cx, cy, sxx, syy, sxy in comps:
        dx, dy = x - cx, y - cy
        det = sxx * syy - sxy * sxy
        q = (syy * dx * dx - 2 * sxy * dx * dy + sxx * dy * dy) / det
        im += amp * np.exp(-0.5 * q)
    return im + noise * rng.standard_normal((ny, nx))


def source_images():
    IMAGES['psf32'] = _blob(32, 32, [(1., 0.2, -0.1, 3.0, 2.4, 0.5), (0.08, 0.5, 0.3, 12., 10., -2.)],
                            2e-4, 11)
    IMAGES['psf31x33'] = _blob(31, 33, [(1., -0.3, 0.4, 2.2, 3.1, -0.6), (0.05, 0., 0., 9., 14., 1.)],
                               1e-4, 12)
    IMAGES['gal24'] = _blob(24, 24, [(2., 1.0, -0.5, 6.0, 3.0, 1.5), (1., -2.0, 1.5, 2.0, 2.5, 0.)],
                            5e-3, 13)
    IMAGES['pad40'] = 1e-3 * np.random.default_rng(14).standard_normal((40, 40))
    return IMAGES


II_PSF = ('ii', 'psf32', 0.2, {})
INTERP_DRAW_CASES = [
    # (name, spec, nx, ny, scale, dtype, offset)
    ('ii_conv_exp', ('conv', [('shear', 0.2, 0.1, ('exp', 0.5, 2.)), II_PSF]), 48, 48, 0.2, 'f8', (0., 0.)),
    ('ii_alone_cubic_linear_offset', ('ii', 'psf31x33', 0.25, {'x_interpolant': 'cubic',
                                                                'k_interpolant': 'linear',
                                                                'offset': (0.3, -0.2)}),
     40, 40, 0.25, 'f8', (0.1, 0.05)),
    ('ii_general_jac_sersic', ('conv', [('sersic', 1.5, 0.4, 1e3),
                                        ('rotate', 25., ('shear', 0.1, 0.2, ('ii', 'psf32', 0.2,
                                                                             {'flux': 5.})))]),
     48, 48, 0.2, 'f4', (0., 0.)),
    ('ii_sb_rescaled', ('ii', 'gal24', 0.3, {'normalization': 'sb'}), 64, 64, 0.15, 'f8', (0., 0.)),
    ('ii_pad2_nocalc', ('conv', [('ii', 'gal24', 0.2, {'pad_factor': 2., 'calculate_stepk': False,
                                                        'calculate_maxk': False}),
                                 ('moffat', 3.0, 0.6, 1.)]), 40, 40, 0.2, 'f8', (0., 0.)),
    ('ii_forced', ('conv', [('exp', 0.4, 1.), ('ii', 'psf32', 0.2, {'_force_stepk': 0.8,
                                                                    '_force_maxk': 12.})]),
     48, 48, 0.2, 'f8', (0., 0.)),
    ('ii_nearest_quintic', ('conv', [('gauss', 0.3, 1.), ('ii', 'psf31x33', 0.2,
                                                          {'x_interpolant': 'nearest'})]),
     32, 32, 0.2, 'f8', (0., 0.)),
    ('ii_linear_pad_image', ('conv', [('gauss', 0.25, 1.), ('ii', 'psf32', 0.2,
                                                            {'x_interpolant': 'linear',
                                                             'k_interpolant': 'linear',
                                                             'pad_image': 'pad40'})]),
     40, 40, 0.2, 'f8', (0., 0.)),
    ('ii_delta_x', ('ii', 'gal24', 0.2, {'x_interpolant': 'delta'}), 32, 32, 0.2, 'f8', (0., 0.)),
    ('ii_two_images', ('conv', [('sum', [('ii', 'gal24', 0.2, {'flux': 40.}), ('exp', 0.6, 20.)]),
                                II_PSF]), 48, 48, 0.2, 'f4', (0., 0.)),
    # Gaussian noise padding (the padding's noise from a seeded BaseDeviate), inside the
    # pad_factor frame and larger than it
    ('ii_noise_pad', ('conv', [('exp', 0.4, 1.), ('ii', 'psf32', 0.2, {'noise_pad_size': 8.,
                                                                       'noise_pad': 1e-4,
                                                                       'rng_seed': 2024})]),
     48, 48, 0.2, 'f8', (0., 0.)),
    ('ii_noise_pad_big', ('ii', 'gal24', 0.3, {'noise_pad_size': 30., 'noise_pad': 2e-3,
                                               'rng_seed': 77, 'pad_factor': 2.}),
     64, 64, 0.3, 'f8', (0., 0.)),
    # Lanczos x interpolants (their transform from the reference's spline table), with and
    # without the DC correction, FP64 and FP32 draws
    ('ii_lanczos5_x', ('conv', [('exp', 0.4, 1.), ('ii', 'psf32', 0.2, {'x_interpolant': 'lanczos5'})]),
     48, 48, 0.2, 'f8', (0., 0.)),
    ('ii_lanczos3F_x_cubic_k', ('ii', 'gal24', 0.25, {'x_interpolant': 'lanczos3F',
                                                      'k_interpolant': 'cubic'}),
     40, 40, 0.25, 'f8', (0.2, -0.1)),
    ('ii_lanczos7_x_f4', ('conv', [('sersic', 2.5, 0.5, 1e3), ('ii', 'psf31x33', 0.2,
                                                               {'x_interpolant': 'lanczos7'})]),
     48, 48, 0.2, 'f4', (0., 0.)),
    # Lanczos k interpolants (n <= 3), with and without the DC correction
    ('ii_lanczos3_k', ('conv', [('exp', 0.4, 1.), ('ii', 'psf32', 0.2, {'k_interpolant': 'lanczos3'})]),
     48, 48, 0.2, 'f8', (0., 0.)),
    ('ii_lanczos2F_k_f4', ('ii', 'gal24', 0.25, {'x_interpolant': 'lanczos5', 'k_interpolant': 'lanczos2F'}),
     40, 40, 0.25, 'f4', (0.1, 0.2)),
    # the sinc x interpolant (its transform a box; stepk forced, as its support is infinite;
    # drawn at another scale than the image's, so that no k point falls on the box's edge,
    # where the transform jumps)
    ('ii_sinc_x', ('conv', [('exp', 0.4, 1.), ('ii', 'psf32', 0.2, {'x_interpolant': 'sinc',
                                                                    '_force_stepk': 0.6})]),
     56, 56, 0.17, 'f8', (0., 0.)),
    ('ii_calc_floats', ('conv', [('exp', 0.3, 1.), ('ii', 'psf32', 0.2, {'calculate_maxk': 3.0,
                                                                         'calculate_stepk': 0.5})]),
     48, 48, 0.2, 'f8', (0., 0.)),
    ('ii_shift_dilate', ('shift', 0.3, -0.15, ('dilate', 1.4, ('ii', 'psf31x33', 0.2, {}))),
     40, 40, 0.2, 'f8', (0., 0.)),
]

INTERP_KIMAGE_CASES = [
    ('k_ii', ('ii', 'psf31x33', 0.25, {}), 0.3, 21),
    ('k_ii_shear', ('shear', 0.15, -0.1, ('ii', 'psf32', 0.2, {'x_interpolant': 'cubic'})), 0.35, 21),
    ('k_ii_lanczos', ('shear', 0.1, 0.05, ('ii', 'psf31x33', 0.2, {'x_interpolant': 'lanczos5',
                                                                  'k_interpolant': 'lanczos3'})), 0.3, 21),
]

INTERP_SIZE_CASES = [c[1] for c in INTERP_DRAW_CASES if c[1][0] == 'ii'] + [
    II_PSF, ('ii', 'psf32', 0.2, {'k_interpolant': 'cubic', 'x_interpolant': 'linear'}),
    ('ii', 'gal24', 0.5, {'pad_factor': 6.}), ('ii', 'psf31x33', 0.1, {'use_true_center': False})]


# ---- cases ------------------------------------------------------------------------------
C1 = ('conv', [('shift', 0.13, -0.07, ('shear', 0.05, -0.03, ('exp', 1.0, 1.e4))),
               ('moffat', 3.0, 0.7, 1.0), ('pixel', 0.2)])

DRAW_CASES = [
    # (name, spec, nx, ny, scale, dtype, offset)
    ('c1_exp_moffat_pixel', C1, 64, 64, 0.2, 'f8', (0., 0.)),
    ('gauss_sheared', ('shear', 0.2, 0.1, ('gauss', 0.8, 100.)), 32, 32, 0.2, 'f8', (0., 0.)),
    ('gauss_round_odd', ('gauss', 0.5, 10.), 33, 31, 0.25, 'f4', (0.3, -0.2)),
    ('exp_sheared_shift', ('shift', 0.4, 0.2, ('shear', -0.3, 0.2, ('exp', 0.7, 50.))), 40, 40, 0.2, 'f8', (0., 0.)),
    ('sersic_25_kolm', ('conv', [('shear', 0.1, -0.25, ('sersic', 2.5, 0.5, 1.e4)),
                                  ('kolmogorov', 0.75, 1.0), ('pixel', 0.2)]), 48, 48, 0.2, 'f4', (0., 0.)),
    ('sersic_1_moffat25', ('conv', [('sersic', 1.0, 0.8, 1.e3), ('moffat', 2.5, 0.8, 1.0),
                                     ('pixel', 0.2)]), 48, 48, 0.2, 'f8', (0.1, 0.05)),
    ('bulge_disk_moffat_gen', ('conv', [('sum', [('shear', 0.2, 0.1, ('sersic', 4.0, 0.4, 300.)),
                                                 ('shear', -0.3, 0.2, ('exp', 0.8, 700.))]),
                                        ('moffat', 3.7, 0.7, 1.0), ('pixel', 0.2)]), 48, 48, 0.2, 'f4', (0., 0.)),
    ('airy_obsc', ('conv', [('sersic', 0.8, 0.3, 10.), ('airy', 0.1, 0.3, 1.0)]), 40, 40, 0.05, 'f8', (0., 0.)),
    ('airy_unobsc', ('airy', 0.2, 0.0, 5.), 32, 32, 0.1, 'f8', (0., 0.)),
    ('box_rotate', ('conv', [('rotate', 30., ('box', 0.6, 0.3, 2.)), ('gauss', 0.3, 1.)]), 32, 32, 0.1, 'f8', (0., 0.)),
    ('moffat_15_dilate', ('dilate', 1.3, ('moffat', 1.5, 0.9, 20.)), 32, 32, 0.2, 'f8', (0., 0.)),
    ('moffat_2', ('moffat', 2.0, 0.9, 20.), 32, 32, 0.2, 'f8', (0., 0.)),
    ('moffat_35_4', ('conv', [('moffat', 3.5, 0.9, 20.), ('moffat', 4.0, 0.5, 1.)]), 32, 32, 0.2, 'f8', (0., 0.)),
    ('kolm_scaled', ('scaleflux', 3.0, ('kolmogorov', 0.6, 7.)), 32, 32, 0.2, 'f8', (0., 0.)),
    ('sum_shifted', ('sum', [('shift', 0.5, 0., ('gauss', 0.3, 5.)), ('shift', -0.5, 0.3, ('exp', 0.4, 5.))]),
     40, 40, 0.15, 'f8', (0., 0.)),
]

KIMAGE_CASES = [
    ('k_gauss', ('gauss', 0.8, 3.), 0.3, 21),
    ('k_gauss_shear', ('shear', 0.2, 0.1, ('gauss', 0.8, 3.)), 0.3, 21),
    ('k_exp', ('exp', 0.7, 2.), 0.25, 21),
    ('k_exp_shear_shift', ('shift', 0.2, -0.1, ('shear', 0.3, -0.2, ('exp', 0.7, 2.))), 0.25, 25),
    ('k_sersic', ('sersic', 3.3, 0.6, 1.), 0.2, 21),
    ('k_moffat_gen', ('moffat', 2.7, 1.0, 1.), 0.3, 21),
    ('k_kolm', ('kolmogorov', 0.8, 1.), 0.3, 21),
    ('k_airy', ('airy', 0.5, 0.2, 1.), 0.5, 21),
    ('k_box', ('box', 0.5, 0.8, 1.), 0.5, 21),
]

SIZE_CASES = [('gauss', 0.7, 1.), ('exp', 0.9, 1.), ('moffat', 3.0, 0.7, 1.), ('moffat', 2.5, 0.8, 1.),
              ('moffat', 3.7, 0.6, 1.), ('moffat', 4.5, 1.0, 1.), ('moffat', 1.5, 0.8, 1.),
              ('kolmogorov', 0.7, 1.), ('airy', 0.1, 0.3, 1.), ('airy', 0.1, 0.0, 1.),
              ('box', 0.2, 0.2, 1.)] + \
             [('sersic', n, 0.5, 1.) for n in (0.5, 0.8, 1.0, 1.5, 2.5, 4.0, 6.0)]


# Large-FFT cases (N > 1024, the precision-study configuration: Sersic n 3..5.5 with an
# obscured Airy at 0.05" pixels).  The images have millions of pixels, so the fixture keeps a
# sample: the central 64 x 64 block, a strided grid, and the added flux.
LARGE_CASES = [
    ('sersic3_airy_1200', ('conv', [('sersic', 3.0, 1.0, 1e4), ('airy', 0.1, 0.3, 1.0), ('pixel', 0.05)]),
     1200, 1200, 0.05, 'f4'),
    ('sersic45_airy_auto', ('conv', [('sersic', 4.5, 2.0, 1e5), ('airy', 0.1, 0.3, 1.0), ('pixel', 0.05)]),
     None, None, 0.05, 'f4'),
    ('sersic55_airy_auto_f8', ('conv', [('shear', 0.1, -0.05, ('sersic', 5.5, 2.5, 1e5)),
                                        ('airy', 0.1, 0.3, 1.0), ('pixel', 0.05)]),
     None, None, 0.05, 'f8'),
]
LARGE_STRIDE = (29, 31)


def large_sample(a):
    """(central 64 x 64 block, strided grid) of an image array."""
    ny, nx = a.shape
    cy, cx = ny // 2, nx // 2
    return a[cy - 32:cy + 32, cx - 32:cx + 32].copy(), a[::LARGE_STRIDE[0], ::LARGE_STRIDE[1]].copy()


def main_large(ref_root):
    from ref_import import import_reference_galsim
    galsim = import_reference_galsim(ref_root)
    out = {}
    for name, spec, nx, ny, scale, dt in LARGE_CASES:
        im = profile(galsim, spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type, method='fft')
        block, grid = large_sample(im.array)
        out['large_' + name + '_block'] = block
        out['large_' + name + '_grid'] = grid
        out['large_' + name + '_shape'] = np.array(im.array.shape)
        out['large_' + name + '_flux'] = np.array(im.added_flux)
        out['large_' + name + '_peak'] = np.array(np.abs(im.array).max())
    np.savez_compressed(os.path.join(HERE, 'reference_large.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_large.npz'), len(out), 'arrays')


# Gradients of the fit-step model by central differences of the reference's own drawImage:
# L(p) = sum(w * image(p)) for Convolve(Sersic(n, hlr, flux).shear(g1, g2).shift(dx, dy),
# Moffat(2.5, fwhm=0.8), Pixel(0.2)) drawn into 48 x 48 float64 at scale 0.2; step 1e-4
# (relative for flux and hlr, absolute for the others).
GRAD_PARAMS = [(1.2e4, 0.55, 1.7, 0.07, -0.04, 0.05, -0.08),
               (6.0e3, 0.9, 2.6, -0.12, 0.09, -0.11, 0.03),
               (2.0e4, 0.35, 1.1, 0.02, 0.15, 0.0, 0.12)]


def fit_model(galsim, p):
    flux, hlr, n, g1, g2, dx, dy = p
    gal = galsim.Sersic(n=n, half_light_radius=hlr, flux=flux).shear(g1=g1, g2=g2).shift(dx, dy)
    return galsim.Convolve(gal, galsim.Moffat(beta=2.5, fwhm=0.8), galsim.Pixel(0.2))


def main_grad(ref_root):
    from ref_import import import_reference_galsim
    galsim = import_reference_galsim(ref_root)
    w = np.random.default_rng(2024).standard_normal((len(GRAD_PARAMS), 48, 48))
    grads = np.zeros((len(GRAD_PARAMS), 7))
    for s, p in enumerate(GRAD_PARAMS):
        for j in range(7):
            h = 1e-4 * (p[j] if j in (0, 1) else 1.)
            val = []
            for sgn in (1., -1.):
                q = list(p)
                q[j] += sgn * h
                im = fit_model(galsim, q).drawImage(nx=48, ny=48, scale=0.2, dtype=np.float64, method='fft')
                val.append(float((w[s] * im.array).sum()))
            grads[s, j] = (val[0] - val[1]) / (2. * h)
    np.savez_compressed(os.path.join(HERE, 'reference_grad.npz'), params=np.array(GRAD_PARAMS), w=w,
                        fd_grad=grads)
    print('wrote', os.path.join(HERE, 'reference_grad.npz'))


# Config-driven stamps (galsim/config): the reference's BuildStamps for each object.
CONFIG_NOBJ = 6
CONFIG_CASE = {
    'gal': {
        'type': 'Sum',
        'items': [
            {'type': 'Sersic', 'n': {'type': 'List', 'items': [1.5, 2.5, 4.0, 0.8, 3.2, 1.1]},
             'half_light_radius': {'type': 'List', 'items': [0.4, 0.6, 0.3, 0.8, 0.5, 0.45]},
             'flux': {'type': 'Sequence', 'first': 300., 'step': 50.}},
            {'type': 'Exponential', 'half_light_radius': 0.9,
             'flux': {'type': 'List', 'items': [500., 800.]},
             'ellip': {'type': 'E1E2', 'e1': 0.2, 'e2': {'type': 'List', 'items': [-0.1, 0.15, 0.0]}}},
        ],
        'ellip': {'type': 'G1G2', 'g1': {'type': 'List', 'items': [0.05, -0.12, 0.2]},
                  'g2': {'type': 'Sequence', 'first': -0.1, 'step': 0.04}},
        'rotate': {'type': 'List', 'items': ['10 deg', '-25 deg', '40 deg', '0 deg']},
        'dilate': {'type': 'Sequence', 'first': 1.0, 'step': 0.05, 'repeat': 2},
        'magnify': 1.02,
        'shift': {'type': 'XY', 'x': {'type': 'List', 'items': [0.1, -0.05]}, 'y': 0.03},
    },
    'psf': {'type': 'Moffat', 'beta': {'type': 'List', 'items': [2.5, 3.0, 3.7]}, 'fwhm': 0.7},
    'stamp': {'type': 'Basic', 'size': 48, 'offset': {'type': 'XY', 'x': 0.2, 'y': -0.1}},
    'image': {'type': 'Single', 'pixel_scale': 0.2},
}


def main_config(ref_root):
    import copy
    from ref_import import import_reference_galsim
    galsim = import_reference_galsim(ref_root)
    images = galsim.config.BuildStamps(CONFIG_NOBJ, copy.deepcopy(CONFIG_CASE), do_noise=False)[0]
    out = {'stamp_%d' % i: im.array.astype(np.float64) for i, im in enumerate(images)}
    out['flux'] = np.array([im.array.sum() for im in images])
    np.savez_compressed(os.path.join(HERE, 'reference_config.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_config.npz'))


def main_interp(ref_root):
    from ref_import import import_reference_galsim
    galsim = import_reference_galsim(ref_root)
    source_images()
    out = {'img_' + k: v for k, v in IMAGES.items()}
    for name, spec, nx, ny, scale, dt, off in INTERP_DRAW_CASES:
        obj = profile(galsim, spec)
        im = obj.drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type, method='fft',
                           offset=off)
        out['draw_' + name] = im.array
        out['draw_' + name + '_flux'] = np.array(im.added_flux)
    for name, spec, dk, n in INTERP_KIMAGE_CASES:
        im = profile(galsim, spec).drawKImage(nx=n, ny=n, scale=dk)
        out['kimg_' + name] = im.array
        out['kimg_' + name + '_xmin'] = np.array([im.bounds.xmin, im.bounds.ymin])
    out['sizes'] = np.array([(profile(galsim, sp).stepk, profile(galsim, sp).maxk)
                             for sp in INTERP_SIZE_CASES])
    # k values of the image-unit SBInterpolatedImage at scattered points (kValue, with the
    # integer-position shortcut of the separable fill at integer sample positions)
    rng = np.random.default_rng(99)
    kpts = np.concatenate([rng.uniform(-3., 3., (40, 2)), np.array([[0., 0.], [0.5, -1.25]])])
    ii = profile(galsim, ('ii', 'psf31x33', 0.25, {}))
    ii._sbp
    out['kvalue_pts'] = kpts
    out['kvalue_ii_psf31x33'] = np.array([ii._sbii.kValue(galsim._galsim.PositionD(a, b))
                                          for a, b in kpts])
    np.savez_compressed(os.path.join(HERE, 'reference_interp.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_interp.npz'), len(out), 'arrays')


# Noise: the reference's addNoise on seeded images.  Inputs are drawn by the reference (a bright
# sheared Sersic for Poisson means from 0 to a few thousand, covering the inversion and PTRD
# branches) and stored with the outputs.
NOISE_CASES = [
    # (name, kind, image source, dtype, seed, params)
    ('gauss_zero_f4', 'gauss', 'zero', 'f4', 5, dict(sigma=3.)),
    ('gauss_gal_f8', 'gauss', 'gal', 'f8', 123, dict(sigma=0.7)),
    ('poisson_gal_f4_sky', 'poisson', 'gal', 'f4', 77, dict(sky_level=12.3)),
    ('poisson_gal_f8', 'poisson', 'gal', 'f8', 78, dict(sky_level=0.)),
    ('ccd_gal_f4', 'ccd', 'gal', 'f4', 91, dict(sky_level=35.5, gain=1.7, read_noise=4.4)),
    ('ccd_gal_f8_gain0', 'ccd', 'gal', 'f8', 92, dict(sky_level=20., gain=0., read_noise=3.)),
    ('ccd_odd_f4', 'ccd', 'odd', 'f4', 93, dict(sky_level=5.25, gain=2.5, read_noise=0.)),
    # integer images: numpy's unsafe casts, the integer part of the sky subtracted after the cast
    ('gauss_gal_i4', 'gauss', 'gal', 'i4', 94, dict(sigma=2.5)),
    ('gauss_odd_u2', 'gauss', 'odd', 'u2', 95, dict(sigma=1.5)),
    ('poisson_gal_i2_sky', 'poisson', 'gal', 'i2', 96, dict(sky_level=12.3)),
    ('poisson_odd_u4', 'poisson', 'odd', 'u4', 97, dict(sky_level=3.)),
    ('ccd_gal_u2', 'ccd', 'gal', 'u2', 98, dict(sky_level=40.7, gain=1.7, read_noise=4.4)),
    ('ccd_gal_i4_gain0', 'ccd', 'gal', 'i4', 99, dict(sky_level=20.5, gain=0., read_noise=3.)),
]
NOISE_BATCH_SEEDS = [1001, 1002, 1003, 1004]
# VariableGaussianNoise: (name, image source, dtype, seed); the variance image is
# 0.25 + 0.01 * |input| + a ramp, so it varies from pixel to pixel and stays positive
VARNOISE_CASES = [
    ('var_gal_f4', 'gal', 'f4', 311),
    ('var_odd_f8', 'odd', 'f8', 312),
    ('var_zero_f4', 'zero', 'f4', 313),
]


def variance_image(arr):
    ny, nx = arr.shape
    ramp = np.add.outer(np.arange(ny) * 0.03, np.arange(nx) * 0.02)
    return 0.25 + 0.01 * np.abs(arr.astype(np.float64)) + ramp


def deviate_sequences(galsim):
    """Draws from the reference's deviates (or the product's, with the same API): single calls
    and generate() interleaved (the Gaussian pair cache across them), generate_from_variance,
    the Poisson inversion / PTRD / normal (mean 0 and above 2^30) branches,
    generate_from_expectation, streams shared between deviates, and DeviateNoise on images."""
    out = {}
    u = galsim.UniformDeviate(1234)
    a = [u() for _ in range(5)]
    g = np.empty(7)
    u.generate(g)
    out['uniform'] = np.concatenate([a, g, [u(), u()]])
    gd = galsim.GaussianDeviate(2345, mean=1.5, sigma=2.5)
    a = [gd() for _ in range(3)]
    g = np.empty(5)
    gd.generate(g)
    b = [gd(), gd()]
    v = np.array([0.5, 2., 0., 9.])
    gd.generate_from_variance(v)
    out['gaussian'] = np.concatenate([a, g, b, v, [gd()]])
    pd = galsim.PoissonDeviate(3456, mean=7.3)
    a = [pd() for _ in range(4)]
    g = np.empty(6)
    pd.generate(g)
    pd2 = galsim.PoissonDeviate(pd, mean=120.)
    b = [pd2() for _ in range(3)]
    g2 = np.empty(5)
    pd2.generate(g2)
    pz = galsim.PoissonDeviate(pd, mean=0.)
    c = [pz() for _ in range(3)]
    ph = galsim.PoissonDeviate(pd, mean=float(2 ** 31))
    d = [ph() for _ in range(3)]
    g3 = np.empty(3)
    ph.generate(g3)
    d.append(ph())
    e = np.array([0., 3.2, 50., 0., float(2 ** 31), 7.])
    pd.generate_from_expectation(e)
    out['poisson'] = np.concatenate([a, g, b, g2, c, d, g3, e, [pd()]])
    # the host-drawn deviates: Weibull, Gamma with k < 1, = 1 and > 1, Chi-square
    wd = galsim.WeibullDeviate(2468, a=1.7, b=2.2)
    g = np.empty(6)
    wd.generate(g)
    out['weibull'] = np.concatenate([[wd(), wd()], g, [wd()]])
    vals = []
    for k, th in ((0.6, 1.3), (1., 2.), (3.5, 0.7)):
        gm = galsim.GammaDeviate(1357 + int(10 * k), k=k, theta=th)
        g = np.empty(7)
        gm.generate(g)
        vals.append(np.concatenate([[gm(), gm()], g, [gm()]]))
    out['gamma'] = np.concatenate(vals)
    cd = galsim.Chi2Deviate(9753, n=5.)
    g = np.empty(5)
    cd.generate(g)
    out['chi2'] = np.concatenate([[cd(), cd()], g, [cd()]])
    # binomial: inversion (small N p; one word per value) with generate and single draws, and
    # BTRD with single draws (the reference's generate splits BTRD draws over its OpenMP threads
    # by word counts, so its array depends on the thread count), p below and above 1/2
    vals = []
    for N, pr in ((20, 0.2), (15, 0.8)):
        bd = galsim.BinomialDeviate(4321 + N, N=N, p=pr)
        g = np.empty(6)
        bd.generate(g)
        vals.append(np.concatenate([[bd(), bd()], g, [bd()]]))
    for N, pr in ((200, 0.3), (500, 0.75)):
        bd = galsim.BinomialDeviate(4321 + N, N=N, p=pr)
        vals.append(np.array([bd() for _ in range(9)]))
    out['binomial'] = np.concatenate(vals)
    # DistDeviate from a tabulated density (trapezoid CDF, linear inverse)
    tab = galsim.LookupTable([0.5, 1., 1.7, 2.5, 4., 6.], [0.2, 1.5, 2.2, 1.1, 0.4, 0.05], interpolant='linear')
    dd = galsim.DistDeviate(8642, function=tab)
    g = np.empty(7)
    dd.generate(g)
    out['dist'] = np.concatenate([[dd(), dd()], g, [dd(), dd.val(0.37)]])
    # one stream shared: a uniform, then Gaussian values, then uniforms again
    s = galsim.UniformDeviate(4567)
    sg = galsim.GaussianDeviate(s, sigma=3.)
    out['shared'] = np.array([s(), sg(), sg(), sg(), s(), s()])
    for name, dev in (('uniform', galsim.UniformDeviate(5678)),
                      ('gauss', galsim.GaussianDeviate(6789, mean=-2., sigma=0.5)),
                      ('poisson', galsim.PoissonDeviate(7890, mean=4.5))):
        im = galsim.ImageF(7, 5, init_value=10.)
        im.addNoise(galsim.DeviateNoise(dev))
        imi = galsim.ImageI(6, 3, init_value=3)
        imi.addNoise(galsim.DeviateNoise(dev))
        out['devnoise_' + name] = im.array.copy()
        out['devnoise_i_' + name] = imi.array.copy()
    return out


def noise_input(galsim, src, dtype):
    if src == 'zero':
        return galsim.Image(17, 13, dtype=dtype, init_value=0.)
    if src == 'odd':
        return galsim.Gaussian(sigma=0.4, flux=3e3).drawImage(nx=31, ny=27, scale=0.2, dtype=dtype)
    gal = galsim.Convolve(galsim.Sersic(n=2.5, half_light_radius=0.6, flux=2e5).shear(g1=0.2, g2=-0.1),
                          galsim.Moffat(beta=3., fwhm=0.7))
    return gal.drawImage(nx=48, ny=40, scale=0.2, dtype=dtype)


def make_noise(galsim, kind, seed, p):
    rng = galsim.BaseDeviate(seed)
    if kind == 'gauss':
        return galsim.GaussianNoise(rng, **p)
    if kind == 'poisson':
        return galsim.PoissonNoise(rng, **p)
    return galsim.CCDNoise(rng, **p)


def main_noise(ref_root):
    from ref_import import import_reference_galsim
    galsim = import_reference_galsim(ref_root)
    out = {}
    for name, kind, src, dt, seed, p in NOISE_CASES:
        im = noise_input(galsim, src, np.dtype(dt).type)
        out['in_' + name] = im.array.copy()
        im.addNoise(make_noise(galsim, kind, seed, p))
        out['out_' + name] = im.array.copy()
    # one stream used twice: the second image continues where the first ended
    rng = galsim.BaseDeviate(4242)
    a = galsim.ImageF(9, 7, init_value=0.)
    b = galsim.ImageF(10, 5, init_value=0.)
    a.addNoise(galsim.GaussianNoise(rng, sigma=1.))
    b.addNoise(galsim.PoissonNoise(rng, sky_level=3.5))
    out['stream_a'] = a.array.copy()
    out['stream_b'] = b.array.copy()
    # a stamp batch with one seed per stamp (the config layer's per-object seeding)
    gal = galsim.Convolve(galsim.Exponential(half_light_radius=0.5, flux=5e3), galsim.Moffat(beta=3., fwhm=0.7))
    for i, seed in enumerate(NOISE_BATCH_SEEDS):
        im = gal.drawImage(nx=32, ny=32, scale=0.2)
        out['batch_in_%d' % i] = im.array.copy()
        im.addNoise(galsim.CCDNoise(galsim.BaseDeviate(seed), sky_level=50., gain=1.3, read_noise=5.))
        out['batch_out_%d' % i] = im.array.copy()
    for name, src, dt, seed in VARNOISE_CASES:
        im = noise_input(galsim, src, np.dtype(dt).type)
        out['in_' + name] = im.array.copy()
        out['var_' + name] = variance_image(im.array)
        im.addNoise(galsim.VariableGaussianNoise(galsim.BaseDeviate(seed), galsim.ImageD(out['var_' + name])))
        out['out_' + name] = im.array.copy()
    out.update({'dev_' + k: v for k, v in deviate_sequences(galsim).items()})
    # variable noise on an odd-sized image, then Gaussian noise from the same stream
    rng = galsim.BaseDeviate(4343)
    a = galsim.ImageF(9, 7, init_value=0.)
    b = galsim.ImageF(6, 5, init_value=1.)
    a.addNoise(galsim.VariableGaussianNoise(rng, galsim.ImageD(variance_image(a.array))))
    b.addNoise(galsim.GaussianNoise(rng, sigma=2.))
    out['varstream_a'] = a.array.copy()
    out['varstream_b'] = b.array.copy()
    np.savez_compressed(os.path.join(HERE, 'reference_noise.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_noise.npz'), len(out), 'arrays')


# FITS fixture files of the reference's test_image.py (test<T>.fits[.gz|.bz2] for T in S, I,
# F, D, US, UI: the 5 x 7 ref_array in each type), kept as raw bytes so that the FITS reader is
# checked against files astropy wrote, without the reference tree.
FITS_FIXTURES = ['test%s.fits%s' % (t, e) for t in ('S', 'I', 'F', 'D', 'US', 'UI')
                 for e in ('', '.gz', '.bz2')]


def main_fits(ref_root):
    src = os.path.join(ref_root, 'tests', 'Image_comparison_images')
    out = {}
    for name in FITS_FIXTURES:
        with open(os.path.join(src, name), 'rb') as f:
            out[name.replace('.', '_')] = np.frombuffer(f.read(), np.uint8)
    np.savez_compressed(os.path.join(HERE, 'reference_fits.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_fits.npz'), len(out), 'files')


# The batched configurations at their own settings: stamps of bench.py's seeded generators
# drawn one by one by the reference's drawImage.  Per stamp: its shape, the centred
# CFG_BLOCK x CFG_BLOCK block, a CFG_STRIDE-strided pixel grid, the added flux, the peak and
# the (N, Nk) that the reference's drawFFT_makeKImage chose (recorded by wrapping it).
#   batched forward: the leading CFG_C2_STAMPS stamps of the 4096-stamp workload (seed 1234),
#     default GSParams, automatically sized float32 images at scale 0.2;
#   mixed bulge+disk: GSParams(minimum_fft_size=32), the leading CFG_C4_LEADING stamps of the
#     16384-stamp workload (seed 2468) and up to CFG_C4_PER_N more per FFT size among the first
#     CFG_C4_POOL stamps, so that every size of the batch is covered.
CFG_BLOCK = 24
CFG_STRIDE = 7
CFG_C2_STAMPS = 256
CFG_C4_LEADING = 16
CFG_C4_PER_N = 3
CFG_C4_POOL = 4096


def bench_module():
    sys.path.insert(0, ROOT)
    import bench
    return bench


def config_sample(a):
    """The centred block and the strided grid of a stamp (shared with the tests)."""
    ny, nx = a.shape
    b = min(CFG_BLOCK, nx, ny)
    y0, x0 = (ny - b) // 2, (nx - b) // 2
    return a[y0:y0 + b, x0:x0 + b], a[::CFG_STRIDE, ::CFG_STRIDE]


def c2_object(galsim, p):
    n, hlr, flux, g1, g2, fwhm = p
    gal = galsim.Sersic(n=n, half_light_radius=hlr, flux=flux).shear(g1=g1, g2=g2)
    return galsim.Convolve(gal, galsim.Kolmogorov(fwhm=fwhm), galsim.Pixel(0.2))


def c4_object(galsim, m, i, gsp):
    bulge = galsim.Sersic(n=4., half_light_radius=m['bh'][i], flux=m['flux'][i] * m['bf'][i],
                          gsparams=gsp).shear(g1=m['g_b'][i, 0], g2=m['g_b'][i, 1])
    disk = galsim.Exponential(half_light_radius=m['dh'][i], flux=m['flux'][i] * (1. - m['bf'][i]),
                              gsparams=gsp).shear(g1=m['g_d'][i, 0], g2=m['g_d'][i, 1])
    psf = galsim.Moffat(beta=m['beta'][i], fwhm=m['fwhm'][i], gsparams=gsp)
    return galsim.Convolve(galsim.Add(bulge, disk), psf, galsim.Pixel(0.2, gsparams=gsp))


def _record_sizes(galsim):
    """Wrap the reference's drawFFT_makeKImage so that each draw leaves its (N, Nk)."""
    rec = []
    orig = galsim.GSObject.drawFFT_makeKImage

    def wrapped(self, image):
        kimage, N = orig(self, image)
        rec.append((int(N), int(kimage.bounds.xmax * 2)))
        return kimage, N
    galsim.GSObject.drawFFT_makeKImage = wrapped
    return rec


def main_configs(ref_root):
    from ref_import import import_reference_galsim
    galsim = import_reference_galsim(ref_root)
    bench = bench_module()
    sizes = _record_sizes(galsim)
    out = {}

    def store(prefix, ims):
        out[prefix + '_shape'] = np.array([im.array.shape for im in ims])
        out[prefix + '_flux'] = np.array([im.added_flux for im in ims])
        out[prefix + '_peak'] = np.array([np.abs(im.array).max() for im in ims])
        out[prefix + '_N_Nk'] = np.array(sizes[-len(ims):])
        blocks, grids = zip(*[config_sample(im.array) for im in ims])
        out[prefix + '_block'] = np.concatenate([b.ravel() for b in blocks])
        out[prefix + '_grid'] = np.concatenate([g.ravel() for g in grids])

    p2 = bench.workload_params(CFG_C2_STAMPS)
    ims = [c2_object(galsim, p).drawImage(scale=0.2, dtype=np.float32, method='fft') for p in p2]
    store('c2', ims)
    out['c2_params'] = p2

    gsp = galsim.GSParams(minimum_fft_size=32)
    m = bench.mixed_params()
    # the FFT size of each pool stamp, from the reference's own sizing (a draw of the stamp)
    pool_N = []
    for i in range(CFG_C4_POOL):
        c4_object(galsim, m, i, gsp).drawImage(scale=0.2, dtype=np.float32, method='fft')
        pool_N.append(sizes[-1][0])
    pick = list(range(CFG_C4_LEADING))
    for N in sorted(set(pool_N)):
        cand = [i for i in range(CFG_C4_POOL) if pool_N[i] == N and i not in pick]
        pick += cand[:CFG_C4_PER_N]
    ims = [c4_object(galsim, m, i, gsp).drawImage(scale=0.2, dtype=np.float32, method='fft') for i in pick]
    store('c4', ims)
    out['c4_index'] = np.array(pick)
    out['c4_pool_N'] = np.array(pool_N)
    out['cfg_block'] = np.array(CFG_BLOCK)
    out['cfg_stride'] = np.array(CFG_STRIDE)
    np.savez_compressed(os.path.join(HERE, 'reference_configs.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_configs.npz'), len(out), 'arrays;',
          'C4 sizes', dict(zip(*np.unique(out['c4_N_Nk'][:, 0], return_counts=True))))


# The reference's compiled hot-path steps one at a time (for the standalone C-ABI entry points):
# SBProfile.drawK through _drawKImage(image, jac) (the Jacobian composition of
# Transformation._drawKImage included), ApplyKImagePhases, Image.wrap on real and complex
# non-Hermitian images, and irfft with each combination of its shift flags, Nx != Ny.
STANDALONE_DRAWK = [
    # (name, spec, dk, bounds (xmin, xmax, ymin, ymax), jac (row-major) or None, dtype)
    ('exp_jac_general', ('exp', 0.8, 3.), 0.35, (0, 20, -20, 20), (1.1, 0.2, -0.1, 0.9), 'c16'),
    ('conv_shift_jac_diag', ('conv', [('shift', 0.15, -0.1, ('shear', 0.1, 0.05, ('gauss', 0.5, 2.))),
                                      ('moffat', 3.0, 0.7, 1.)]), 0.4, (-10, 10, -12, 12), (0.8, 0., 0., 1.3), 'c16'),
    ('sum_sersic_exp_jac', ('sum', [('sersic', 2.2, 0.6, 5.), ('rotate', 20., ('exp', 0.9, 2.))]), 0.3,
     (0, 16, -16, 16), (0.9, -0.15, 0.2, 1.05), 'c8'),
    ('conv_nojac', ('conv', [('exp', 0.5, 1.), ('kolmogorov', 0.7, 1.), ('pixel', 0.2)]), 0.5,
     (-8, 8, -8, 8), None, 'c16'),
]
STANDALONE_IRFFT = [(8, 12), (16, 8), (12, 12)]


def main_standalone(ref_root):
    from ref_import import import_reference_galsim
    galsim = import_reference_galsim(ref_root)
    out = {}
    for name, spec, dk, b, jac, dt in STANDALONE_DRAWK:
        im = galsim.Image(galsim.BoundsI(*b), dtype=np.complex128 if dt == 'c16' else np.complex64, scale=dk)
        j = None if jac is None else np.array(jac, dtype=float).reshape(2, 2)
        profile(galsim, spec)._drawKImage(im, j)
        out['drawk_' + name] = im.array.copy()
    rng = np.random.default_rng(31)
    # ApplyKImagePhases on a random complex image, general Jacobian and none
    for tag, jac in (('jac', (0.9, 0.3, -0.2, 1.1)), ('nojac', None)):
        a = rng.normal(size=(21, 13)) + 1j * rng.normal(size=(21, 13))
        im = galsim.ImageCD(a.copy(), xmin=0, ymin=-10, scale=0.3)
        j = None if jac is None else np.array(jac, dtype=float).reshape(2, 2)
        galsim._galsim.ApplyKImagePhases(im._image, im.scale, 0 if j is None else j.__array_interface__['data'][0],
                                         0.37, -0.61, 1.7)
        out['phase_in_' + tag] = a
        out['phase_out_' + tag] = im.array.copy()
    # wrap: non-Hermitian real and complex images
    a = rng.normal(size=(18, 17))
    im = galsim.ImageD(a.copy(), xmin=-7, ymin=-5)
    out['wrapr_in'] = a
    out['wrapr_out'] = im.wrap(galsim.BoundsI(-2, 3, -1, 4)).array.copy()
    a = rng.normal(size=(15, 12)) + 1j * rng.normal(size=(15, 12))
    im = galsim.ImageCD(a.copy(), xmin=-4, ymin=-6)
    out['wrapc_in'] = a
    out['wrapc_out'] = im.wrap(galsim.BoundsI(-1, 4, -3, 2)).array.copy()
    # irfft with each flag combination
    for Nx, Ny in STANDALONE_IRFFT:
        k = rng.normal(size=(Ny, Nx // 2 + 1)) + 1j * rng.normal(size=(Ny, Nx // 2 + 1))
        kim = galsim.ImageCD(k.copy(), xmin=0, ymin=-Ny // 2)
        out['irfft_in_%d_%d' % (Nx, Ny)] = k
        for si in (0, 1):
            for so in (0, 1):
                real = galsim.Image(galsim.BoundsI(-Nx // 2, Nx // 2 + 1, -Ny // 2, Ny // 2 - 1), dtype=float)
                galsim._galsim.irfft(kim._image, real._image, bool(si), bool(so))
                out['irfft_out_%d_%d_%d%d' % (Nx, Ny, si, so)] = real.array[:, :Nx].copy()
    np.savez_compressed(os.path.join(HERE, 'reference_standalone.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_standalone.npz'), len(out), 'arrays')


# Truncated Sersic profiles (sersic.py:196-265, SersicInfo with trunc > 0): drawImage through the
# reference, and the leaves' stepk / maxk.
TRUNC_CASES = [
    # (name, spec, nx, ny, scale, dtype, offset)
    ('t_n15_hlr_moffat', ('conv', [('sersict', 1.5, 0.5, 100., 2.0, False, 'hlr'), ('moffat', 3.0, 0.6, 1.),
                                   ('pixel', 0.2)]), 48, 48, 0.2, 'f8', (0., 0.)),
    ('t_n3_shear_kolm_f4', ('conv', [('shear', 0.1, -0.2, ('sersict', 3.0, 0.4, 1e3, 1.5, False, 'hlr')),
                                     ('kolmogorov', 0.7, 1.), ('pixel', 0.2)]), 48, 48, 0.2, 'f4', (0., 0.)),
    ('t_n4_fluxuntrunc', ('conv', [('sersict', 4.0, 0.5, 100., 3.0, True, 'hlr'), ('moffat', 3.0, 0.6, 1.),
                                   ('pixel', 0.2)]), 48, 48, 0.2, 'f8', (0.2, -0.1)),
    ('t_n25_r0_airy', ('conv', [('sersict', 2.5, 0.1, 50., 0.6, False, 'r0'), ('airy', 0.1, 0.3, 1.),
                                ('pixel', 0.05)]), 40, 40, 0.05, 'f8', (0., 0.)),
    ('t_n1_alone', ('sersict', 1.0, 0.6, 20., 1.2, False, 'hlr'), 32, 32, 0.2, 'f8', (0., 0.)),
    ('t_bulge_disk_f4', ('conv', [('sum', [('sersict', 4.0, 0.3, 300., 1.5, False, 'hlr'),
                                           ('shear', -0.2, 0.1, ('exp', 0.8, 700.))]),
                                  ('moffat', 3.7, 0.7, 1.), ('pixel', 0.2)]), 48, 48, 0.2, 'f4', (0., 0.)),
]
TRUNC_SIZE_CASES = [('sersict', n, 0.5, 1., t, fu, kind) for n, t, fu, kind in
                    ((0.7, 1.0, False, 'hlr'), (1.5, 2.0, False, 'hlr'), (3.0, 1.5, False, 'hlr'),
                     (4.0, 3.0, True, 'hlr'), (5.5, 2.5, False, 'r0'), (2.0, 0.9, False, 'hlr'))]


# Truncated Moffat profiles (moffat.py:79-125, SBMoffat with trunc > 0: the FT from a spline of
# the truncated Hankel transform): drawImage through the reference, and the profiles' sizes.
TRUNC_MOFFAT_CASES = [
    ('tm_b25_fwhm_gauss', ('conv', [('gauss', 0.4, 100.), ('moffatt', 2.5, 0.7, 1., 2.0, 'fwhm'),
                                    ('pixel', 0.2)]), 48, 48, 0.2, 'f8', (0., 0.)),
    ('tm_b105_hlr_alone', ('moffatt', 1.05, 0.4, 30., 1.5, 'hlr'), 40, 40, 0.2, 'f8', (0.1, 0.3)),
    ('tm_b3_r0_shear_f4', ('conv', [('shear', 0.15, 0.05, ('exp', 0.5, 1e3)),
                                    ('moffatt', 3.0, 0.5, 1., 1.6, 'r0'), ('pixel', 0.2)]), 48, 48, 0.2, 'f4',
                           (0., 0.)),
    ('tm_b45_hlr_sersic', ('conv', [('sersic', 2.0, 0.3, 50.), ('moffatt', 4.5, 0.35, 1., 0.9, 'hlr'),
                                    ('pixel', 0.1)]), 40, 40, 0.1, 'f8', (0., 0.)),
    ('tm_b08_r0_sum', ('sum', [('moffatt', 0.8, 0.3, 10., 1.2, 'r0'), ('gauss', 0.5, 5.)]), 32, 32, 0.2, 'f8',
                      (0., 0.)),
]
TRUNC_MOFFAT_SIZE_CASES = [('moffatt', b, sz, 1., t, kind) for b, sz, t, kind in
                           ((2.5, 0.7, 2.0, 'fwhm'), (1.05, 0.4, 1.5, 'hlr'), (3.0, 0.5, 1.6, 'r0'),
                            (4.5, 0.35, 0.9, 'hlr'), (0.8, 0.3, 1.2, 'r0'), (1.5, 0.6, 3.0, 'hlr'),
                            (6.0, 1.0, 2.0, 'fwhm'), (2.0, 0.5, 0.8, 'hlr'))]
TRUNC_MOFFAT_KIMAGE_CASES = [
    # (name, spec, dk, n): drawKImage on an n x n grid centred on k = 0
    ('tmk_b25', ('moffatt', 2.5, 0.7, 3., 2.0, 'fwhm'), 0.3, 41),
    ('tmk_b08_shear', ('shear', 0.1, 0.2, ('moffatt', 0.8, 0.3, 2., 1.2, 'r0')), 0.5, 51),
    ('tmk_b45_far', ('moffatt', 4.5, 0.35, 1., 0.9, 'hlr'), 2.0, 61),
]


def main_trunc(ref_root):
    from ref_import import import_reference_galsim
    galsim = import_reference_galsim(ref_root)
    out = {}
    for name, spec, nx, ny, scale, dt, off in TRUNC_CASES:
        im = profile(galsim, spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type, method='fft',
                                             offset=off)
        out['draw_' + name] = im.array
        out['draw_' + name + '_flux'] = np.array(im.added_flux)
    out['sizes'] = np.array([(profile(galsim, sp).stepk, profile(galsim, sp).maxk) for sp in TRUNC_SIZE_CASES])
    out['scale_radius'] = np.array([profile(galsim, sp).scale_radius for sp in TRUNC_SIZE_CASES])
    out['flux'] = np.array([profile(galsim, sp).flux for sp in TRUNC_SIZE_CASES])
    for name, spec, nx, ny, scale, dt, off in TRUNC_MOFFAT_CASES:
        im = profile(galsim, spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type, method='fft',
                                             offset=off)
        out['draw_' + name] = im.array
        out['draw_' + name + '_flux'] = np.array(im.added_flux)
    objs = [profile(galsim, sp) for sp in TRUNC_MOFFAT_SIZE_CASES]
    out['moffat_sizes'] = np.array([(o.stepk, o.maxk) for o in objs])
    out['moffat_scale_radius'] = np.array([o.scale_radius for o in objs])
    out['moffat_hlr'] = np.array([o.half_light_radius for o in objs])
    for name, spec, dk, n in TRUNC_MOFFAT_KIMAGE_CASES:
        out['kimg_' + name] = profile(galsim, spec).drawKImage(nx=n, ny=n, scale=dk).array
    np.savez_compressed(os.path.join(HERE, 'reference_trunc.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_trunc.npz'), len(out), 'arrays')


# Real-space drawing (drawImage with method 'no_pixel' / 'sb' on profiles analytic in real
# space: GSObject.drawReal, gsobject.py:1846-1898, SBProfile::draw).
REAL_CASES = [
    # (name, spec, nx, ny, scale, dtype, method, offset)
    ('r_gauss_f8', ('gauss', 0.7, 10.), 32, 32, 0.2, 'f8', 'no_pixel', (0., 0.)),
    ('r_exp_shear_f4', ('shear', 0.2, -0.1, ('exp', 0.6, 50.)), 33, 31, 0.2, 'f4', 'no_pixel', (0.3, -0.2)),
    ('r_sersic_f8', ('sersic', 2.5, 0.5, 20.), 40, 40, 0.1, 'f8', 'no_pixel', (0., 0.)),
    ('r_sersict_f8', ('sersict', 3.0, 0.4, 8., 1.5, False, 'hlr'), 40, 40, 0.1, 'f8', 'sb', (0.1, 0.)),
    ('r_moffat_f8', ('moffat', 3.5, 0.8, 5.), 32, 32, 0.2, 'f8', 'no_pixel', (0., 0.25)),
    ('r_moffatt_f4', ('moffatt', 2.0, 0.5, 3., 1.2, 'r0'), 32, 32, 0.1, 'f4', 'no_pixel', (0., 0.)),
    ('r_kolm_f8', ('kolmogorov', 0.7, 4.), 48, 48, 0.1, 'f8', 'no_pixel', (0., 0.)),
    ('r_kolm_dilate_shift_f4', ('shift', 0.05, -0.03, ('dilate', 1.1, ('kolmogorov', 0.6, 2.))), 40, 40, 0.08,
     'f4', 'no_pixel', (0., 0.)),
    ('r_airy_obs_f8', ('airy', 0.2, 0.3, 1.), 40, 40, 0.05, 'f8', 'no_pixel', (0., 0.)),
    ('r_airy_f8', ('rotate', 20., ('airy', 0.25, 0.0, 2.)), 40, 40, 0.05, 'f8', 'no_pixel', (0.2, 0.)),
    ('r_box_f8', ('box', 1.05, 0.7, 3.), 16, 16, 0.2, 'f8', 'no_pixel', (0., 0.)),
    ('r_box_rot_f8', ('rotate', 30., ('box', 1.3, 0.9, 3.)), 16, 16, 0.2, 'f8', 'no_pixel', (0.1, 0.1)),
    ('r_sum_f8', ('sum', [('gauss', 0.5, 3.), ('shift', 0.3, 0.2, ('exp', 0.4, 2.)),
                          ('shear', 0.1, 0.3, ('moffat', 2.5, 0.6, 1.))]), 36, 36, 0.15, 'f8', 'no_pixel', (0., 0.)),
    # InterpolatedImages drawn in real space (their x interpolant over the image's pixels)
    ('r_ii_quintic_f8', ('ii', 'psf32', 0.2, {}), 40, 40, 0.15, 'f8', 'no_pixel', (0.1, -0.2)),
    ('r_ii_lanczos3_shear_f8', ('shear', 0.1, -0.05, ('ii', 'gal24', 0.25, {'x_interpolant': 'lanczos3'})),
     36, 36, 0.2, 'f8', 'no_pixel', (0., 0.)),
    ('r_ii_cubic_sum_f4', ('sum', [('ii', 'psf31x33', 0.2, {'x_interpolant': 'cubic', 'flux': 3.}),
                                   ('gauss', 0.4, 1.)]), 32, 32, 0.2, 'f4', 'no_pixel', (0., 0.)),
    ('r_ii_linear_same_scale_f8', ('ii', 'gal24', 0.2, {'x_interpolant': 'linear'}), 24, 24, 0.2, 'f8',
     'no_pixel', (0., 0.)),
]


def main_real(ref_root):
    from ref_import import import_reference_galsim
    galsim = import_reference_galsim(ref_root)
    source_images()
    out = {}
    for name, spec, nx, ny, scale, dt, method, off in REAL_CASES:
        im = profile(galsim, spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type, method=method,
                                             offset=off)
        out['draw_' + name] = im.array
        out['draw_' + name + '_flux'] = np.array(im.added_flux)
    np.savez_compressed(os.path.join(HERE, 'reference_real.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_real.npz'), len(out), 'arrays')


def main_chromatic(ref_root):
    """Chromatic drawing through bandpasses (chromatic.py) and the host-side numbers it uses."""
    import chromatic_cases as CC
    from ref_import import import_reference_galsim
    galsim = import_reference_galsim(ref_root)
    out = {}
    for name in CC.CASES:
        im = CC.draw(galsim, name)
        out['draw_' + name] = im.array
        out['draw_' + name + '_flux'] = np.array(getattr(im, 'added_flux', np.nan))
    for kname, _, _, _ in CC.KCASES:
        im = CC.drawk(galsim, kname)
        out['kdraw_' + kname] = im.array
        out['kdraw_' + kname + '_xmin'] = np.array([im.bounds.xmin, im.bounds.ymin])
    s1, s2 = CC.seds(galsim)
    b1, b2 = CC.bandpasses(galsim)
    out['effective_wavelength'] = np.array([b1.effective_wavelength, b2.effective_wavelength])
    out['sed_flux'] = np.array([s1.calculateFlux(b1), s2.calculateFlux(b2), s1.atRedshift(0.3).calculateFlux(b1),
                                s2.atRedshift(0.3).calculateFlux(b2), (s1 * 2.5).calculateFlux(b2)])
    waves = np.linspace(400., 600., 37)
    out['sed_values'] = np.array([s1(waves), s2(waves), s1.atRedshift(0.3)(waves)])
    out['bp_values'] = np.array([b1(waves), b2(np.linspace(540., 720., 37))])
    w = np.array(CC.REFRACTION_WAVES)
    out['refraction'] = np.array([galsim.dcr.get_refraction(w, 30. * galsim.degrees),
                                  galsim.dcr.get_refraction(w, 45. * galsim.degrees, temperature=280.,
                                                            pressure=75.)])
    np.savez_compressed(os.path.join(HERE, 'reference_chromatic.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_chromatic.npz'), len(out), 'arrays')


def main(ref_root):
    from ref_import import import_reference_galsim
    galsim = import_reference_galsim(ref_root)
    out = {}
    # drawImage cases
    for name, spec, nx, ny, scale, dt, off in DRAW_CASES:
        obj = profile(galsim, spec)
        im = obj.drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type, method='fft',
                           offset=off)
        out['draw_' + name] = im.array
        out['draw_' + name + '_flux'] = np.array(im.added_flux)
    # drawKImage cases (odd-sized grid centred on k = 0, given dk)
    for name, spec, dk, n in KIMAGE_CASES:
        obj = profile(galsim, spec)
        im = obj.drawKImage(nx=n, ny=n, scale=dk)
        out['kimg_' + name] = im.array
        out['kimg_' + name + '_xmin'] = np.array([im.bounds.xmin, im.bounds.ymin])
    # stepk / maxk of leaves
    sizes = []
    for spec in SIZE_CASES:
        obj = profile(galsim, spec)
        sizes.append((obj.stepk, obj.maxk))
    out['sizes'] = np.array(sizes)
    # Sersic scale radii from hlr
    out['sersic_r0'] = np.array([galsim.Sersic(n=n, half_light_radius=1.).scale_radius
                                 for n in (0.5, 0.8, 1.0, 1.5, 2.5, 4.0, 6.0)])
    # goodFFTSize
    gs = np.arange(1, 3000)
    out['good_fft_in'] = gs
    out['good_fft_out'] = np.array([galsim.Image.good_fft_size(int(v)) for v in gs])
    # wrap + irfft of random Hermitian-layout k-images (image.py:789-796, fft.py)
    rng = np.random.default_rng(77)
    for Nk, N in ((16, 8), (20, 8), (12, 12), (24, 12)):
        kim = galsim.ImageCD((rng.normal(size=(Nk + 1, Nk // 2 + 1)) +
                              1j * rng.normal(size=(Nk + 1, Nk // 2 + 1))),
                             xmin=0, ymin=-Nk // 2)
        out['wrap_in_%d_%d' % (Nk, N)] = kim.array.copy()
        w = kim.wrap(galsim.BoundsI(0, N // 2, -N // 2, N // 2 - 1), hermitian='x')
        out['wrap_out_%d_%d' % (Nk, N)] = w.array.copy()
        real = galsim.Image(galsim.BoundsI(-N // 2, N // 2 + 1, -N // 2, N // 2 - 1), dtype=float)
        galsim._galsim.irfft(w._image, real._image, True, True)
        out['irfft_out_%d_%d' % (Nk, N)] = real.array[:, :N].copy()
    np.savez_compressed(os.path.join(HERE, 'reference_draws.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_draws.npz'), len(out), 'arrays')


if __name__ == '__main__':
    args = [a for a in sys.argv[1:] if not a.startswith('--')]
    root = args[0] if args else os.environ.get('GSB_REFERENCE')
    if not root:
        sys.exit('usage: make_golden.py REFERENCE_CHECKOUT [--<part>-only] (or set GSB_REFERENCE)')
    if '--grad-only' in sys.argv:
        main_grad(root)
    elif '--interp-only' in sys.argv:
        main_interp(root)
    elif '--noise-only' in sys.argv:
        main_noise(root)
    elif '--config-only' in sys.argv:
        main_config(root)
    elif '--fits-only' in sys.argv:
        main_fits(root)
    elif '--configs-only' in sys.argv:
        main_configs(root)
    elif '--standalone-only' in sys.argv:
        main_standalone(root)
    elif '--trunc-only' in sys.argv:
        main_trunc(root)
    elif '--chromatic-only' in sys.argv:
        main_chromatic(root)
    elif '--real-only' in sys.argv:
        main_real(root)
    else:
        if '--large-only' not in sys.argv:
            main(root)
        main_large(root)
        main_grad(root)
        main_config(root)
        main_interp(root)
        main_noise(root)
        main_fits(root)
        main_configs(root)
        main_standalone(root)
        main_trunc(root)
        main_chromatic(root)
        main_real(root)

"""GPU parity of chromatic drawing through a bandpass (chromatic.py: ChromaticObject.drawImage,
ChromaticConvolution.drawImage with its effective PSF, ChromaticSum, ChromaticAtmosphere) against
images the reference drew (tests/golden/reference_chromatic.npz).

The integrand at all integration wavelengths is drawn in one batched pass (in real space for the
effective PSF of an analytic PSF, as the reference draws it) and summed on the device.
Tolerances: 2e-5 of the peak (and 2e-5 in flux) wherever an FP32 stage is involved -- the
reference's effective PSF image is float32 whatever the output dtype, and float32 outputs come
from complex64 k-images; 1e-9 for the separable float64 case drawn with FP64 kernels (one FFT
draw of the fiducial profile, no float32 stage)."""
import os
import sys

import numpy as np
import pytest

import galsim_b200 as galsim

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, 'golden'))
import chromatic_cases as CC  # noqa: E402

REF = np.load(os.path.join(HERE, 'golden', 'reference_chromatic.npz'))


def _draw(name, **extra):
    obj, bp, kw = CC.case(galsim, name)
    kw = dict(kw)
    integrator = kw.pop('integrator', 'quadratic')
    kw.update(extra)
    return obj.drawImage(bp, integrator=integrator, **kw)


@pytest.mark.parametrize('name', CC.CASES)
def test_chromatic_draw_vs_reference(name):
    im = _draw(name)
    ref = REF['draw_' + name]
    assert im.array.dtype == ref.dtype
    peak = np.abs(ref).max()
    err = np.abs(im.array.astype(float) - ref).max() / peak
    assert err <= 2e-5, (name, err)
    fref = float(REF['draw_' + name + '_flux'])
    assert abs(im.added_flux - fref) <= 2e-5 * max(abs(fref), 1e-300) or fref == im.added_flux == 0., \
        (name, im.added_flux, fref)


def test_separable_float64_with_fp64_kernels():
    im = _draw('sep_z_kolm_f8', precision='fp64')
    ref = REF['draw_sep_z_kolm_f8']
    assert np.abs(im.array - ref).max() <= 1e-9 * np.abs(ref).max()
    assert abs(im.added_flux - float(REF['draw_sep_z_kolm_f8_flux'])) <= 1e-10 * abs(im.added_flux)


def test_integrand_batch_is_one_draw_per_wavelength():
    """The effective PSF of the Kolmogorov atmosphere case integrates over the merged wave
    list of the SED and the bandpass inside the band: 11 + 1 wavelengths."""
    obj, bp, kw = CC.case(galsim, 'atm_kolm')
    insep = obj.obj_list[1] * obj.obj_list[0].sed
    img = insep.drawImage(bp, scale=0.05, method='no_pixel')
    assert insep._last_n_eval == 12
    assert np.isfinite(img.array).all() and img.array.sum() > 0.


def test_chromatic_batch_matches_single_draws():
    """draw_batch of a batched bulge + disk through a ChromaticAtmosphere (two effective PSFs,
    each integrated once for the batch) draws what drawImage draws galaxy by galaxy."""
    s1, s2 = CC.seds(galsim)
    b1, _ = CC.bandpasses(galsim)
    psf = galsim.ChromaticAtmosphere(galsim.Kolmogorov(fwhm=0.7), 500., zenith_angle=30. * galsim.degrees)
    hlr = np.array([0.3, 0.5, 0.8])
    g1 = np.array([0.1, -0.2, 0.05])

    def gal(h, g):
        return (galsim.DeVaucouleurs(half_light_radius=h * 0.5, flux=0.3) * s1 +
                galsim.Exponential(half_light_radius=h, flux=0.7).shear(g1=g, g2=0.1) * s2)
    st = galsim.draw_batch(galsim.Convolve(gal(hlr, g1), psf), nx=32, ny=32, scale=0.2, bandpass=b1)
    for i in range(3):
        im = galsim.Convolve(gal(hlr[i], g1[i]), psf).drawImage(b1, nx=32, ny=32, scale=0.2)
        a = st.array(i)
        assert np.abs(a - im.array).max() <= 1e-5 * np.abs(im.array).max(), i


@pytest.mark.parametrize('kname', [k[0] for k in CC.KCASES])
def test_chromatic_drawkimage_vs_reference(kname):
    """ChromaticObject.drawKImage through a bandpass: the k-images at the integrator's
    wavelengths drawn as one batch and summed with the rule's weights (FP64)."""
    im = CC.drawk(galsim, kname)
    ref = REF['kdraw_' + kname]
    assert im.array.shape == ref.shape and im.array.dtype == ref.dtype
    assert (im.bounds.xmin, im.bounds.ymin) == tuple(REF['kdraw_' + kname + '_xmin'])
    assert np.abs(im.array - ref).max() <= 1e-9 * np.abs(ref).max(), (kname, np.abs(im.array - ref).max())

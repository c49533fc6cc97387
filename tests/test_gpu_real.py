"""GPU parity of real-space drawing (drawImage with method 'no_pixel' / 'sb' on profiles that are
analytic in real space; GSObject.drawReal, gsobject.py:1846-1898) against images the reference
drew (tests/golden/reference_real.npz), through gsb_draw_real.

Tolerances: float64 images 1e-12 of the peak and 1e-12 in flux (the same FP64 formulas; the
reference's fmath exponential and power differ from CUDA's by a few ulp), except the
Kolmogorov profile, whose radial spline nodes sit at exp(-3 + i dlogr) here and at the
reference's running sum of dlogr there (1e-10); float32 images 1e-6 (rounding of the stored
values and of the reference's float32 accumulation of Sum members)."""
import os

import numpy as np
import pytest

import galsim_b200 as galsim
import make_golden as MG

pytestmark = pytest.mark.gpu
REF = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'reference_real.npz'))
import specs  # noqa: E402
specs.load_interp_images(np.load(os.path.join(specs.HERE, 'reference_interp.npz')))   # the 'ii' cases' images


@pytest.mark.parametrize('case', MG.REAL_CASES, ids=[c[0] for c in MG.REAL_CASES])
def test_real_space_draw_vs_reference(case):
    name, spec, nx, ny, scale, dt, method, off = case
    im = MG.profile(galsim, spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type, method=method,
                                            offset=off)
    ref = REF['draw_' + name]
    assert im.array.dtype == ref.dtype
    if dt == 'f4':
        tol = 1e-6
    else:
        tol = 1e-10 if 'kolm' in name else 1e-12
    peak = np.abs(ref).max()
    err = np.abs(im.array.astype(float) - ref).max() / peak
    assert err <= tol, (name, err)
    fref = float(REF['draw_' + name + '_flux'])
    assert abs(im.added_flux - fref) <= tol * abs(fref), (name, im.added_flux, fref)


def test_real_space_batch_equals_single_draws():
    """draw_batch(method='no_pixel') of batched analytic profiles (one gsb_draw_real launch)
    draws what drawImage draws stamp by stamp; automatic sizes too."""
    sig = np.array([0.4, 0.6, 0.9])
    obj = galsim.Add(galsim.Gaussian(sigma=sig, flux=2.), galsim.Moffat(beta=3., fwhm=0.7).shift(0.1, 0.))
    st = galsim.draw_batch(obj.shear(g1=0.1, g2=0.05), scale=0.2, dtype=np.float64, method='no_pixel')
    for i in range(3):
        one = galsim.Add(galsim.Gaussian(sigma=sig[i], flux=2.), galsim.Moffat(beta=3., fwhm=0.7).shift(0.1, 0.))
        im = one.shear(g1=0.1, g2=0.05).drawImage(scale=0.2, dtype=np.float64, method='no_pixel')
        a = st.array(i)
        assert a.shape == im.array.shape
        assert np.abs(a - im.array).max() <= 1e-14 * np.abs(im.array).max()
        assert abs(st.added_flux[i] - im.added_flux) <= 1e-12 * abs(im.added_flux)


def test_real_space_add_to_image():
    g = galsim.Gaussian(sigma=0.5)
    im = g.drawImage(nx=20, ny=20, scale=0.2, method='no_pixel', dtype=np.float64)
    im2 = g.drawImage(image=im.copy(), method='no_pixel', add_to_image=True)
    assert np.allclose(im2.array, 2. * im.array, rtol=1e-15, atol=0)
    assert abs(im2.added_flux - im.added_flux) <= 1e-14

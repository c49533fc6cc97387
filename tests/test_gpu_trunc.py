"""GPU parity of truncated Sersic profiles (sersic.py:196-265, SersicInfo with trunc > 0) against
draws and sizes made by the reference itself (tests/golden/reference_trunc.npz): the sizes from
the FP64 root finds on the device (SersicTruncatedScale, SersicIntegratedFlux), the table from
the truncated Hankel transform on the device.

Tolerances: FP32 kernels to the contract, 1e-5 x peak and 1e-6 in flux.  FP64 kernels to
2e-7 x peak and 2e-7 in flux: the reference integrates the truncated transform adaptively to a
relative error of 1e-6 (math::hankel_trunc), this library to near FP64 precision, and the two
tables differ by the reference's integration error, a few 1e-8 of the peak in the images
(the FP64 oracle, with an exact integral, shows the same difference).
"""
import os

import numpy as np
import pytest

import galsim_b200 as galsim
import make_golden as MG

pytestmark = pytest.mark.gpu
TRUNC = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'reference_trunc.npz'))


@pytest.mark.parametrize('case', MG.TRUNC_CASES, ids=[c[0] for c in MG.TRUNC_CASES])
@pytest.mark.parametrize('precision', ['fp32', 'fp64'])
def test_truncated_sersic_draw_vs_reference(case, precision):
    name, spec, nx, ny, scale, dt, off = case
    im = MG.profile(galsim, spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type, method='fft',
                                            offset=off, precision=precision)
    ref = TRUNC['draw_' + name]
    peak = np.abs(ref).max()
    ptol, ftol = (1e-5, 1e-6) if precision == 'fp32' else (2e-7, 2e-7)
    err = np.abs(im.array.astype(float) - ref).max() / peak
    assert err <= ptol, (name, precision, err)
    fref = float(TRUNC['draw_' + name + '_flux'])
    assert abs(im.added_flux - fref) <= ftol * abs(fref), (name, precision, im.added_flux, fref)


def test_truncated_sersic_sizes_vs_reference():
    for k, spec in enumerate(MG.TRUNC_SIZE_CASES):
        obj = MG.profile(galsim, spec)
        sk, mk = TRUNC['sizes'][k]
        assert abs(obj.scale_radius - TRUNC['scale_radius'][k]) <= 1e-9 * TRUNC['scale_radius'][k], spec
        assert abs(obj.flux - TRUNC['flux'][k]) <= 1e-10 * TRUNC['flux'][k], spec
        assert abs(obj.stepk - sk) <= 1e-9 * sk, spec
        assert abs(obj.maxk - mk) <= 1e-6 * mk, spec


def test_truncated_sersic_batch_matches_single_draws():
    """A batch of truncated profiles with different n and trunc (one table per (n, trunc / r0))
    draws what the one-stamp path draws."""
    n = np.array([1.2, 2.5, 4.0])
    tr = np.array([1.5, 2.0, 2.5])
    obj = galsim.Convolve(galsim.Sersic(n=n, half_light_radius=0.5, flux=100., trunc=tr),
                          galsim.Moffat(beta=3., fwhm=0.7), galsim.Pixel(0.2))
    st = galsim.draw_batch(obj, nx=40, ny=40, scale=0.2, dtype=np.float64, precision='fp64')
    for i, a in enumerate(st.arrays()):
        one = galsim.Convolve(galsim.Sersic(n=n[i], half_light_radius=0.5, flux=100., trunc=tr[i]),
                              galsim.Moffat(beta=3., fwhm=0.7), galsim.Pixel(0.2))
        im = one.drawImage(nx=40, ny=40, scale=0.2, dtype=np.float64, method='fft', precision='fp64')
        assert np.abs(a - im.array).max() <= 1e-13 * np.abs(im.array).max()


def test_truncated_sersic_argument_errors():
    with pytest.raises(galsim.GalSimRangeError):
        galsim.Sersic(n=2., half_light_radius=1., trunc=1.2)
    with pytest.raises(galsim.GalSimRangeError):
        galsim.Sersic(n=2., half_light_radius=1., trunc=-1.)

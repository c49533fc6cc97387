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


# Truncated Moffat profiles (moffat.py:79-125, SBMoffat::setupFT).  The reference's adaptive
# integral of the smooth Moffat integrand reaches near FP64 precision (the oracle's exact one
# agrees with its tables to ~1e-14), so FP64 kernels are held to the main parity tolerance,
# 1e-9 x peak and 1e-10 in flux; FP32 kernels to 1e-5 x peak and 1e-6 in flux.

@pytest.mark.parametrize('case', MG.TRUNC_MOFFAT_CASES, ids=[c[0] for c in MG.TRUNC_MOFFAT_CASES])
@pytest.mark.parametrize('precision', ['fp32', 'fp64'])
def test_truncated_moffat_draw_vs_reference(case, precision):
    name, spec, nx, ny, scale, dt, off = case
    im = MG.profile(galsim, spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type, method='fft',
                                            offset=off, precision=precision)
    ref = TRUNC['draw_' + name]
    peak = np.abs(ref).max()
    if precision == 'fp32' or dt == 'f4':
        ptol, ftol = 1e-5, 1e-6
    else:
        ptol, ftol = 1e-9, 1e-10
    err = np.abs(im.array.astype(float) - ref).max() / peak
    assert err <= ptol, (name, precision, err)
    fref = float(TRUNC['draw_' + name + '_flux'])
    assert abs(im.added_flux - fref) <= ftol * abs(fref), (name, precision, im.added_flux, fref)


@pytest.mark.parametrize('case', MG.TRUNC_MOFFAT_KIMAGE_CASES, ids=[c[0] for c in MG.TRUNC_MOFFAT_KIMAGE_CASES])
def test_truncated_moffat_kimage_vs_reference(case):
    name, spec, dk, n = case
    im = MG.profile(galsim, spec).drawKImage(nx=n, ny=n, scale=dk)
    ref = TRUNC['kimg_' + name]
    assert np.abs(im.array - ref).max() <= 1e-9 * np.abs(ref).max(), name


def test_truncated_moffat_sizes_vs_reference():
    for k, spec in enumerate(MG.TRUNC_MOFFAT_SIZE_CASES):
        obj = MG.profile(galsim, spec)
        sk, mk = TRUNC['moffat_sizes'][k]
        assert abs(obj.scale_radius - TRUNC['moffat_scale_radius'][k]) <= 1e-9 * TRUNC['moffat_scale_radius'][k], spec
        assert abs(obj.half_light_radius - TRUNC['moffat_hlr'][k]) <= 1e-9 * TRUNC['moffat_hlr'][k], spec
        assert abs(obj.stepk - sk) <= 1e-9 * sk, spec
        assert abs(obj.maxk - mk) <= 1e-7 * mk, spec


def test_truncated_moffat_table_vs_oracle():
    """The device table (nodes used, maxk) against the oracle's restatement of setupFT."""
    import specs
    from galsim_b200 import _lib
    beta = np.array([0.8, 1.05, 2.5, 4.5])
    tr = np.array([4.0, 10.95, 2.0 / 0.2712, 0.9 / 0.78])
    tabs = _lib.Tables()
    gsp = galsim.GSParams()
    tabs.build_moffat(beta, tr, gsp)
    info = tabs.moffat_info()
    for i in range(len(beta)):
        o = specs.O.OMoffat(beta[i], r0=1., trunc=tr[i])
        assert int(info[i, _lib.MH_NUSED]) == len(o.ft.x), i
        assert abs(info[i, _lib.MH_KSQMAX] - o.ft.x[-1]) <= 1e-12 * o.ft.x[-1], i
        assert abs(info[i, _lib.MH_MAXK] - o.maxk_rd) <= 1e-9 * o.maxk_rd, i
        assert abs(info[i, _lib.MH_FLUXFACTOR] - o.flux_factor) <= 1e-14 * abs(o.flux_factor), i


def test_truncated_moffat_mixed_batch_matches_single_draws():
    """A batch mixing untruncated and truncated Moffat PSFs with different beta: one table per
    truncated (beta, trunc / rD); each stamp draws what the one-stamp path draws."""
    beta = np.array([2.5, 3.0, 1.5, 4.0])
    tr = np.array([0., 1.5, 2.5, 1.5])
    obj = galsim.Convolve(galsim.Exponential(half_light_radius=0.4, flux=50.),
                          galsim.Moffat(beta=beta, fwhm=0.7, trunc=tr), galsim.Pixel(0.2))
    st = galsim.draw_batch(obj, nx=40, ny=40, scale=0.2, dtype=np.float64, precision='fp64')
    for i, a in enumerate(st.arrays()):
        one = galsim.Convolve(galsim.Exponential(half_light_radius=0.4, flux=50.),
                              galsim.Moffat(beta=beta[i], fwhm=0.7, trunc=tr[i]), galsim.Pixel(0.2))
        im = one.drawImage(nx=40, ny=40, scale=0.2, dtype=np.float64, method='fft', precision='fp64')
        assert np.abs(a - im.array).max() <= 1e-13 * np.abs(im.array).max(), i


def test_truncated_moffat_argument_errors():
    with pytest.raises(galsim.GalSimRangeError):
        galsim.Moffat(beta=1.05, fwhm=1.)                         # beta <= 1.1 needs trunc
    with pytest.raises(galsim.GalSimRangeError):
        galsim.Moffat(beta=2.5, half_light_radius=1., trunc=1.4)  # trunc <= sqrt(2) hlr
    with pytest.raises(galsim.GalSimRangeError):
        galsim.Moffat(beta=2.5, fwhm=1., trunc=-1.)
    with pytest.raises(galsim.GalSimError, match='Solve error'):
        galsim.Moffat(beta=0.8, half_light_radius=0.3, trunc=1.2)   # no bracket, as the reference
    with pytest.raises(galsim.GalSimError, match='beta'):
        galsim.Moffat(beta=1.0, scale_radius=0.3, trunc=1.2).maxk   # 0/0 normalisation
    m = galsim.Moffat(beta=2.5, fwhm=0.7, trunc=2.0)
    assert m.has_hard_edges and not galsim.Moffat(beta=2.5, fwhm=0.7).has_hard_edges
    from galsim_b200.autodiff import RecordPlan
    with pytest.raises(galsim.GalSimNotImplementedError):
        RecordPlan(galsim.Convolve(galsim.Gaussian(sigma=0.5), m), 32, 32, 0.2)

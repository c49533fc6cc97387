"""The oracle's InterpolatedImage against fixtures made by the reference itself
(tests/golden/make_golden.py main_interp).  CPU only: pins the checker of the GPU
InterpolatedImage path (k-image, k interpolation, x-interpolant transform, stepk / maxk)."""
import numpy as np
import pytest

import galsim_oracle as O
import make_golden as MG
import specs

GOLD = np.load(specs.HERE + '/reference_interp.npz')
specs.load_interp_images(GOLD)


@pytest.mark.parametrize('case', MG.INTERP_DRAW_CASES, ids=[c[0] for c in MG.INTERP_DRAW_CASES])
def test_interp_draw_matches_reference(case):
    name, spec, nx, ny, scale, dt, off = case
    arr, flux, N, Nk = O.draw_image(specs.oracle_profile(spec), nx, ny, scale, off)
    ref = GOLD['draw_' + name]
    peak = np.abs(ref).max()
    tol = 1e-12 if dt == 'f8' else 2e-7
    assert np.abs(arr.astype(ref.dtype) - ref).max() <= tol * peak
    assert abs(flux - float(GOLD['draw_' + name + '_flux'])) <= (1e-12 if dt == 'f8' else 1e-6) * abs(flux)


@pytest.mark.parametrize('case', MG.INTERP_KIMAGE_CASES, ids=[c[0] for c in MG.INTERP_KIMAGE_CASES])
def test_interp_kimage_matches_reference(case):
    name, spec, dk, n = case
    x0, y0 = GOLD['kimg_' + name + '_xmin']
    kim = O.draw_kimage(specs.oracle_profile(spec), n, n, int(x0), int(y0), dk)
    ref = GOLD['kimg_' + name]
    assert np.abs(kim - ref).max() <= 1e-12 * np.abs(ref).max()


def test_interp_sizes_match_reference():
    for spec, (sk, mk) in zip(MG.INTERP_SIZE_CASES, GOLD['sizes']):
        s, m = specs.oracle_profile(spec).stepk_maxk()
        assert s == sk, spec
        assert m == mk, spec


def test_interp_kvalue_matches_reference():
    oi = specs.oracle_profile(('ii', 'psf31x33', 0.25, {}))
    pts = GOLD['kvalue_pts']
    ref = GOLD['kvalue_ii_psf31x33']
    mine = oi.leaf.kv(pts[:, 0], pts[:, 1], True)
    assert np.abs(mine - ref).max() <= 1e-13 * np.abs(ref).max()


def test_interpolant_kernels():
    """Kernel identities the reference's interpolants satisfy: unit value at 0, zeros at the
    other integers, partition of unity, and the transform at 0 equal to the kernel's integral."""
    x = np.linspace(0., 1., 11)
    for name in ('nearest', 'linear', 'cubic', 'quintic'):
        xr = int(np.ceil(O.INTERP_XRANGE[name]))
        assert O.interp_xval(name, 0.) == 1.
        for k in range(1, xr + 1):
            assert abs(O.interp_xval(name, float(k))) < 1e-15
        if name != 'nearest':
            tot = sum(O.interp_xval(name, x - k) for k in range(-xr - 1, xr + 2))
            assert np.abs(tot - 1.).max() < 1e-14
        assert abs(O.interp_uval(name, 0.) - 1.) < 1e-15

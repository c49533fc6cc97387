"""Host-side InterpolatedImage logic (CPU, no GPU): the reference's constructor errors, the
padded frame, flux rules, interpolant parsing, and the flattened program."""
import math

import numpy as np
import pytest

import galsim_b200 as galsim
from galsim_b200 import _lib
from galsim_b200.program import Program


def _img(nx=32, ny=32, scale=0.2, seed=1):
    a = np.random.default_rng(seed).uniform(0.1, 1., (ny, nx))
    return galsim.Image(a, scale=scale)


def test_constructor_errors_follow_the_reference():
    im = _img()
    with pytest.raises(TypeError):
        galsim.InterpolatedImage(np.zeros((4, 4)))
    with pytest.raises(galsim.GalSimValueError):
        galsim.InterpolatedImage(im, normalization='counts')
    with pytest.raises(galsim.GalSimRangeError):
        galsim.InterpolatedImage(im, pad_factor=0.)
    with pytest.raises(galsim.GalSimIncompatibleValuesError):
        galsim.InterpolatedImage(im, scale=0.2, wcs=galsim.PixelScale(0.2))
    with pytest.raises(galsim.GalSimIncompatibleValuesError):
        galsim.InterpolatedImage(galsim.Image(np.ones((8, 8))))
    with pytest.raises(TypeError):
        galsim.InterpolatedImage(im, wcs=0.2)
    with pytest.raises(galsim.GalSimValueError):
        galsim.InterpolatedImage(galsim.Image(np.zeros((8, 8)), scale=0.2))
    with pytest.raises(galsim.GalSimUndefinedBoundsError):
        galsim.InterpolatedImage(galsim.Image(scale=0.2))
    # noise padding: the argument rules of _buildRealImage / _buildNoisePadImage (the Gaussian
    # padding itself is drawn on the GPU; correlated-noise padding is not built)
    with pytest.raises(galsim.GalSimIncompatibleValuesError):
        galsim.InterpolatedImage(im, noise_pad=0.1)
    with pytest.raises(galsim.GalSimIncompatibleValuesError):
        galsim.InterpolatedImage(im, noise_pad_size=10)
    with pytest.raises(galsim.GalSimValueError):
        galsim.InterpolatedImage(im, noise_pad_size=-1, noise_pad=0.1)
    with pytest.raises(galsim.GalSimRangeError):
        galsim.InterpolatedImage(im, noise_pad_size=10, noise_pad=-0.1)
    with pytest.raises(galsim.GalSimNotImplementedError):
        galsim.InterpolatedImage(im, noise_pad_size=10, noise_pad=galsim.ImageD(8, 8))
    with pytest.raises(galsim.GalSimValueError):
        galsim.InterpolatedImage(im, noise_pad_size=10, noise_pad=[1, 2])
    with pytest.raises(galsim.GalSimNotImplementedError):
        galsim.InterpolatedImage(im, depixelize=True)
    with pytest.raises(galsim.GalSimValueError):
        galsim.InterpolatedImage(im, x_interpolant='bilinear')


def test_padded_frame_and_flux():
    for nx, ny, pf, N in ((32, 32, 4., 128), (31, 33, 4., 192), (24, 24, 2., 48), (40, 37, 1., 48)):
        a = np.random.default_rng(nx).uniform(0., 1., (ny, nx))
        ii = galsim.InterpolatedImage(galsim.Image(a, scale=0.3), pad_factor=pf)
        src = ii._sources[0]
        assert src.N == N
        assert (src.x0, src.y0) == (-(nx // 2), -(ny // 2))
        assert np.array_equal(src.region, a)
        assert ii.flux == float(np.sum(a))
    a = np.random.default_rng(3).uniform(0., 1., (20, 20))
    ii = galsim.InterpolatedImage(galsim.Image(a, scale=0.5), normalization='sb')
    assert ii.flux == float(np.sum(a)) * 0.25
    assert galsim.InterpolatedImage(galsim.Image(a, scale=0.5), flux=7.).flux == 7.


def test_pad_image_region():
    a = np.random.default_rng(4).uniform(0., 1., (16, 16))
    pad = np.random.default_rng(5).uniform(0., 1e-3, (30, 30))
    ii = galsim.InterpolatedImage(galsim.Image(a, scale=0.2), pad_image=galsim.Image(pad))
    src = ii._sources[0]
    assert src.region.shape == (30, 30)
    assert (src.x0, src.y0) == (-15, -15)
    assert np.array_equal(src.region[7:23, 7:23], a)
    assert src.region[0, 0] == pad[0, 0]


def test_interpolants():
    assert galsim.Interpolant.from_name('quintic') == galsim.Quintic()
    assert galsim.Interpolant.from_name('lanczos5F') == galsim.Lanczos(5, conserve_dc=False)
    assert galsim.Interpolant.from_name('Cubic').xrange == 2.
    g = galsim.GSParams(kvalue_accuracy=1e-4)
    q = galsim.Quintic(gsparams=g)
    assert q.krange == 1.6058208066649935 / 1e-4 ** (1. / 3.)
    assert galsim.Linear().krange == 2. / 1e-5 ** 0.5
    assert galsim.Nearest().ixrange == 1 and galsim.Quintic().ixrange == 6
    assert galsim.Delta().krange == 2. * math.pi / 1e-5
    # Lanczos: the transform's extent is its table's uMax (Lanczos::urange); the transform is 1
    # at u = 0 and, conserving DC, vanishes at the other integers to the table's accuracy
    lz = galsim.Lanczos(5)
    assert lz.krange == 2. * math.pi * lz.urange and 3. < lz.urange < 6.
    assert abs(lz.uval(0.) - 1.) < 1e-5 and abs(lz.uval(1.)) < 1e-5
    assert galsim.Lanczos(3, tol=1e-4).urange < galsim.Lanczos(3).urange


def test_program_layout():
    ii = galsim.InterpolatedImage(_img())          # even size: a -0.5 offset becomes a phase
    obj = galsim.Convolve(galsim.Exponential(half_light_radius=0.5), ii)
    p = Program(obj)
    t = p.tpl
    assert list(t.leaf_type[:t.n_leaves]) == [_lib.EXPONENTIAL, _lib.INTERPOLATED]
    assert t.n_phases == 1
    rec = p.bld.leaves[1]
    assert rec['p'][0, 0] == _lib.INTERP_QUINTIC and rec['p'][0, 1] == _lib.INTERP_QUINTIC
    # image units -> world: the leaf's Jacobian is the pixel scale
    assert np.allclose(rec['jac'][0], (0.2, 0., 0., 0.2))
    assert p.bld.image_sources[1][0] is ii._sources[0]
    # a batch of two images and a single image broadcast over a batch of galaxies
    iib = galsim.InterpolatedImage([_img(seed=1), _img(24, 28, seed=2)])
    gal = galsim.Exponential(half_light_radius=np.array([0.4, 0.6]))
    p2 = Program(galsim.Convolve(gal, iib))
    assert p2.B == 2 and len(p2.bld.image_sources[1]) == 2
    # a Lanczos x interpolant is built (its transform from a device table), and a Lanczos k
    # interpolant up to n = 3 (7 taps per axis)
    p3 = Program(galsim.InterpolatedImage(_img(), x_interpolant='lanczos5', k_interpolant='lanczos3'))
    assert p3.bld.leaves[0]['p'][0, 0] == _lib.INTERP_LANCZOS
    assert p3.bld.leaves[0]['p'][0, 1] == _lib.INTERP_LANCZOS
    assert p3.bld.image_kinterp[0].n == 3
    with pytest.raises(galsim.GalSimNotImplementedError):
        Program(galsim.InterpolatedImage(_img(), k_interpolant='lanczos4'))
    with pytest.raises(galsim.GalSimNotImplementedError):
        Program(galsim.InterpolatedImage(_img(), k_interpolant='delta'))


def test_image_desc_layout_matches_the_c_struct():
    d = _lib.IMAGE_DESC_DTYPE
    assert d.itemsize == 88
    assert d.fields['pix_offset'][1] == 48 and d.fields['maxk_limit'][1] == 72
    assert d.fields['x_table'][1] == 80

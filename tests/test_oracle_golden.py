"""The FP64 oracle against fixtures made by the reference itself (tests/golden/make_golden.py).
CPU only: this pins the checker before it is used to judge the GPU kernels."""
import numpy as np
import pytest

import galsim_oracle as O
import make_golden as MG
import specs

GOLD = np.load(specs.HERE + '/reference_draws.npz')


@pytest.mark.parametrize('case', MG.DRAW_CASES, ids=[c[0] for c in MG.DRAW_CASES])
def test_draw_image_matches_reference(case):
    name, spec, nx, ny, scale, dt, off = case
    if name in ('bulge_disk_moffat_gen', 'moffat_15_dilate'):
        pytest.skip('slow in the oracle; covered by the GPU parity tests')
    arr, flux, N, Nk = O.draw_image(specs.oracle_profile(spec), nx, ny, scale, off)
    ref = GOLD['draw_' + name]
    peak = np.abs(ref).max()
    # the reference draws float32 images through complex64 k-images
    tol = 1e-12 if dt == 'f8' else 2e-7
    assert np.abs(arr.astype(ref.dtype) - ref).max() <= tol * peak
    assert abs(flux - float(GOLD['draw_' + name + '_flux'])) <= (1e-12 if dt == 'f8' else 1e-6) * abs(flux)


@pytest.mark.parametrize('case', MG.KIMAGE_CASES, ids=[c[0] for c in MG.KIMAGE_CASES])
def test_kimage_matches_reference(case):
    name, spec, dk, n = case
    x0, y0 = GOLD['kimg_' + name + '_xmin']
    kim = O.draw_kimage(specs.oracle_profile(spec), n, n, int(x0), int(y0), dk)
    ref = GOLD['kimg_' + name]
    assert np.abs(kim - ref).max() <= 1e-12 * np.abs(ref).max()


def test_leaf_sizes_match_reference():
    ref = GOLD['sizes']
    for spec, (sk, mk) in zip(MG.SIZE_CASES, ref):
        s, m = specs.oracle_profile(spec).stepk_maxk()
        # Kolmogorov's stepk goes through fmath::expd, the reference's approximate exp
        # (include/galsim/fmath/fmath.hpp:457-478), which moves it at the 1e-8 level.
        assert abs(s - sk) <= 1e-7 * sk, spec
        assert abs(m - mk) <= 1e-6 * mk, spec


def test_sersic_scale_radius():
    for n, r0 in zip((0.5, 0.8, 1.0, 1.5, 2.5, 4.0, 6.0), GOLD['sersic_r0']):
        assert abs(1. / O.sersic_info(n).re - r0) <= 1e-12 * r0


def test_good_fft_size():
    out = [O.good_fft_size(int(v)) for v in GOLD['good_fft_in']]
    assert np.array_equal(out, GOLD['good_fft_out'])


@pytest.mark.parametrize('Nk,N', [(16, 8), (20, 8), (12, 12), (24, 12)])
def test_wrap_and_irfft(Nk, N):
    kim = GOLD['wrap_in_%d_%d' % (Nk, N)].copy()
    w = O.wrap_hermx(kim, -Nk // 2, N)
    assert np.abs(w - GOLD['wrap_out_%d_%d' % (Nk, N)]).max() < 1e-12
    real = O.irfft_shifted(np.array(w), N)
    assert np.abs(real - GOLD['irfft_out_%d_%d' % (Nk, N)]).max() < 1e-12


CFG = np.load(specs.HERE + '/reference_configs.npz')


def _cfg_stamp(prefix, i):
    """Stamp i of a configuration sample: shape, (N, Nk), block, grid, flux, peak."""
    shapes = CFG[prefix + '_shape']
    bo = go = 0
    for j in range(i):
        b = min(MG.CFG_BLOCK, *shapes[j])
        bo += b * b
        go += len(range(0, shapes[j][0], MG.CFG_STRIDE)) * len(range(0, shapes[j][1], MG.CFG_STRIDE))
    b = min(MG.CFG_BLOCK, *shapes[i])
    ng = len(range(0, shapes[i][0], MG.CFG_STRIDE)) * len(range(0, shapes[i][1], MG.CFG_STRIDE))
    return (tuple(shapes[i]), tuple(CFG[prefix + '_N_Nk'][i]), CFG[prefix + '_block'][bo:bo + b * b],
            CFG[prefix + '_grid'][go:go + ng], float(CFG[prefix + '_flux'][i]), float(CFG[prefix + '_peak'][i]))


def _check_oracle_stamp(prefix, i, o, gsp):
    shape, sizes, block, grid, flux, peak = _cfg_stamp(prefix, i)
    arr, f, N, Nk = O.draw_image(o, shape[1], shape[0], 0.2, gsp=gsp)
    assert (N, Nk) == sizes
    b, g = MG.config_sample(arr)
    # float32 reference images (complex64 k-images)
    assert np.abs(b.ravel() - block).max() <= 2e-7 * peak
    assert np.abs(g.ravel() - grid).max() <= 2e-7 * peak
    assert abs(f - flux) <= 1e-6 * abs(flux)


@pytest.mark.parametrize('i', [0, 1, 2])
def test_batched_forward_sample_stamps(i):
    n, hlr, flux, g1, g2, fwhm = CFG['c2_params'][i]
    o = O.OConvolve(O.OSersic(n, hlr=hlr, flux=flux).shear(g1, g2), O.OKolmogorov(fwhm=fwhm), O.OBox(0.2))
    _check_oracle_stamp('c2', i, o, O.DEFAULT)


def test_mixed_sample_stamp_minimum_fft_size_32():
    """A bulge+disk stamp with GSParams(minimum_fft_size=32): the sizing rule below the default
    minimum (the smallest FFT size in the sample)."""
    m = MG.bench_module().mixed_params()
    sizes = CFG['c4_N_Nk'][:, 0]
    j = int(np.argmin(sizes))
    i = int(CFG['c4_index'][j])
    bulge = O.OSersic(4., hlr=m['bh'][i], flux=m['flux'][i] * m['bf'][i]).shear(*m['g_b'][i])
    disk = O.OExponential(m['dh'][i] / 1.6783469900166605, m['flux'][i] * (1. - m['bf'][i])).shear(*m['g_d'][i])
    o = O.OConvolve(O.OSum(bulge, disk), O.OMoffat(m['beta'][i], fwhm=m['fwhm'][i]), O.OBox(0.2))
    _check_oracle_stamp('c4', j, o, O.OGSParams(minimum_fft_size=32))


STD = np.load(specs.HERE + '/reference_standalone.npz')


@pytest.mark.parametrize('case', MG.STANDALONE_DRAWK, ids=[c[0] for c in MG.STANDALONE_DRAWK])
def test_drawk_with_jacobian_matches_reference(case):
    """SBProfile.drawK through the tree's _drawKImage(image, jac): the oracle's drawK with the
    same Jacobian composed as Transformation._drawKImage does."""
    name, spec, dk, b, jac, dt = case
    kim = np.zeros((b[3] - b[2] + 1, b[1] - b[0] + 1), complex)
    j = None if jac is None else np.array(jac, dtype=float).reshape(2, 2)
    specs.oracle_profile(spec).drawK(kim, b[0], b[2], dk, j)
    ref = STD['drawk_' + name]
    tol = 1e-12 if dt == 'c16' else 2e-7
    assert np.abs(kim - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.parametrize('tag', ['jac', 'nojac'])
def test_apply_phases_matches_reference(tag):
    a = STD['phase_in_' + tag].copy()
    jac = None if tag == 'nojac' else np.array((0.9, 0.3, -0.2, 1.1)).reshape(2, 2)
    O.apply_phases(a, 0, -10, 0.3, jac, 0.37, -0.61, 1.7)
    assert np.abs(a - STD['phase_out_' + tag]).max() <= 1e-12 * np.abs(a).max()


@pytest.mark.parametrize('Nx,Ny', MG.STANDALONE_IRFFT)
@pytest.mark.parametrize('si', [0, 1])
@pytest.mark.parametrize('so', [0, 1])
def test_irfft_flags_match_reference(Nx, Ny, si, so):
    """irfft's shift_in / shift_out (Image.cpp:848-898) restated with numpy: the rows taken in
    FFT order, the (-1)^(i+j) factor, then a c2r transform (which ignores the imaginary parts of
    the kx = 0 and Nx/2 columns after the y transform)."""
    k = STD['irfft_in_%d_%d' % (Nx, Ny)]
    K = np.concatenate([k[Ny // 2:], k[:Ny // 2]], axis=0) if si else k.copy()
    if so:
        r = np.arange(Ny)[:, None]
        c = np.arange(Nx // 2 + 1)[None, :]
        K = K * np.where((r + c) % 2 == 0, 1., -1.)
    out = np.fft.irfft2(K, s=(Ny, Nx))
    ref = STD['irfft_out_%d_%d_%d%d' % (Nx, Ny, si, so)]
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()


TRUNC = np.load(specs.HERE + '/reference_trunc.npz')


@pytest.mark.parametrize('case', MG.TRUNC_CASES, ids=[c[0] for c in MG.TRUNC_CASES])
def test_truncated_sersic_draw_matches_reference(case):
    """Truncated Sersic profiles: the oracle's exact truncated Hankel transform against the
    reference's adaptive Gauss-Kronrod-Patterson one (relerr 1e-6) -- they agree to the
    reference's integration error, a few 1e-8 of the peak."""
    name, spec, nx, ny, scale, dt, off = case
    arr, flux, N, Nk = O.draw_image(specs.oracle_profile(spec), nx, ny, scale, off)
    ref = TRUNC['draw_' + name]
    peak = np.abs(ref).max()
    assert np.abs(arr.astype(ref.dtype) - ref).max() <= 2e-7 * peak
    assert abs(flux - float(TRUNC['draw_' + name + '_flux'])) <= 2e-7 * abs(flux)


def test_truncated_sersic_sizes_match_reference():
    for k, spec in enumerate(MG.TRUNC_SIZE_CASES):
        o = specs.oracle_profile(spec)
        s, m = o.stepk_maxk()
        sk, mk = TRUNC['sizes'][k]
        assert abs(s - sk) <= 1e-9 * sk, spec
        assert abs(m - mk) <= 1e-6 * mk, spec
        assert abs(o.r0 - TRUNC['scale_radius'][k]) <= 1e-9 * o.r0, spec
        assert abs(o.flux - TRUNC['flux'][k]) <= 1e-10 * o.flux, spec


@pytest.mark.parametrize('case', MG.TRUNC_MOFFAT_CASES, ids=[c[0] for c in MG.TRUNC_MOFFAT_CASES])
def test_truncated_moffat_draw_matches_reference(case):
    """Truncated Moffat profiles: the oracle's spline over k^2 of the exact truncated Hankel
    transform against the reference's spline of its adaptive one (relerr 1e-6)."""
    name, spec, nx, ny, scale, dt, off = case
    arr, flux, N, Nk = O.draw_image(specs.oracle_profile(spec), nx, ny, scale, off)
    ref = TRUNC['draw_' + name]
    peak = np.abs(ref).max()
    assert np.abs(arr.astype(ref.dtype) - ref).max() <= 2e-7 * peak
    assert abs(flux - float(TRUNC['draw_' + name + '_flux'])) <= 2e-7 * abs(flux)


def test_truncated_moffat_sizes_match_reference():
    for k, spec in enumerate(MG.TRUNC_MOFFAT_SIZE_CASES):
        o = specs.oracle_profile(spec)
        s, m = o.stepk_maxk()
        sk, mk = TRUNC['moffat_sizes'][k]
        assert abs(s - sk) <= 1e-9 * sk, spec
        assert abs(m - mk) <= 1e-6 * mk, spec
        assert abs(o.r0 - TRUNC['moffat_scale_radius'][k]) <= 1e-9 * o.r0, spec


@pytest.mark.parametrize('case', MG.TRUNC_MOFFAT_KIMAGE_CASES, ids=[c[0] for c in MG.TRUNC_MOFFAT_KIMAGE_CASES])
def test_truncated_moffat_kimage_matches_reference(case):
    """k-values of truncated Moffat profiles on odd grids centred on k = 0, out to beyond the
    table's last argument (where the reference returns 0)."""
    name, spec, dk, n = case
    kim = O.draw_kimage(specs.oracle_profile(spec), n, n, -(n // 2), -(n // 2), dk)
    ref = TRUNC['kimg_' + name]
    assert np.abs(kim - ref).max() <= 1e-12 * np.abs(ref).max()


REAL = np.load(specs.HERE + '/reference_real.npz')
specs.load_interp_images(np.load(specs.HERE + '/reference_interp.npz'))    # the 'ii' cases' images


@pytest.mark.parametrize('case', MG.REAL_CASES, ids=[c[0] for c in MG.REAL_CASES])
def test_real_space_draw_matches_reference(case):
    """drawImage with method 'no_pixel' / 'sb' on analytic profiles (drawReal): the oracle's
    restatement of the _drawReal walk and the profiles' xValues against the reference."""
    name, spec, nx, ny, scale, dt, method, off = case
    arr, flux = O.draw_image_real(specs.oracle_profile(spec), nx, ny, scale, off, method)
    ref = REAL['draw_' + name]
    tol = 2e-7 if dt == 'f4' else (1e-10 if 'kolm' in name else 1e-12)
    assert np.abs(arr.astype(ref.dtype).astype(float) - ref).max() <= tol * np.abs(ref).max(), name
    assert abs(flux - float(REAL['draw_' + name + '_flux'])) <= max(tol, 1e-7 if dt == 'f4' else 0) * abs(flux)

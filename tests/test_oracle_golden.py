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

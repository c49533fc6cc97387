"""GPU parity of the large-FFT path (1024 < N <= 16384; the precision-study configuration:
Sersic n 3..5.5 with an obscured Airy at 0.05" pixels, images of 1200 to 5150 pixels) against
fixtures drawn by the reference itself (tests/golden/reference_large.npz: the central 64 x 64
block, a strided pixel grid and the added flux of each image).

Tolerances: pixels max |diff| <= 1e-5 x peak for the FP32 kernels (and for float32 images,
which the reference itself computes with complex64 k-images), <= 1e-9 x peak for the FP64
kernels on float64 images; added flux <= 1e-6 relative for FP32 kernels and float32 images,
<= 1e-10 relative for FP64 kernels on float64 images.  (The FP32 Airy k-value is evaluated
as lens areas through atan2: the reference's asin(h / r) form, rounded to FP32, drops the
first-order term of the disc overlap on the innermost k rings of these grids, dk ~ 5e-4,
which had biased the FP32 flux by 1e-5 .. 1e-4.)
"""
import os

import numpy as np
import pytest

import galsim_b200 as galsim
import make_golden as MG

pytestmark = pytest.mark.gpu
LARGE = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'reference_large.npz'))


@pytest.mark.parametrize('case', MG.LARGE_CASES, ids=[c[0] for c in MG.LARGE_CASES])
@pytest.mark.parametrize('precision', ['fp32', 'fp64'])
def test_large_fft_draw_vs_reference(case, precision):
    name, spec, nx, ny, scale, dt = case
    im = MG.profile(galsim, spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type,
                                            method='fft', precision=precision)
    key = 'large_' + name
    assert tuple(im.array.shape) == tuple(LARGE[key + '_shape'])
    block, grid = MG.large_sample(im.array)
    peak = float(LARGE[key + '_peak'])
    tol = 1e-5 if (precision == 'fp32' or dt == 'f4') else 1e-9
    err = max(np.abs(block.astype(float) - LARGE[key + '_block']).max(),
              np.abs(grid.astype(float) - LARGE[key + '_grid']).max())
    assert err <= tol * peak, (name, precision, err / peak)
    fref = float(LARGE[key + '_flux'])
    ftol = 1e-6 if (precision == 'fp32' or dt == 'f4') else 1e-10
    assert abs(im.added_flux - fref) <= ftol * abs(fref), (name, precision, im.added_flux, fref)

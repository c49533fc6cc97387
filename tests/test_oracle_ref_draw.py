"""The CPU reference arm's orchestration (oracle/ref_draw.py: drawFFT restated over the
reference's own C++ drawK / ApplyKImagePhases / wrapImage / irfft / stepK / maxK in
oracle/_ref/libgsref.so) against stamps drawn by the reference's own Python drawImage
(tests/golden/reference_configs.npz): same automatic image size, same (N, Nk), pixels to the
float32 rounding of the fixture.  CPU only; skipped when libgsref.so is not built."""
import numpy as np
import pytest

import ref_draw as R
import test_oracle_golden as TG

pytestmark = pytest.mark.skipif(not R.available(), reason='oracle/_ref/libgsref.so not built')


@pytest.mark.parametrize('i', [0, 1, 2, 3, 4, 5])
def test_reference_arm_stamp_matches_reference_drawimage(i):
    n, hlr, flux, g1, g2, fwhm = TG.CFG['c2_params'][i]
    shape, sizes, block, grid, fref, peak = TG._cfg_stamp('c2', i)
    arr, f, N, Nk = R.draw_image(R.c2_profile(n, hlr, flux, g1, g2, fwhm, 0.2), None, None, 0.2)
    assert arr.shape == shape
    assert (N, Nk) == sizes
    b, g = TG.MG.config_sample(arr)
    assert np.abs(b.ravel() - block).max() <= 2e-7 * peak
    assert np.abs(g.ravel() - grid).max() <= 2e-7 * peak
    assert abs(f - fref) <= 1e-6 * abs(fref)

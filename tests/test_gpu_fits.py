"""FITS file images of stamp batches made on the device (gsb_fits_pack): byte for byte the file
the host writer makes from the same stamps (fits.writeMulti / writeCube of StampBatch.images()),
and read back to the drawn pixels, for FP32 and FP64 batches, auto-sized (ragged) and fixed
stamps."""
import numpy as np
import pytest

import galsim_b200 as galsim
from galsim_b200 import fits

pytestmark = pytest.mark.gpu


def _batch(dtype, nx=None):
    hlr = np.array([0.3, 0.5, 0.9, 1.4, 0.6])
    gal = galsim.Sersic(n=np.array([1., 2.5, 4., 1.5, 3.]), half_light_radius=hlr, flux=1e3)
    obj = galsim.Convolve(gal, galsim.Moffat(beta=3., fwhm=0.7))
    return galsim.draw_batch(obj, nx=nx, ny=nx, scale=0.2, dtype=dtype)


@pytest.mark.parametrize('dtype', [np.float32, np.float64])
def test_multi_file_image_matches_host_writer(tmp_path, dtype):
    sb = _batch(dtype)                      # automatic sizes: the stamps differ in size
    assert len(set(np.asarray(sb.nx).tolist())) > 1
    dev = sb.fits_bytes()
    host_file = str(tmp_path / 'host.fits')
    fits.writeMulti(sb.images(), host_file)
    assert dev == open(host_file, 'rb').read()
    f = str(tmp_path / 'dev.fits.gz')
    sb.writeMulti(f)
    back = fits.readMulti(f)
    assert len(back) == len(sb)
    for i, im in enumerate(back):
        np.testing.assert_array_equal(im.array, sb.array(i))
        assert im.array.dtype == dtype
        assert im.wcs == galsim.PixelScale(0.2)


@pytest.mark.parametrize('dtype', [np.float32, np.float64])
def test_cube_file_image_matches_host_writer(tmp_path, dtype):
    sb = _batch(dtype, nx=40)
    dev = sb.fits_bytes(cube=True)
    host_file = str(tmp_path / 'host.fits')
    fits.writeCube(sb.images(), host_file)
    assert dev == open(host_file, 'rb').read()
    f = str(tmp_path / 'cube.fits')
    galsim.fits.writeCube(sb, f)
    back = fits.readCube(f)
    for i, im in enumerate(back):
        np.testing.assert_array_equal(im.array, sb.array(i))


def test_ragged_batch_is_not_a_cube():
    with pytest.raises(galsim.GalSimValueError):
        _batch(np.float32).fits_bytes(cube=True)

"""FITS files (CPU): the reader against the reference's own FITS test files (the files its
test_image.py reads, kept as bytes in tests/golden/reference_fits.npz by make_golden.py
main_fits; they hold the 5 x 7 array that test states), write / read round trips of every
Image type, multi-extension files and cubes, file compression, header cards, and the
reference's error behaviour (fits.py)."""
import os

import numpy as np
import pytest

import galsim_b200 as galsim
from galsim_b200 import fits

GOLD = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'reference_fits.npz'))

# test_image.py's ref_array: the contents of the testS/I/F/D/US/UI fixture files
REF_ARRAY = (np.arange(1, 8)[None, :] * 10 + np.arange(1, 6)[:, None]).astype(np.int16)
TYPES = (('S', np.int16), ('I', np.int32), ('F', np.float32), ('D', np.float64),
         ('US', np.uint16), ('UI', np.uint32))


def test_ref_array_restatement():
    assert REF_ARRAY[0].tolist() == [11, 21, 31, 41, 51, 61, 71]
    assert REF_ARRAY[:, 0].tolist() == [11, 12, 13, 14, 15]


def _fixture(tmp_path, name):
    path = str(tmp_path / name)
    with open(path, 'wb') as f:
        f.write(GOLD[name.replace('.', '_')].tobytes())
    return path


@pytest.mark.parametrize('tchar,dt', TYPES)
@pytest.mark.parametrize('ext', ['', '.gz', '.bz2'])
def test_read_reference_fixtures(tmp_path, tchar, dt, ext):
    path = _fixture(tmp_path, 'test%s.fits%s' % (tchar, ext))
    im = fits.read(path)
    assert im.array.dtype == dt
    np.testing.assert_array_equal(im.array, REF_ARRAY.astype(dt))
    assert im.bounds == galsim.BoundsI(1, 7, 1, 5)
    # the same through an explicit compression and through an HDUList
    comp = {'': None, '.gz': 'gzip', '.bz2': 'bzip2'}[ext]
    np.testing.assert_array_equal(fits.read(path, compression=comp).array, REF_ARRAY.astype(dt))
    hl = fits.readFile(path)
    np.testing.assert_array_equal(fits.read(hdu_list=hl).array, REF_ARRAY.astype(dt))


def test_reference_header_cards(tmp_path):
    h = fits.FitsHeader(file_name=_fixture(tmp_path, 'testD.fits'))
    assert h['BITPIX'] == -64 and h['NAXIS1'] == 7 and h['NAXIS2'] == 5
    assert h['SIMPLE'] is True


@pytest.mark.parametrize('dt', [t[1] for t in TYPES])
def test_write_read_round_trip(tmp_path, dt):
    a = REF_ARRAY.astype(dt)
    for xmin, ymin, scale in ((1, 1, 0.2), (-3, 7, 0.35), (1, 1, None)):
        im = galsim.Image(a, xmin=xmin, ymin=ymin, scale=scale)
        f = str(tmp_path / 'rt.fits')
        im.write(f)
        back = fits.read(f)
        assert back.array.dtype == a.dtype
        np.testing.assert_array_equal(back.array, a)
        assert back.bounds == im.bounds
        if scale is None:
            assert back.wcs == galsim.PixelScale(1.)      # no WCS keys: unit pixel scale
        else:
            assert back.wcs == galsim.PixelScale(scale)
        raw = open(f, 'rb').read()
        assert len(raw) % fits.BLOCK == 0


def test_reference_header_keys(tmp_path):
    f = str(tmp_path / 'h.fits')
    galsim.Image(REF_ARRAY.astype(np.float32), scale=0.2).write(f)
    h = fits.read(f, read_header=True).header
    assert h['GS_XMIN'] == 1 and h['GS_YMIN'] == 1
    assert h['GS_WCS'] == 'PixelScale' and h['GS_SCALE'] == 0.2
    assert h['CTYPE1'] == 'LINEAR' and h['CD1_1'] == 0.2 and h['CD2_2'] == 0.2
    assert h['CD1_2'] == 0. and h['CRPIX1'] == 0.
    galsim.Image(REF_ARRAY.astype(np.float32), xmin=-2, ymin=4, scale=0.3).write(f)
    h = fits.read(f, read_header=True).header
    assert h['GS_WCS'] == 'OffsetWCS'
    assert (h['GS_X0'], h['GS_Y0']) == (3, -3)
    assert (h['CRPIX1'], h['CRPIX2']) == (3, -3)


def test_multi_and_cube(tmp_path):
    rng = np.random.default_rng(3)
    ims = [galsim.Image(rng.normal(size=(ny, nx)).astype(np.float32), scale=0.2)
           for nx, ny in ((10, 12), (7, 7), (33, 20))]
    for ext in ('fits', 'fits.gz', 'fits.bz2'):
        f = str(tmp_path / ('m.' + ext))
        fits.writeMulti(ims, f)
        back = fits.readMulti(f)
        assert len(back) == 3
        for a, b in zip(ims, back):
            np.testing.assert_array_equal(a.array, b.array)
            assert b.wcs == galsim.PixelScale(0.2)
    same = [galsim.Image(rng.normal(size=(9, 11)), scale=0.5) for _ in range(4)]
    f = str(tmp_path / 'c.fits')
    fits.writeCube(same, f)
    back = fits.readCube(f)
    assert len(back) == 4
    for a, b in zip(same, back):
        np.testing.assert_array_equal(a.array, b.array)
        assert b.wcs == galsim.PixelScale(0.5)
    fits.writeCube(np.stack([s.array for s in same]), f)
    np.testing.assert_array_equal(fits.readCube(f)[2].array, same[2].array)
    with pytest.raises(galsim.GalSimValueError):
        fits.writeCube(same[:2] + [galsim.Image(np.zeros((3, 3)))], f)
    with pytest.raises(galsim.GalSimValueError):
        fits.writeCube([], f)


def test_hdu_list_and_write_file(tmp_path):
    hl = fits.HDUList()
    fits.write(galsim.Image(REF_ARRAY.astype(np.int32)), hdu_list=hl)
    fits.write(galsim.Image(REF_ARRAY.astype(np.float64) * 0.5, scale=0.1), hdu_list=hl)
    f = str(tmp_path / 'hl.fits')
    fits.writeFile(f, hl)
    back = fits.readMulti(f)
    np.testing.assert_array_equal(back[0].array, REF_ARRAY)
    np.testing.assert_array_equal(back[1].array, REF_ARRAY * 0.5)
    np.testing.assert_array_equal(fits.read(f, hdu=1).array, REF_ARRAY * 0.5)


def test_errors_follow_the_reference(tmp_path):
    f = str(tmp_path / 'e.fits')
    im = galsim.Image(REF_ARRAY.astype(np.float32))
    im.write(f)
    with pytest.raises(ValueError):
        fits.read(f, compression='invalid')
    with pytest.raises(ValueError):
        im.write(f, compression='invalid')
    with pytest.raises(OSError):
        fits.read(f, compression='rice')
    with pytest.raises(OSError):
        fits.read(str(tmp_path / 'invalid.fits'))
    with pytest.raises(OSError):
        fits.read(f, hdu=1)
    with pytest.raises(TypeError):
        fits.read()
    with pytest.raises(TypeError):
        fits.read(f, hdu_list=fits.HDUList())
    with pytest.raises(TypeError):
        im.write()
    with pytest.raises(OSError):
        im.write(f, clobber=False)
    with pytest.raises(ValueError):
        galsim.Image(np.ones((3, 3), np.complex128)).write(f)
    with pytest.raises(galsim.GalSimNotImplementedError):
        im.write(str(tmp_path / 'e.fits.fz'))


def test_header_cards():
    c = fits._card('GS_SCALE', 0.2, 'GalSim image scale')
    assert len(c) == 80 and c.startswith('GS_SCALE= ') and c[10:30].strip() == '0.2'
    assert c[30:].startswith(' / GalSim image scale')
    assert fits._card('NAXIS1', 7)[10:30] == ' ' * 19 + '7'
    assert fits._card('SIMPLE', True)[29] == 'T'
    s = fits._card('CTYPE1', 'LINEAR')
    assert s[10:20] == "'LINEAR  '"
    for x in (0.1, 1e-300, -2.5e17, 1 / 3., 12345.678, 0., 7.):
        v = fits._parse_value(fits._format_value(x))[0]
        assert v == x and isinstance(v, float)
    assert fits._parse_value(fits._format_value("it's"))[0] == "it's"
    h = fits.FitsHeader({'A': 1, 'B': (2.5, 'two and a half')})
    assert h['A'] == 1 and h.comment('B') == 'two and a half' and 'a' in h
    h['A'] = 3
    assert h.keys() == ['A', 'B'] and h['A'] == 3
    del h['A']
    assert len(h) == 1 and h.get('A', 'x') == 'x'
    h.extend({'C': 'text'})
    assert h.items() == [('B', 2.5), ('C', 'text')]
    hdu = fits.PrimaryHDU(np.zeros((2, 3), np.float32), h)
    text = hdu.header_bytes().decode()
    assert len(text) == fits.BLOCK
    cards = [text[i:i + 80] for i in range(0, len(text), 80)]
    keys = [c[:8].strip() for c in cards]
    assert keys[:6] == ['SIMPLE', 'BITPIX', 'NAXIS', 'NAXIS1', 'NAXIS2', 'EXTEND']
    assert 'END' in keys and keys.index('B') < keys.index('END')

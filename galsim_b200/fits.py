"""FITS files of Images and stamp batches (galsim/fits.py, galsim/fitsheader.py).

The reference reads and writes FITS through astropy.io.fits; here the format itself is
written and parsed (FITS Standard 4.0: 80-byte header cards in 2880-byte blocks, big-endian
data padded to a block), so that no astropy is needed:

* ``write`` / ``writeMulti`` / ``writeCube`` / ``writeFile`` and ``read`` / ``readMulti`` /
  ``readCube`` / ``readFile`` with the reference's arguments, errors and file compression
  ('gzip', 'bzip2', or chosen from the extension).  Tile compression ('rice', 'gzip_tile',
  'hcompress', 'plio', the '.fz' files) is not built and raises GalSimNotImplementedError.
* The header keys the reference writes for an Image: GS_XMIN / GS_YMIN and the WCS of a
  PixelScale image (wcs.py:720-770, 1582-1585, 2083-2090, 2287-2298); reading maps GS_WCS
  PixelScale / OffsetWCS back to a PixelScale (a header is never evaluated as code).
* ``FitsHeader``: the reference's dict-like header (fitsheader.py).
* Stamp batches leave the device as a finished file image: ``StampBatch.writeMulti`` /
  ``writeCube`` (galsim_b200/batch.py) build every header here and let ``gsb_fits_pack``
  (csrc/gsb_fits.cu) place headers, byte-swapped pixels and block padding in one device buffer,
  which is read back once and written with one call.

``HDUList``, ``PrimaryHDU`` and ``ImageHDU`` stand in for astropy's classes where the
reference's functions take or return an ``hdu_list``.
"""
import bz2
import gzip
import os

import numpy as np

from .errors import (GalSimIncompatibleValuesError, GalSimNotImplementedError,
                     GalSimValueError, galsim_warn)

BLOCK = 2880
CARD = 80

# BITPIX of each numpy type; unsigned types are stored signed with BZERO (FITS Standard 5.3)
_BITPIX = {np.dtype(np.uint8): 8, np.dtype(np.int16): 16, np.dtype(np.int32): 32,
           np.dtype(np.int64): 64, np.dtype(np.float32): -32, np.dtype(np.float64): -64,
           np.dtype(np.uint16): 16, np.dtype(np.uint32): 32}
_BZERO = {np.dtype(np.uint16): 32768, np.dtype(np.uint32): 2147483648}
_FROM_BITPIX = {8: '>u1', 16: '>i2', 32: '>i4', 64: '>i8', -32: '>f4', -64: '>f8'}
_STRUCTURAL = ('SIMPLE', 'XTENSION', 'BITPIX', 'NAXIS', 'EXTEND', 'PCOUNT', 'GCOUNT', 'BZERO',
               'BSCALE', 'END')
_COMMENTARY = ('COMMENT', 'HISTORY', '')


# ------------------------------------------------------------------------------------------
# Header cards
# ------------------------------------------------------------------------------------------
def _format_float(x):
    """A float in the fixed-format value field: the shortest representation that reads back
    to the same double, with a decimal point and an 'E' exponent, at most 20 characters."""
    if not np.isfinite(x):
        raise GalSimValueError("FITS header values must be finite", x)
    s = repr(float(x)).upper()
    if 'E' in s:
        mant, ex = s.split('E')
        if '.' not in mant:
            mant += '.0'
        sign = '-' if ex.startswith('-') else '+'
        s = mant + 'E' + sign + ex.lstrip('+-').zfill(2)
    elif '.' not in s:
        s += '.0'
    if len(s) > 20:
        digits = 16
        while len(s) > 20 and digits > 1:
            s = '%.*E' % (digits, x)
            digits -= 1
    return s


def _format_value(v):
    if isinstance(v, (bool, np.bool_)):
        return ('T' if v else 'F').rjust(20)
    if isinstance(v, (int, np.integer)):
        return str(int(v)).rjust(20)
    if isinstance(v, (float, np.floating)):
        return _format_float(float(v)).rjust(20)
    if isinstance(v, str):
        s = "'" + v.replace("'", "''").ljust(8) + "'"
        if len(s) > 70:
            raise GalSimValueError("FITS string value too long for one card", v)
        return s.ljust(20)
    if v is None:
        return ' ' * 20
    raise GalSimValueError("Unsupported FITS header value type", v)


def _card(key, value, comment=''):
    """One 80-character card (FITS Standard 4.1-4.2)."""
    key = key.upper()
    if key in _COMMENTARY:
        return (key.ljust(8) + str(value))[:CARD].ljust(CARD)
    if len(key) > 8 or not all(c.isalnum() or c in '-_' for c in key):
        head = 'HIERARCH ' + key + ' = '
    else:
        head = key.ljust(8) + '= '
    card = head + _format_value(value)
    if comment:
        card += ' / ' + comment
    if len(card) > CARD:
        if len(head) + len(_format_value(value).rstrip()) > CARD:
            raise GalSimValueError("FITS header card too long", (key, value))
        card = card[:CARD]
    return card.ljust(CARD)


def _parse_value(s):
    """Value and comment of the value field of a card (the text after '= ')."""
    s = s.strip()
    if s.startswith("'"):
        i, out = 1, []
        while i < len(s):
            if s[i] == "'":
                if i + 1 < len(s) and s[i + 1] == "'":
                    out.append("'")
                    i += 2
                    continue
                break
            out.append(s[i])
            i += 1
        rest = s[i + 1:]
        comment = rest.split('/', 1)[1].strip() if '/' in rest else ''
        return ''.join(out).rstrip(), comment
    val, _, comment = s.partition('/')
    val = val.strip()
    comment = comment.strip()
    if val == 'T':
        return True, comment
    if val == 'F':
        return False, comment
    if val == '':
        return None, comment
    try:
        return int(val), comment
    except ValueError:
        pass
    try:
        return float(val.replace('D', 'E')), comment
    except ValueError:
        raise OSError("Unparseable FITS header value: %r" % val)


class FitsHeader(object):
    """A FITS header as an ordered mapping of keys to values with comments (fitsheader.py).

    FitsHeader(header) copies a dict, a list of (key, value[, comment]) items or another
    FitsHeader; FitsHeader(file_name=...) reads the header of one HDU of a file."""

    def __init__(self, header=None, file_name=None, dir=None, hdu_list=None, hdu=None,
                 compression='auto', text_file=False):
        self._cards = []       # [KEY, value, comment]
        if header is not None and (file_name is not None or hdu_list is not None):
            raise GalSimIncompatibleValuesError(
                "Cannot provide both header and file_name or hdu_list", header=header,
                file_name=file_name, hdu_list=hdu_list)
        if file_name is not None or hdu_list is not None:
            if text_file:
                path = os.path.join(dir, file_name) if dir else file_name
                with open(path) as f:
                    text = f.read().replace('\n', '')
                header = _parse_header_text(text)
            else:
                hl = hdu_list
                if file_name is not None:
                    hl = readFile(file_name, dir, hdu, compression)
                h = 0 if hdu is None else hdu
                if isinstance(hl, _HDU):
                    header = hl.header
                else:
                    if len(hl) <= h:
                        raise OSError('Expecting at least %d HDUs in FitsHeader' % (h + 1))
                    header = hl[h].header
        if header is not None:
            self.extend(header)

    def _index(self, key):
        key = key.upper()
        for i, c in enumerate(self._cards):
            if c[0] == key:
                return i
        return -1

    def __getitem__(self, key):
        i = self._index(key)
        if i < 0:
            raise KeyError(key)
        return self._cards[i][1]

    def __setitem__(self, key, value):
        comment = ''
        if isinstance(value, tuple):
            value, comment = value[0], (value[1] if len(value) > 1 else '')
        key = key.upper()
        i = self._index(key)
        if i >= 0 and key not in _COMMENTARY:
            self._cards[i][1] = value
            if comment:
                self._cards[i][2] = comment
        else:
            self._cards.append([key, value, comment])

    def __delitem__(self, key):
        i = self._index(key)
        if i < 0:
            raise KeyError(key)
        del self._cards[i]

    def __contains__(self, key):
        return self._index(key) >= 0

    def __len__(self):
        return len(self._cards)

    def __iter__(self):
        return iter(self.keys())

    def __eq__(self, other):
        return isinstance(other, FitsHeader) and self.items() == other.items()

    def __ne__(self, other):
        return not self.__eq__(other)

    __hash__ = None

    def get(self, key, default=None):
        i = self._index(key)
        return self._cards[i][1] if i >= 0 else default

    def comment(self, key):
        i = self._index(key)
        if i < 0:
            raise KeyError(key)
        return self._cards[i][2]

    def keys(self):
        return [c[0] for c in self._cards]

    def values(self):
        return [c[1] for c in self._cards]

    def items(self):
        return [(c[0], c[1]) for c in self._cards]

    def cards(self):
        return [tuple(c) for c in self._cards]

    def append(self, key, value, comment='', useblanks=True):
        self._cards.append([key.upper(), value, comment])

    def extend(self, other, useblanks=True, update=False):
        """Add the cards of another header (dict, list of items, or FitsHeader); with
        update=True a key already present is overwritten instead of repeated."""
        if isinstance(other, FitsHeader):
            items = other.cards()
        elif isinstance(other, dict):
            items = list(other.items())
        else:
            items = list(other)
        for it in items:
            key = it[0]
            val = it[1:] if len(it) > 2 else it[1]
            if update or key.upper() not in self:
                self[key] = val if isinstance(val, tuple) else (val,)
            else:
                v = val if isinstance(val, tuple) else (val,)
                self._cards.append([key.upper(), v[0], v[1] if len(v) > 1 else ''])

    def update(self, dict2):
        for k, v in (dict2.items() if hasattr(dict2, 'items') else dict2):
            self[k] = v

    def pop(self, key, default=None):
        i = self._index(key)
        if i < 0:
            return default
        return self._cards.pop(i)[1]

    def clear(self):
        self._cards = []

    def __repr__(self):
        return 'galsim.FitsHeader(header=%r)' % [tuple(c) for c in self._cards]


def _parse_header_text(text):
    """Cards of a header given as text (80-character cards up to END)."""
    cards = []
    for i in range(0, len(text), CARD):
        c = text[i:i + CARD]
        key = c[:8].strip().upper()
        if key == 'END':
            break
        if key in _COMMENTARY:
            if key or c.strip():
                cards.append((key, c[8:].rstrip(), ''))
            continue
        if key == 'HIERARCH':
            k, _, v = c[9:].partition('=')
            val, com = _parse_value(v)
            cards.append((k.strip().upper(), val, com))
            continue
        if c[8:10] != '= ':
            cards.append(('COMMENT', c[8:].rstrip(), ''))
            continue
        val, com = _parse_value(c[10:])
        cards.append((key, val, com))
    return cards


# ------------------------------------------------------------------------------------------
# HDUs
# ------------------------------------------------------------------------------------------
class _HDU(object):
    _primary = False

    def __init__(self, data=None, header=None):
        if data is not None:
            data = np.asarray(data)
            if data.dtype.kind == 'c':
                raise GalSimValueError("Cannot write complex data to a fits file", data.dtype)
            if data.dtype.newbyteorder('=') not in _BITPIX:
                data = data.astype(np.float64)
        self.data = data
        self.header = FitsHeader(header) if header is not None else FitsHeader()

    def structural_cards(self):
        """The mandatory cards in the order the standard requires (4.4.1)."""
        d = self.data
        shape = () if d is None else d.shape[::-1]
        dt = np.dtype(np.uint8) if d is None else d.dtype.newbyteorder('=')
        if self._primary:
            cards = [('SIMPLE', True, 'conforms to FITS standard')]
        else:
            cards = [('XTENSION', 'IMAGE', 'Image extension')]
        cards.append(('BITPIX', _BITPIX[dt], 'array data type'))
        cards.append(('NAXIS', len(shape), 'number of array dimensions'))
        for i, n in enumerate(shape):
            cards.append(('NAXIS%d' % (i + 1), int(n), ''))
        if self._primary:
            cards.append(('EXTEND', True, ''))
        else:
            cards.append(('PCOUNT', 0, 'number of parameters'))
            cards.append(('GCOUNT', 1, 'number of groups'))
        if dt in _BZERO:
            cards.append(('BZERO', _BZERO[dt], ''))
            cards.append(('BSCALE', 1, ''))
        return cards

    def header_bytes(self):
        cards = [_card(*c) for c in self.structural_cards()]
        for key, val, com in self.header.cards():
            if key in _STRUCTURAL or (key.startswith('NAXIS') and key[5:].isdigit()):
                continue
            cards.append(_card(key, val, com))
        cards.append('END'.ljust(CARD))
        text = ''.join(cards)
        text += ' ' * (-len(text) % BLOCK)
        return text.encode('ascii')

    def data_bytes(self):
        d = self.data
        if d is None or d.size == 0:
            return b''
        dt = d.dtype.newbyteorder('=')
        if dt in _BZERO:
            d = (d.astype(np.int64) - _BZERO[dt]).astype(_FROM_BITPIX[_BITPIX[dt]])
        else:
            d = d.astype(dt.newbyteorder('>'))
        b = np.ascontiguousarray(d).tobytes()
        return b + b'\0' * (-len(b) % BLOCK)

    def tobytes(self):
        return self.header_bytes() + self.data_bytes()


class PrimaryHDU(_HDU):
    _primary = True


class ImageHDU(_HDU):
    _primary = False


class HDUList(list):
    """A list of HDUs (the first a PrimaryHDU) that can be written as one file."""

    def writeto(self, file_name, overwrite=False):
        writeFile(file_name, self, clobber=overwrite, compression=None)

    def close(self):
        pass


def _file_bytes(hdu_list):
    out = []
    for i, h in enumerate(hdu_list):
        if i == 0 and not h._primary:
            p = PrimaryHDU(h.data, h.header)
            out.append(p.tobytes())
        elif i > 0 and h._primary:
            e = ImageHDU(h.data, h.header)
            out.append(e.tobytes())
        else:
            out.append(h.tobytes())
    return b''.join(out)


def _parse_file(raw):
    """The HDUs of a FITS file image (image HDUs; other extensions are kept as header-only
    HDUs with data None)."""
    hdus = []
    pos = 0
    n = len(raw)
    while pos + BLOCK <= n:
        cards = []
        end = False
        while not end:
            if pos + BLOCK > n:
                raise OSError("Truncated FITS header")
            blk = raw[pos:pos + BLOCK].decode('ascii', errors='replace')
            pos += BLOCK
            for i in range(0, BLOCK, CARD):
                if blk[i:i + 8].strip() == 'END' and blk[i:i + 8].rstrip() == 'END':
                    end = True
                    break
            cards.append(blk)
        parsed = _parse_header_text(''.join(cards))
        h = dict((k, v) for k, v, _ in parsed if k not in _COMMENTARY)
        if not hdus and 'SIMPLE' not in h:
            raise OSError("Not a FITS file (no SIMPLE card)")
        bitpix = int(h.get('BITPIX', 8))
        naxis = int(h.get('NAXIS', 0))
        shape = [int(h.get('NAXIS%d' % (i + 1), 0)) for i in range(naxis)]
        nelem = int(np.prod(shape)) if naxis else 0
        nbytes = abs(bitpix) // 8 * int(h.get('GCOUNT', 1)) * (int(h.get('PCOUNT', 0)) + nelem)
        is_image = not hdus or str(h.get('XTENSION', '')).strip() == 'IMAGE'
        data = None
        if is_image and nelem > 0:
            if bitpix not in _FROM_BITPIX or pos + abs(bitpix) // 8 * nelem > n:
                raise OSError("Invalid FITS image data")
            data = np.frombuffer(raw, dtype=_FROM_BITPIX[bitpix], count=nelem, offset=pos)
            data = data.reshape(shape[::-1])
            bzero = h.get('BZERO', 0)
            bscale = h.get('BSCALE', 1)
            if bscale == 1 and bitpix == 16 and bzero == 32768:
                data = (data.astype(np.int32) + 32768).astype(np.uint16)
            elif bscale == 1 and bitpix == 32 and bzero == 2147483648:
                data = (data.astype(np.int64) + 2147483648).astype(np.uint32)
            elif bscale == 1 and bitpix == 8 and bzero == -128:
                data = (data.astype(np.int16) - 128).astype(np.int8)
            elif bscale != 1 or bzero != 0:
                data = data.astype(np.float64) * bscale + bzero
            else:
                data = data.astype(data.dtype.newbyteorder('='))
        hdu = (PrimaryHDU if not hdus else ImageHDU)()
        hdu.data = data
        hdu.header = FitsHeader(parsed)
        hdu._is_image = is_image
        hdus.append(hdu)
        pos += nbytes + (-nbytes % BLOCK)
    if not hdus:
        raise OSError("Empty or invalid FITS file")
    return HDUList(hdus)


# ------------------------------------------------------------------------------------------
# Compression and files
# ------------------------------------------------------------------------------------------
_TILE = ('rice', 'gzip_tile', 'hcompress', 'plio')


def _parse_compression(compression, file_name):
    """(file_compress, tile_compress) as in fits.py _parse_compression."""
    if compression == 'rice' or compression == 'RICE_1':
        return None, 'RICE_1'
    if compression == 'gzip_tile' or compression == 'GZIP_1':
        return None, 'GZIP_1'
    if compression == 'hcompress' or compression == 'HCOMPRESS_1':
        return None, 'HCOMPRESS_1'
    if compression == 'plio' or compression == 'PLIO_1':
        return None, 'PLIO_1'
    if compression == 'gzip':
        return 'gzip', None
    if compression == 'bzip2':
        return 'bzip2', None
    if compression == 'none' or compression is None:
        return None, None
    if compression == 'auto':
        if file_name:
            if file_name.lower().endswith('.fz'):
                return None, 'RICE_1'
            if file_name.lower().endswith('.gz'):
                return 'gzip', None
            if file_name.lower().endswith('.bz2'):
                return 'bzip2', None
        return None, None
    raise GalSimValueError("Invalid compression", compression,
                           ('rice', 'gzip_tile', 'hcompress', 'plio', 'gzip', 'bzip2', 'none',
                            'auto'))


def _no_tiles(tile_compress):
    if tile_compress:
        raise GalSimNotImplementedError(
            "Tile-compressed FITS (%s) is not built; use compression 'gzip', 'bzip2' or None"
            % tile_compress)


def _path(file_name, dir):
    return os.path.join(dir, file_name) if dir else file_name


def _write_bytes(file_name, dir, data, clobber, file_compress):
    path = _path(file_name, dir)
    d = os.path.dirname(path)
    if d and not os.path.exists(d):
        os.makedirs(d)
    if os.path.isfile(path):
        if clobber:
            os.remove(path)
        else:
            raise OSError('File %r already exists' % path)
    if file_compress == 'gzip':
        with gzip.open(path, 'wb') as f:
            f.write(data)
    elif file_compress == 'bzip2':
        with bz2.BZ2File(path, 'wb') as f:
            f.write(data)
    else:
        with open(path, 'wb') as f:
            f.write(data)


def _read_bytes(file_name, dir, file_compress):
    path = _path(file_name, dir)
    if not os.path.isfile(path):
        raise OSError("File %r not found" % path)
    if file_compress == 'gzip':
        with gzip.open(path, 'rb') as f:
            return f.read()
    if file_compress == 'bzip2':
        with bz2.BZ2File(path, 'rb') as f:
            return f.read()
    with open(path, 'rb') as f:
        return f.read()


def readFile(file_name, dir=None, hdu=None, compression='auto'):
    """The HDUList of a FITS file (fits.py readFile; here the list is the parsed file)."""
    file_compress, tile = _parse_compression(compression, file_name)
    _no_tiles(tile)
    return _parse_file(_read_bytes(file_name, dir, file_compress))


def writeFile(file_name, hdu_list, dir=None, clobber=True, compression='auto'):
    """Write an HDUList to a file (fits.py:650-701)."""
    file_compress, tile = _parse_compression(compression, file_name)
    _no_tiles(tile)
    _write_bytes(file_name, dir, _file_bytes(hdu_list), clobber, file_compress)


def closeHDUList(hdu_list, fin=None):
    """Nothing stays open here; kept for the reference's calling pattern."""


# ------------------------------------------------------------------------------------------
# Image headers (wcs.py writeToFitsHeader / readFromFitsHeader for a PixelScale)
# ------------------------------------------------------------------------------------------
def image_header_cards(bounds, wcs, header=None):
    """The cards the reference adds for an Image: its extra header, then GS_XMIN / GS_YMIN and
    the WCS.  A PixelScale image whose origin is not (1, 1) is written as the reference's
    shifted OffsetWCS (origin 1 - xmin, 1 - ymin)."""
    h = FitsHeader(header) if header is not None else FitsHeader()
    if wcs is None:
        return h
    from .wcs import PixelScale
    if not isinstance(wcs, PixelScale):
        raise GalSimNotImplementedError("Only a PixelScale WCS is written to FITS here")
    h['GS_XMIN'] = (int(bounds.xmin), 'GalSim image minimum x coordinate')
    h['GS_YMIN'] = (int(bounds.ymin), 'GalSim image minimum y coordinate')
    s = wcs.scale
    if bounds.xmin != 1 or bounds.ymin != 1:
        x0, y0 = 1 - int(bounds.xmin), 1 - int(bounds.ymin)
        h['GS_WCS'] = ('OffsetWCS', 'GalSim WCS name')
        h['GS_SCALE'] = (s, 'GalSim image scale')
        h['GS_X0'] = (x0, 'GalSim image origin x')
        h['GS_Y0'] = (y0, 'GalSim image origin y')
        h['GS_U0'] = (0., 'GalSim world origin u')
        h['GS_V0'] = (0., 'GalSim world origin v')
    else:
        x0 = y0 = 0.
        h['GS_WCS'] = ('PixelScale', 'GalSim WCS name')
        h['GS_SCALE'] = (s, 'GalSim image scale')
    h['CTYPE1'] = ('LINEAR', 'name of the world coordinate axis')
    h['CTYPE2'] = ('LINEAR', 'name of the world coordinate axis')
    h['CRVAL1'] = (0., 'world coordinate at reference pixel = u0')
    h['CRVAL2'] = (0., 'world coordinate at reference pixel = v0')
    h['CRPIX1'] = (x0, 'image coordinate of reference pixel = x0')
    h['CRPIX2'] = (y0, 'image coordinate of reference pixel = y0')
    h['CD1_1'] = (s, 'CD1_1 = dudx')
    h['CD1_2'] = (0., 'CD1_2 = dudy')
    h['CD2_1'] = (0., 'CD2_1 = dvdx')
    h['CD2_2'] = (s, 'CD2_2 = dvdy')
    return h


def _wcs_from_header(header, suppress_warning=True):
    """(wcs, origin) of a header (wcs.py readFromFitsHeader) for the WCS types built here."""
    from .position import _PositionI
    from .wcs import PixelScale
    xmin = int(header.get('GS_XMIN', 1))
    ymin = int(header.get('GS_YMIN', 1))
    name = header.get('GS_WCS', None)
    wcs = None
    if name == 'PixelScale':
        wcs = PixelScale(header['GS_SCALE'])
    elif name == 'OffsetWCS':
        # The origin written is 1 - xmin (the shift applied on writing); reading shifts back,
        # which leaves a plain pixel scale when the world origin is 0.
        if (header.get('GS_X0', 0) + xmin - 1 == 0 and header.get('GS_Y0', 0) + ymin - 1 == 0 and
                header.get('GS_U0', 0.) == 0. and header.get('GS_V0', 0.) == 0.):
            wcs = PixelScale(header['GS_SCALE'])
    elif name is None:
        cd11 = header.get('CD1_1', header.get('CDELT1', None))
        cd22 = header.get('CD2_2', header.get('CDELT2', None))
        cross = header.get('CD1_2', 0.) or header.get('CD2_1', 0.)
        if cd11 is None and cd22 is None:
            wcs = PixelScale(1.)
        elif cd11 == cd22 and not cross:
            wcs = PixelScale(cd11)
    if wcs is None:
        if not suppress_warning:
            galsim_warn("The WCS of this FITS header is not built here; the image has no WCS")
    return wcs, _PositionI(xmin, ymin)


def _image_hdu_cls(first):
    return PrimaryHDU if first else ImageHDU


def _image_hdu(image, first):
    if image.iscomplex:
        raise GalSimValueError("Cannot write complex Images to a fits file. "
                               "Write image.real and image.imag separately.", image)
    hdr = image_header_cards(image.bounds, image.wcs, getattr(image, 'header', None))
    return _image_hdu_cls(first)(image.array, hdr)


def _target(file_name, hdu_list):
    if file_name and hdu_list is not None:
        raise GalSimIncompatibleValuesError(
            "Cannot provide both file_name and hdu_list", file_name=file_name, hdu_list=hdu_list)
    if not (file_name or hdu_list is not None):
        raise GalSimIncompatibleValuesError(
            "Must provide either file_name or hdu_list", file_name=file_name, hdu_list=hdu_list)


# ------------------------------------------------------------------------------------------
# Writers
# ------------------------------------------------------------------------------------------
def write(image, file_name=None, dir=None, hdu_list=None, clobber=True, compression='auto'):
    """Write one Image to a FITS file, or append it to an HDUList (fits.py:378-443)."""
    if image.iscomplex:
        raise GalSimValueError("Cannot write complex Images to a fits file. "
                               "Write image.real and image.imag separately.", image)
    file_compress, tile = _parse_compression(compression, file_name)
    _target(file_name, hdu_list)
    _no_tiles(tile)
    hl = HDUList() if hdu_list is None else hdu_list
    hl.append(_image_hdu(image, len(hl) == 0))
    if file_name:
        _write_bytes(file_name, dir, _file_bytes(hl), clobber, file_compress)


def writeMulti(image_list, file_name=None, dir=None, hdu_list=None, clobber=True,
               compression='auto'):
    """Write a list of Images as a multi-extension FITS file (fits.py:445-527).  A
    StampBatch is written from the device (StampBatch.writeMulti)."""
    from .image import Image
    if hasattr(image_list, 'writeMulti') and not isinstance(image_list, (list, tuple)):
        if hdu_list is not None:
            raise GalSimNotImplementedError("A StampBatch is written to a file, not an hdu_list")
        return image_list.writeMulti(file_name, dir=dir, clobber=clobber, compression=compression)
    if any(im.iscomplex for im in image_list if isinstance(im, Image)):
        raise GalSimValueError("Cannot write complex Images to a fits file. "
                               "Write image.real and image.imag separately.", image_list)
    file_compress, tile = _parse_compression(compression, file_name)
    _target(file_name, hdu_list)
    _no_tiles(tile)
    hl = HDUList() if hdu_list is None else hdu_list
    for im in image_list:
        if isinstance(im, Image):
            hl.append(_image_hdu(im, len(hl) == 0))
        else:
            hl.append(im)
    if file_name:
        _write_bytes(file_name, dir, _file_bytes(hl), clobber, file_compress)


def writeCube(image_list, file_name=None, dir=None, hdu_list=None, clobber=True,
              compression='auto'):
    """Write Images of one size (or numpy arrays) as a data cube (fits.py:529-648); the header
    carries the first image's bounds and WCS."""
    if hasattr(image_list, 'writeCube') and not isinstance(image_list, (list, tuple, np.ndarray)):
        if hdu_list is not None:
            raise GalSimNotImplementedError("A StampBatch is written to a file, not an hdu_list")
        return image_list.writeCube(file_name, dir=dir, clobber=clobber, compression=compression)
    if isinstance(image_list, np.ndarray):
        is_all_numpy = True
        if image_list.dtype.kind == 'c':
            raise GalSimValueError("Cannot write complex numpy arrays to a fits file. "
                                   "Write array.real and array.imag separately.", image_list)
    elif len(image_list) == 0:
        raise GalSimValueError("In writeCube: image_list has no images", image_list)
    elif all(isinstance(item, np.ndarray) for item in image_list):
        is_all_numpy = True
        if any(a.dtype.kind == 'c' for a in image_list):
            raise GalSimValueError("Cannot write complex numpy arrays to a fits file. "
                                   "Write array.real and array.imag separately.", image_list)
    else:
        is_all_numpy = False
        if any(im.iscomplex for im in image_list):
            raise GalSimValueError("Cannot write complex images to a fits file. "
                                   "Write image.real and image.imag separately.", image_list)
    file_compress, tile = _parse_compression(compression, file_name)
    _target(file_name, hdu_list)
    _no_tiles(tile)
    hl = HDUList() if hdu_list is None else hdu_list
    if is_all_numpy:
        cube = np.asarray(image_list)
        hdr = None
    else:
        im0 = image_list[0]
        nx = im0.xmax - im0.xmin + 1
        ny = im0.ymax - im0.ymin + 1
        cube = np.zeros((len(image_list), ny, nx), dtype=im0.array.dtype)
        for k, im in enumerate(image_list):
            nx_k = im.xmax - im.xmin + 1
            ny_k = im.ymax - im.ymin + 1
            if nx_k != nx or ny_k != ny:
                raise GalSimValueError("In writeCube: image %d has the wrong shape. "
                                       "Shape is (%d,%d) should be (%d,%d)" % (k, nx_k, ny_k, nx, ny),
                                       im)
            cube[k] = im.array
        hdr = image_header_cards(im0.bounds, im0.wcs, getattr(im0, 'header', None))
    hl.append(_image_hdu_cls(len(hl) == 0)(cube, hdr))
    if file_name:
        _write_bytes(file_name, dir, _file_bytes(hl), clobber, file_compress)


# ------------------------------------------------------------------------------------------
# Readers
# ------------------------------------------------------------------------------------------
def _source(file_name, dir, hdu_list, compression):
    file_compress, tile = _parse_compression(compression, file_name)
    if file_name and hdu_list is not None:
        raise GalSimIncompatibleValuesError(
            "Cannot provide both file_name and hdu_list", file_name=file_name, hdu_list=hdu_list)
    if not (file_name or hdu_list is not None):
        raise GalSimIncompatibleValuesError(
            "Must provide either file_name or hdu_list", file_name=file_name, hdu_list=hdu_list)
    if file_name:
        if tile:
            path = _path(file_name, dir)
            if not os.path.isfile(path):
                raise OSError("File %r not found" % path)
            hl = _parse_file(_read_bytes(file_name, dir, file_compress))
            if len(hl) <= 1 or not str(hl[1].header.get('ZCMPTYPE', '')):
                raise OSError('Found invalid HDU type reading FITS file (expected a CompImageHDU)')
            _no_tiles(tile)
        return _parse_file(_read_bytes(file_name, dir, file_compress)), tile
    return hdu_list, tile


def _pick(hl, hdu):
    if isinstance(hl, _HDU):
        return hl
    if hdu is None:
        hdu = 0
    if len(hl) <= hdu:
        raise OSError('Expecting at least %d HDUs in galsim.read' % (hdu + 1))
    h = hl[hdu]
    if not getattr(h, '_is_image', True):
        raise OSError('Found invalid HDU type reading FITS file (expected an ImageHDU)')
    return h


def _to_image(hdu, read_header, suppress_warning):
    from .image import Image
    if hdu.data is None:
        raise OSError("HDU is empty.  (data is None)")
    wcs, origin = _wcs_from_header(hdu.header, suppress_warning)
    data = hdu.data
    if data.dtype.type not in Image._valid_dtypes:
        galsim_warn("No Image type for data type %s. Using numpy.float64 instead." % data.dtype)
        data = data.astype(np.float64)
    im = Image(array=data)
    im.setOrigin(origin)
    im.wcs = wcs
    if read_header:
        im.header = FitsHeader(hdu.header)
    return im


def read(file_name=None, dir=None, hdu_list=None, hdu=None, compression='auto',
         read_header=False, suppress_warning=True):
    """One Image from a FITS file or HDUList (fits.py:703-801)."""
    hl, _ = _source(file_name, dir, hdu_list, compression)
    return _to_image(_pick(hl, hdu), read_header, suppress_warning)


def readMulti(file_name=None, dir=None, hdu_list=None, compression='auto', read_headers=False,
              suppress_warning=True):
    """Every HDU of a multi-extension FITS file as an Image (fits.py:803-901); as there, an
    HDU without image data raises OSError."""
    if file_name is None and hdu_list is not None and not isinstance(hdu_list, HDUList):
        raise TypeError("In readMulti, hdu_list is not an HDUList")
    hl, _ = _source(file_name, dir, hdu_list, compression)
    if len(hl) < 1:
        raise OSError('Expecting at least one HDU in galsim.readMulti')
    return [_to_image(_pick(hl, i), read_headers, suppress_warning) for i in range(len(hl))]


def readCube(file_name=None, dir=None, hdu_list=None, hdu=None, compression='auto',
             suppress_warning=True):
    """The images of a data cube (fits.py:903-1000): a list of Images sharing the header's
    bounds and WCS."""
    from .image import Image
    hl, _ = _source(file_name, dir, hdu_list, compression)
    h = _pick(hl, hdu)
    if h.data is None:
        raise OSError("HDU is empty.  (data is None)")
    wcs, origin = _wcs_from_header(h.header, suppress_warning)
    cube = h.data if h.data.ndim == 3 else h.data[None]
    out = []
    for k in range(cube.shape[0]):
        im = Image(array=np.ascontiguousarray(cube[k]))
        im.setOrigin(origin)
        im.wcs = wcs
        out.append(im)
    return out


__all__ = ['FitsHeader', 'HDUList', 'PrimaryHDU', 'ImageHDU', 'write', 'writeMulti', 'writeCube',
           'writeFile', 'read', 'readMulti', 'readCube', 'readFile', 'closeHDUList']

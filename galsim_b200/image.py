"""Image: a numpy array with integer bounds and a pixel-scale WCS (galsim/image.py).

Only what the FFT drawing path and its users need is built: construction from
(ncol, nrow) / bounds / array, views, sub-images, centre handling, arithmetic used by
drawImage (copy / add), and good_fft_size.  Pixel data stay in host numpy arrays, as in the
reference; the drawing kernels write into device buffers that are copied back.
"""
import numpy as np

from .bounds import BoundsI, _BoundsI
from .errors import (GalSimImmutableError, GalSimIncompatibleValuesError, GalSimValueError,
                     GalSimUndefinedBoundsError)
from .position import PositionI, _PositionI, parse_pos_args
from .wcs import BaseWCS, PixelScale


class Image(object):
    _valid_dtypes = (np.uint16, np.uint32, np.int16, np.int32, np.float32, np.float64,
                     np.complex64, np.complex128)
    _alias_dtypes = {int: np.int32, float: np.float64, complex: np.complex128, np.int64: np.int32}

    def __init__(self, *args, **kwargs):
        ncol = nrow = array = bounds = image = None
        dtype = kwargs.pop('dtype', None)
        init_value = kwargs.pop('init_value', None)
        xmin = kwargs.pop('xmin', 1)
        ymin = kwargs.pop('ymin', 1)
        make_const = kwargs.pop('make_const', False)
        copy = kwargs.pop('copy', False)
        scale = kwargs.pop('scale', None)
        wcs = kwargs.pop('wcs', None)
        if len(args) == 2:
            ncol, nrow = args
        elif len(args) == 1:
            if isinstance(args[0], np.ndarray):
                array = args[0]
            elif isinstance(args[0], BoundsI):
                bounds = args[0]
            elif isinstance(args[0], Image):
                image = args[0]
            else:
                raise TypeError("Unable to parse %s as an array, bounds, or image." % args[0])
        elif len(args) > 2:
            raise TypeError("Error, too many unnamed arguments to Image constructor")
        ncol = kwargs.pop('ncol', ncol)
        nrow = kwargs.pop('nrow', nrow)
        bounds = kwargs.pop('bounds', bounds)
        array = kwargs.pop('array', array)
        image = kwargs.pop('image', image)
        if kwargs:
            raise TypeError("Image constructor got unexpected keyword arguments: %s" % kwargs)
        if dtype is not None:
            dtype = self._alias_dtypes.get(dtype, dtype)
            dtype = np.dtype(dtype).type
            if dtype not in self._valid_dtypes:
                raise GalSimValueError("Invalid dtype.", dtype, self._valid_dtypes)
        if array is not None:
            if dtype is None:
                dtype = array.dtype.type
                if dtype not in self._valid_dtypes:
                    dtype = self._alias_dtypes.get(dtype, np.float64)
            self._array = np.array(array, dtype=dtype, copy=True) if (copy or array.dtype.type != dtype) \
                else array
            self._bounds = _BoundsI(xmin, xmin + array.shape[1] - 1, ymin, ymin + array.shape[0] - 1)
        elif image is not None:
            dtype = dtype or image.dtype
            self._array = np.array(image.array, dtype=dtype, copy=True)
            self._bounds = image.bounds
            if wcs is None and scale is None:
                wcs = image.wcs
        else:
            dtype = dtype or np.float32
            if ncol is not None or nrow is not None:
                if ncol is None or nrow is None:
                    raise GalSimIncompatibleValuesError("Both nrow and ncol must be provided",
                                                        ncol=ncol, nrow=nrow)
                if ncol != int(ncol) or nrow != int(nrow):
                    raise TypeError("nrow, ncol must be integers")
                ncol, nrow = int(ncol), int(nrow)
                self._bounds = _BoundsI(xmin, xmin + ncol - 1, ymin, ymin + nrow - 1)
            elif bounds is not None:
                if not isinstance(bounds, BoundsI):
                    raise TypeError("bounds must be a galsim.BoundsI instance")
                self._bounds = bounds
            else:
                self._bounds = BoundsI()
            shape = self._bounds.numpyShape()
            self._array = np.zeros(shape, dtype=dtype)
            if init_value:
                self._array[:] = init_value
        if scale is not None:
            if wcs is not None:
                raise GalSimIncompatibleValuesError("Cannot provide both scale and wcs to Image "
                                                    "constructor", wcs=wcs, scale=scale)
            wcs = PixelScale(scale)
        if wcs is not None and not isinstance(wcs, BaseWCS):
            raise TypeError("wcs parameters must be a galsim.BaseWCS instance")
        self.wcs = wcs
        self._is_const = make_const

    # -- basic properties --------------------------------------------------------------
    @property
    def array(self):
        return self._array

    @property
    def bounds(self):
        return self._bounds

    @property
    def dtype(self):
        return self._array.dtype.type

    @property
    def iscomplex(self):
        return self._array.dtype.kind == 'c'

    @property
    def isinteger(self):
        return self._array.dtype.kind in ('i', 'u')

    @property
    def isconst(self):
        return self._is_const

    @property
    def iscontiguous(self):
        return self._array.flags.c_contiguous

    @property
    def xmin(self):
        return self._bounds.xmin

    @property
    def xmax(self):
        return self._bounds.xmax

    @property
    def ymin(self):
        return self._bounds.ymin

    @property
    def ymax(self):
        return self._bounds.ymax

    @property
    def ncol(self):
        return self._array.shape[1]

    @property
    def nrow(self):
        return self._array.shape[0]

    @property
    def center(self):
        return self._bounds.center

    @property
    def true_center(self):
        return self._bounds.true_center

    @property
    def scale(self):
        if self.wcs is None:
            return None
        if not self.wcs._isPixelScale:
            raise GalSimValueError("image.wcs is not a simple PixelScale; scale is undefined.",
                                   self.wcs)
        return self.wcs.scale

    @scale.setter
    def scale(self, value):
        if self.wcs is not None and not self.wcs._isPixelScale:
            raise GalSimValueError("Cannot set scale when wcs is not a simple PixelScale", self.wcs)
        self.wcs = None if value is None else PixelScale(value)

    @property
    def real(self):
        return _Image(self._array.real, self._bounds, self.wcs)

    @property
    def imag(self):
        return _Image(self._array.imag, self._bounds, self.wcs)

    # -- geometry ----------------------------------------------------------------------
    def _view(self):
        return _Image(self._array.view(), self._bounds, self.wcs)

    def view(self, scale=None, wcs=None, dtype=None, make_const=False):
        ret = _Image(self._array.view() if dtype is None else self._array.astype(dtype),
                     self._bounds, self.wcs)
        if scale is not None:
            ret.scale = scale
        if wcs is not None:
            ret.wcs = wcs
        ret._is_const = make_const
        return ret

    def shift(self, *args, **kwargs):
        delta = parse_pos_args(args, kwargs, 'dx', 'dy', integer=True)
        self._shift(delta)

    def _shift(self, delta):
        if delta.x != 0 or delta.y != 0:
            self._bounds = self._bounds.shift(delta)

    def setCenter(self, *args, **kwargs):
        cen = parse_pos_args(args, kwargs, 'xcen', 'ycen', integer=True)
        self._shift(cen - self.center)

    def setOrigin(self, *args, **kwargs):
        origin = parse_pos_args(args, kwargs, 'x0', 'y0', integer=True)
        self._shift(origin - _PositionI(self.xmin, self.ymin))

    def resize(self, bounds, wcs=None):
        if not isinstance(bounds, BoundsI):
            raise TypeError("bounds must be a galsim.BoundsI instance")
        self._array = np.zeros(bounds.numpyShape(), dtype=self.dtype)
        self._bounds = bounds
        if wcs is not None:
            self.wcs = wcs

    def subImage(self, bounds):
        if not isinstance(bounds, BoundsI):
            raise TypeError("bounds must be a galsim.BoundsI instance")
        if not self._bounds.includes(bounds):
            raise GalSimValueError("Attempt to access subImage not (fully) in image", bounds)
        i1 = bounds.ymin - self.ymin
        i2 = bounds.ymax - self.ymin + 1
        j1 = bounds.xmin - self.xmin
        j2 = bounds.xmax - self.xmin + 1
        return _Image(self._array[i1:i2, j1:j2], bounds, self.wcs)

    def __getitem__(self, b):
        if isinstance(b, BoundsI):
            return self.subImage(b)
        return self.getValue(*b) if isinstance(b, tuple) else self.getValue(b.x, b.y)

    def getValue(self, x, y):
        return self._array[y - self.ymin, x - self.xmin]

    __call__ = lambda self, *args: (self.getValue(*args) if len(args) == 2 else
                                    self.getValue(args[0].x, args[0].y))

    def setValue(self, x, y, value):
        self._array[y - self.ymin, x - self.xmin] = value

    # -- arithmetic used by drawImage ------------------------------------------------------
    def setZero(self):
        if self._is_const:
            raise GalSimImmutableError("Cannot modify an immutable Image", self)
        self._array[...] = 0

    def fill(self, value):
        self._array[...] = value

    def copyFrom(self, rhs):
        if self._is_const:
            raise GalSimImmutableError("Cannot modify an immutable Image", self)
        if self._bounds.numpyShape() != rhs.bounds.numpyShape():
            raise GalSimIncompatibleValuesError("Trying to copy images that are not the same shape",
                                                self_image=self, rhs=rhs)
        self._copyFrom(rhs)

    def _copyFrom(self, rhs):
        self._array[...] = rhs.array

    def copy(self):
        return _Image(self._array.copy(), self._bounds, self.wcs)

    def addNoise(self, noise):
        """Add noise to the image (image.py addNoise, noise.py:31-39); drawn on the GPU."""
        noise.applyTo(self)

    def write(self, file_name=None, dir=None, hdu_list=None, clobber=True, compression='auto'):
        """Write the image to a FITS file (galsim.fits.write, fits.py:378-443)."""
        from . import fits
        fits.write(self, file_name, dir, hdu_list, clobber, compression)

    def __iadd__(self, other):
        self._array += other.array if isinstance(other, Image) else other
        return self

    def __isub__(self, other):
        self._array -= other.array if isinstance(other, Image) else other
        return self

    def __imul__(self, other):
        self._array *= other.array if isinstance(other, Image) else other
        return self

    def __itruediv__(self, other):
        self._array /= other.array if isinstance(other, Image) else other
        return self

    @classmethod
    def good_fft_size(cls, input_size):
        """Round up to the next 2^k or 3 * 2^k (image.py:1018-1025, via goodFFTSize)."""
        from . import _lib
        return _lib.good_fft_size(int(input_size))

    def __repr__(self):
        return 'galsim.Image(bounds=%r, array=\n%r, wcs=%r)' % (self._bounds, self._array, self.wcs)


def _Image(array, bounds, wcs):
    ret = Image.__new__(Image)
    ret._array = array
    ret._bounds = bounds
    ret.wcs = wcs
    ret._is_const = False
    return ret


def ImageF(*args, **kwargs):
    kwargs['dtype'] = np.float32
    return Image(*args, **kwargs)


def ImageD(*args, **kwargs):
    kwargs['dtype'] = np.float64
    return Image(*args, **kwargs)


def ImageI(*args, **kwargs):
    kwargs['dtype'] = np.int32
    return Image(*args, **kwargs)


def ImageS(*args, **kwargs):
    kwargs['dtype'] = np.int16
    return Image(*args, **kwargs)


def ImageCF(*args, **kwargs):
    kwargs['dtype'] = np.complex64
    return Image(*args, **kwargs)


def ImageCD(*args, **kwargs):
    kwargs['dtype'] = np.complex128
    return Image(*args, **kwargs)


__all__ = ['Image', '_Image', 'ImageF', 'ImageD', 'ImageI', 'ImageS', 'ImageCF', 'ImageCD']

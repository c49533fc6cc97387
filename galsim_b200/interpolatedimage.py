"""InterpolatedImage: a surface-brightness profile interpolated from an image
(galsim/interpolatedimage.py:37-1000, src/SBInterpolatedImage.cpp).

The constructor follows the reference's argument handling, padding and flux rules on the host
(image placement in the zero-padded frame, image flux, errors).  Everything numerical runs on
the GPU: the DFT of each padded image (its k-image, FP64 with an FP32 copy), the stepk radius
scan (CalculateSizeContainingFlux), the maxk scan (calculateMaxK) and, at draw time, the
k interpolation times the x interpolant's transform inside the fused drawing kernels
(galsim_b200/csrc/gsb_images.cu, gsb_interp.cuh).  Like the reference, the profile is the
image-unit SBInterpolatedImage shifted by -offset and mapped to world coordinates by the WCS
(interpolatedimage.py:481-500): here a Transformation of one GSB_INTERPOLATED leaf.

Batches: `image` may be a list of Images (every option applies to each); the object is then
a batch of len(image) profiles, each with its own padded frame.  A single image broadcasts
against batched objects it is combined with.

Noise padding with Gaussian noise of a given variance (noise_pad a number) fills its square of
the frame with the reference's stream (BaseDeviate(rng), drawn on the GPU) before the pad image
and the image are placed.  Not built: padding with correlated noise (a CorrelatedNoise, an
image or a file), depixelize, FITS file names, non-PixelScale WCS, and sinc or Lanczos(n > 3)
as the k interpolant (sinc as the x interpolant is built: its transform is the box |u| < 1/2,
and its infinite support makes stepk tiny unless forced).
"""
import math

import numpy as np

from . import _lib
from .bounds import _BoundsI
from .errors import (GalSimIncompatibleValuesError, GalSimNotImplementedError, GalSimRangeError,
                     GalSimUndefinedBoundsError, GalSimValueError)
from .gsobject import GSObject
from .gsparams import GSParams
from .image import Image
from .interpolant import Delta, Lanczos, Quintic, SincInterpolant, convert_interpolant
from .position import _PositionD
from .wcs import BaseWCS, PixelScale


class _ImageSource(object):
    """One image placed in its padded frame: the nonzero region's pixels and frame position,
    and the scan settings for its stepk / maxk (one gsb_image_desc)."""

    def __init__(self, region, N, x0, y0, stepk_bounds, x_code, flags, nz_flux, stepk_target,
                 maxk_limit, x_interpolant=None):
        self.region = np.ascontiguousarray(region, dtype=np.float64)
        self.N = int(N)
        self.x0, self.y0 = int(x0), int(y0)
        self.stepk_bounds = stepk_bounds
        self.x_code = int(x_code)
        self.flags = int(flags)
        self.nz_flux = float(nz_flux)
        self.stepk_target = float(stepk_target)
        self.maxk_limit = float(maxk_limit)
        self.x_interpolant = x_interpolant   # a Lanczos x interpolant carries a device table

    def desc(self, pix_offset):
        d = np.zeros((), dtype=_lib.IMAGE_DESC_DTYPE)
        d['N'] = self.N
        d['ny'], d['nx'] = self.region.shape
        d['x0'], d['y0'] = self.x0, self.y0
        d['bx0'], d['bx1'], d['by0'], d['by1'] = self.stepk_bounds
        d['x_interp'] = self.x_code
        d['flags'] = self.flags
        d['pix_offset'] = pix_offset
        d['flux'] = self.nz_flux
        d['stepk_target'] = self.stepk_target
        d['maxk_limit'] = self.maxk_limit
        d['x_table'] = (self.x_interpolant._table.device().data_ptr()
                        if isinstance(self.x_interpolant, Lanczos) else 0)
        return d


class _ImageLeaf(GSObject):
    """The image-unit SBInterpolatedImage leaf (batched over its sources)."""
    _is_analytic_x = True

    def __init__(self, sources, x_interpolant, k_interpolant, gsparams):
        self._sources = sources
        self._x_interpolant = x_interpolant
        self._k_interpolant = k_interpolant
        self._gsparams = gsparams
        self._flux = np.array([s.region.sum() for s in sources]) if len(sources) > 1 else \
            float(sources[0].region.sum())
        self._batch = len(sources)

    def _flatten(self, bld, jac):
        xi, ki = self._x_interpolant, self._k_interpolant
        if (xi._code is None or ki._code is None or isinstance(ki, (Delta, SincInterpolant)) or
                (isinstance(ki, Lanczos) and ki.n > 3)):
            raise GalSimNotImplementedError(
                "InterpolatedImage with x interpolant %s and k interpolant %s is not built on the "
                "GPU (x: Delta, Nearest, Linear, Cubic, Quintic, Lanczos, Sinc; k: Nearest, Linear, "
                "Cubic, Quintic, Lanczos(n <= 3))" % (xi, ki))
        bld.add_leaf(_lib.INTERPOLATED, jac, 1., (float(xi._code), float(ki._code), 0.))
        bld.image_sources[len(bld.leaves) - 1] = self._sources
        # a Lanczos k interpolant's coefficient block goes into p[2] when the records are
        # uploaded (Program.upload), where the device exists
        bld.image_kinterp[len(bld.leaves) - 1] = ki if isinstance(ki, Lanczos) else None

    def withGSParams(self, gsparams=None, **kwargs):
        return self


class InterpolatedImage(GSObject):
    """A profile interpolated from an image (interpolatedimage.py:37-300 for the arguments)."""
    _has_hard_edges = False
    _is_axisymmetric = False
    _is_analytic_x = True
    _is_analytic_k = True

    def __init__(self, image, x_interpolant=None, k_interpolant=None, normalization='flux',
                 scale=None, wcs=None, flux=None, pad_factor=4., noise_pad_size=0, noise_pad=0.,
                 rng=None, pad_image=None, calculate_stepk=True, calculate_maxk=True,
                 use_cache=True, use_true_center=True, depixelize=False, offset=None,
                 gsparams=None, _force_stepk=0., _force_maxk=0., hdu=None):
        images = list(image) if isinstance(image, (list, tuple)) else [image]
        if not images:
            raise GalSimValueError("Supplied image list is empty.", image)
        for im in images:
            if isinstance(im, str):
                raise GalSimNotImplementedError("InterpolatedImage from a FITS file is not built")
            if not isinstance(im, Image):
                raise TypeError("Supplied image must be an Image or file name")
            if not im.bounds.isDefined():
                raise GalSimUndefinedBoundsError("Supplied image does not have bounds defined.")
        if not normalization.lower() in ("flux", "f", "surface brightness", "sb"):
            raise GalSimValueError("Invalid normalization requested.", normalization,
                                   ('flux', 'f', 'surface brightness', 'sb'))
        self._gsparams = GSParams.check(gsparams)
        self._x_interpolant = (Quintic(gsparams=self._gsparams) if x_interpolant is None else
                               convert_interpolant(x_interpolant).withGSParams(self._gsparams))
        self._k_interpolant = (Quintic(gsparams=self._gsparams) if k_interpolant is None else
                               convert_interpolant(k_interpolant).withGSParams(self._gsparams))
        if depixelize:
            raise GalSimNotImplementedError("InterpolatedImage(depixelize=True) is not built")
        self._noise_pad = self._check_noise_pad(noise_pad_size, noise_pad)
        self._noise_pad_size = noise_pad_size
        self._rng = rng
        if pad_factor <= 0.:
            raise GalSimRangeError("Invalid pad_factor <= 0 in InterpolatedImage", pad_factor, 0.)
        if scale is not None and wcs is not None:
            raise GalSimIncompatibleValuesError(
                "Cannot provide both scale and wcs to InterpolatedImage", scale=scale, wcs=wcs)
        if wcs is not None and not isinstance(wcs, BaseWCS):
            raise TypeError("wcs parameter is not a galsim.BaseWCS instance")
        if pad_image is not None and not isinstance(pad_image, Image):
            if isinstance(pad_image, str):
                raise GalSimNotImplementedError("pad_image from a FITS file is not built")
            raise TypeError("Supplied pad_image must be an Image.", pad_image)
        self._pad_factor = pad_factor
        self._calculate_stepk = calculate_stepk
        self._calculate_maxk = calculate_maxk
        self._normalization = normalization
        self._flux_arg = flux
        self._use_true_center = use_true_center
        self._force_stepk = float(_force_stepk)
        self._force_maxk = float(_force_maxk)
        self._build_args = (images, scale, wcs, flux, normalization, pad_factor, pad_image, offset,
                            use_true_center, noise_pad_size, noise_pad, rng)
        self._build(*self._build_args)

    # -- construction (interpolatedimage.py:303-400, 590-660) ---------------------------------
    @staticmethod
    def _check_noise_pad(noise_pad_size, noise_pad):
        """The argument checks of _buildRealImage / _buildNoisePadImage for noise padding
        (interpolatedimage.py:463-476, 527-550); returns the variance of the Gaussian padding
        noise (0 for none).  Padding with correlated noise (a CorrelatedNoise, an image or a file
        name) is not built."""
        if noise_pad_size:
            if noise_pad_size < 0:
                raise GalSimValueError("noise_pad_size may not be negative", noise_pad_size)
            if not noise_pad:
                raise GalSimIncompatibleValuesError(
                    "Must provide noise_pad if noise_pad_size > 0",
                    noise_pad=noise_pad, noise_pad_size=noise_pad_size)
        elif noise_pad:
            raise GalSimIncompatibleValuesError(
                "Must provide noise_pad_size if noise_pad != 0",
                noise_pad=noise_pad, noise_pad_size=noise_pad_size)
        if not noise_pad:
            return 0.
        try:
            var = float(noise_pad)
        except (TypeError, ValueError):
            if isinstance(noise_pad, (Image, str)) or hasattr(noise_pad, 'getVariance'):
                raise GalSimNotImplementedError("noise padding with correlated noise (a "
                                                "CorrelatedNoise, an image or a file) is not built")
            raise GalSimValueError(
                "Input noise_pad must be a float/int, a CorrelatedNoise, Image, or filename "
                "containing an image to use to make a CorrelatedNoise.", noise_pad)
        if var < 0.:
            raise GalSimRangeError("Noise variance may not be negative.", var, 0.)
        return var

    def _noise_pad_region(self, noise_pad_size, var, rng, w):
        """The Gaussian noise padding of _buildNoisePadImage (interpolatedimage.py:521-566):
        a noise_pad_size square (in pixels: ceil(size / scale), rounded up to a good FFT
        size) centred on (0, 0), filled with GaussianNoise(BaseDeviate(rng), sqrt(var)) drawn on
        the GPU with the reference's stream.  Returns (bounds, array)."""
        from .noise import BaseDeviate, GaussianNoise
        from .image import ImageD
        n = Image.good_fft_size(int(math.ceil(noise_pad_size / w.scale)))
        half = n // 2
        nim = ImageD(n, n, init_value=0.)
        nim.addNoise(GaussianNoise(BaseDeviate(rng), sigma=math.sqrt(var)))
        return _BoundsI(-half, -half + n - 1, -half, -half + n - 1), nim.array, n

    def _build(self, images, scale, wcs, flux, normalization, pad_factor, pad_image, offset,
               use_true_center, noise_pad_size=0, noise_pad=0., rng=None):
        x_code = self._x_interpolant._code if self._x_interpolant._code is not None else 0
        flags = 0
        if self._force_stepk <= 0. and self._calculate_stepk:
            flags |= _lib.IMAGE_STEPK
        if self._force_maxk <= 0. and self._calculate_maxk:
            flags |= _lib.IMAGE_MAXK
        maxk_limit = 0. if self._calculate_maxk is True else float(self._calculate_maxk or 0.)
        sources, scales, offsets, fluxes, image_fluxes, shapes, images_c = [], [], [], [], [], [], []
        for im in images:
            img = im.view(dtype=np.float64)
            img._array = np.ascontiguousarray(img._array)
            img.setCenter(0, 0)
            if scale is not None:
                w = PixelScale(scale)
            elif wcs is not None:
                w = wcs
            elif im.wcs is None:
                raise GalSimIncompatibleValuesError(
                    "No information given with Image or keywords about pixel scale!",
                    scale=scale, wcs=wcs, image=im)
            else:
                w = im.wcs
            if not w._isPixelScale:
                raise GalSimNotImplementedError("InterpolatedImage needs a PixelScale WCS here")
            img.wcs = w
            off = self._parse_offset(offset)
            off = self._adjust_offset(img.bounds, off, None, use_true_center)
            b = img.bounds
            # padded frame (_buildRealImage)
            pad_size = max(img.array.shape)
            if pad_factor > 1.:
                pad_size = int(math.ceil(pad_factor * pad_size))
            nz = b
            npad = None
            if noise_pad:
                # drawn once per image: a rebuild (withGSParams) keeps the same padding, as the
                # reference's copy keeps its padded image
                cache = self.__dict__.setdefault('_noise_regions', {})
                if len(sources) not in cache:
                    cache[len(sources)] = self._noise_pad_region(noise_pad_size, self._noise_pad, rng, w)
                nb, narr, nsize = cache[len(sources)]
                pad_size = max(pad_size, nsize)
                npad = (nb, narr)
                nz = _BoundsI(min(nz.xmin, nb.xmin), max(nz.xmax, nb.xmax),
                              min(nz.ymin, nb.ymin), max(nz.ymax, nb.ymax))
            pim = None
            if pad_image is not None:
                pim = pad_image.view(dtype=np.float64)
                pim.setCenter(0, 0)
                pad_size = max(pad_size, *pim.array.shape)
                pb = pim.bounds
                nz = _BoundsI(min(nz.xmin, pb.xmin), max(nz.xmax, pb.xmax),
                              min(nz.ymin, pb.ymin), max(nz.ymax, pb.ymax))
            N = Image.good_fft_size(pad_size)
            region = np.zeros((nz.ymax - nz.ymin + 1, nz.xmax - nz.xmin + 1))
            if npad is not None:
                nb, narr = npad
                region[nb.ymin - nz.ymin:nb.ymax - nz.ymin + 1,
                       nb.xmin - nz.xmin:nb.xmax - nz.xmin + 1] = narr
            if pim is not None:
                pb = pim.bounds
                region[pb.ymin - nz.ymin:pb.ymax - nz.ymin + 1,
                       pb.xmin - nz.xmin:pb.xmax - nz.xmin + 1] = pim.array
            region[b.ymin - nz.ymin:b.ymax - nz.ymin + 1, b.xmin - nz.xmin:b.xmax - nz.xmin + 1] = img.array
            if nz.xmin < -(N // 2) or nz.ymin < -(N // 2) or nz.xmax >= N // 2 or nz.ymax >= N // 2:
                raise GalSimValueError("pad_image does not fit in the padded frame", pad_image)
            image_flux = float(np.sum(img.array, dtype=np.float64))
            if ((self._calculate_stepk or self._calculate_maxk or flux is not None) and
                    image_flux == 0.):
                raise GalSimValueError("This input image has zero total flux. It does not define a "
                                       "valid surface brightness profile.", im)
            if flux is None:
                f = image_flux
                if normalization.lower() in ('surface brightness', 'sb'):
                    f *= w.pixelArea()
            else:
                f = flux
            # CalculateSizeContainingFlux is given the whole image (interpolatedimage.py:647-658)
            thresh = (1. - self._gsparams.folding_threshold) * image_flux
            sources.append(_ImageSource(region, N, nz.xmin, nz.ymin, (b.xmin, b.xmax, b.ymin, b.ymax),
                                        x_code, flags, float(np.sum(region, dtype=np.float64)),
                                        thresh, maxk_limit, self._x_interpolant))
            scales.append(w.scale)
            offsets.append((off.x, off.y))
            fluxes.append(f)
            image_fluxes.append(image_flux)
            shapes.append(img.array.shape)
            images_c.append(img)
        self._sources = sources
        self._images = images_c
        B = len(sources)
        self._batch = B
        self._scale = np.array(scales) if B > 1 else scales[0]
        self._image_flux = np.array(image_fluxes) if B > 1 else image_fluxes[0]
        if flux is not None and np.ndim(flux) and B > 1:
            self._flux = np.asarray(flux, dtype=np.float64).reshape(B)
        else:
            self._flux = np.array(fluxes) if B > 1 else fluxes[0]
        self._shapes = shapes
        self._offset_xy = np.array(offsets)
        # the world profile: SBInterpolatedImage shifted by -offset, then _profileToWorld
        from .compound import _Transform
        leaf = _ImageLeaf(sources, self._x_interpolant, self._k_interpolant, self._gsparams)
        ox, oy = self._offset_xy[:, 0], self._offset_xy[:, 1]
        if B == 1:
            ox, oy = float(ox[0]), float(oy[0])
        prof = leaf
        if np.any(np.asarray(ox) != 0.) or np.any(np.asarray(oy) != 0.):
            prof = _Transform(prof, offset=(-ox, -oy))
        flux_ratio = np.where(np.asarray(self._flux) != np.asarray(self._image_flux),
                              np.asarray(self._flux) / np.asarray(self._image_flux), 1.)
        s = np.asarray(self._scale, dtype=np.float64)
        invscale = 1. / s
        if B == 1:
            flux_ratio = float(flux_ratio)
            jac = None if float(s) == 1. else np.array([[float(s), 0.], [0., float(s)]])
            invscale = float(invscale)
        else:
            jac = None if np.all(s == 1.) else np.stack(
                [np.stack([s, np.zeros(B)], -1), np.stack([np.zeros(B), s], -1)], -2)
        self._inner = _Transform(prof, jac, flux_ratio=invscale ** 2 * flux_ratio)

    # -- properties -----------------------------------------------------------------------------
    x_interpolant = property(lambda self: self._x_interpolant)
    k_interpolant = property(lambda self: self._k_interpolant)

    @property
    def image(self):
        """The underlying image (centred on (0, 0)); a list for a batch."""
        return self._images[0] if self._batch == 1 else self._images

    @property
    def flux(self):
        return self._flux

    def withGSParams(self, gsparams=None, **kwargs):
        """interpolatedimage.py:400-414: the interpolants take the new GSParams and the sizes
        are found again."""
        if gsparams == self.gsparams and not kwargs:
            return self
        import copy
        ret = copy.copy(self)
        ret._gsparams = GSParams.check(gsparams, self.gsparams, **kwargs)
        ret._x_interpolant = self._x_interpolant.withGSParams(ret._gsparams, **kwargs)
        ret._k_interpolant = self._k_interpolant.withGSParams(ret._gsparams, **kwargs)
        ret.__dict__.pop('_cached_sizes', None)
        ret._build(*self._build_args)
        return ret

    # -- drawing ----------------------------------------------------------------------------------
    def _flatten(self, bld, jac):
        self._inner._flatten(bld, jac)

    def _size(self, prog, it):
        """stepk / maxk in world units (interpolatedimage.py:647-685): from the GPU's flux
        radius R and scanned maxk (image units) of this object's one leaf."""
        R, maxk_img = prog.leaf_size(next(it))
        B = len(R)
        s = np.broadcast_to(np.asarray(self._scale, dtype=np.float64), (B,))
        if self._force_stepk > 0.:
            stepk = np.full(B, self._force_stepk)
        else:
            if not self._calculate_stepk:
                shp = np.broadcast_to(np.array([max(sh) for sh in self._shapes], float),
                                      (B,))
                R = shp / 2. - 0.5
            R2 = self._x_interpolant.xrange
            stepk = np.array([math.pi / (math.hypot(r, R2) * sc) for r, sc in zip(R, s)])
        if self._force_maxk > 0.:
            maxk = np.full(B, self._force_maxk)
        elif self._calculate_maxk:
            maxk = maxk_img / s
        else:
            maxk = self._x_interpolant.krange / s
        return stepk, maxk

    def __eq__(self, other):
        return self is other or (
            isinstance(other, InterpolatedImage) and self._batch == other._batch and
            all(np.array_equal(a.region, b.region) and a.N == b.N and a.x0 == b.x0 and
                a.y0 == b.y0 for a, b in zip(self._sources, other._sources)) and
            self.x_interpolant == other.x_interpolant and
            self.k_interpolant == other.k_interpolant and
            np.array_equal(self.flux, other.flux) and
            np.array_equal(self._offset_xy, other._offset_xy) and
            np.array_equal(self._scale, other._scale) and
            self.gsparams == other.gsparams and
            self._force_stepk == other._force_stepk and self._force_maxk == other._force_maxk)

    def __hash__(self):
        return hash(("galsim.InterpolatedImage", self.x_interpolant, self.k_interpolant,
                     self._batch, tuple(s.N for s in self._sources),
                     tuple(float(s.region.sum()) for s in self._sources)))

    def __repr__(self):
        return 'galsim.InterpolatedImage(%r, %r, %r, flux=%r, gsparams=%r)' % (
            self.image, self.x_interpolant, self.k_interpolant, self.flux, self.gsparams)

    def __str__(self):
        return 'galsim.InterpolatedImage(image=%s, flux=%s)' % (self.image, self.flux)


__all__ = ['InterpolatedImage']

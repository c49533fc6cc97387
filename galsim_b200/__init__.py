"""galsim_b200: GalSim's FFT drawing path on NVIDIA B200 (sm_100a).

A drop-in for ``GSObject.drawImage(method='fft')`` and ``drawKImage`` on
Convolve / Sum / Transform trees of Gaussian, Exponential, Sersic, Moffat (both also
truncated), Kolmogorov, Airy, Box / Pixel and InterpolatedImage, real-space drawing of analytic
profiles ('no_pixel' / 'sb'), chromatic objects drawn through bandpasses (SED, Bandpass,
ChromaticAtmosphere, chromatic sums and convolutions), the reference's Gaussian / Poisson / CCD
noise applied on the device, and FITS files of Images and stamp batches (galsim_b200.fits; a
batch's file image is assembled on the device).  The host code here mirrors the reference's
Python API; every numerical step of drawing (FP64 sizing and FT tables, k-space evaluation,
Hermitian wrap, inverse FFT, crop and flux sum, real-space evaluation, wavelength integrals of
images) runs in the hand-written CUDA kernels of libgsb.so, called through the C ABI declared in
include/gsb.h.  There is no CPU fallback.
"""
from .errors import *
from .gsparams import GSParams
from .position import Position, PositionD, PositionI, _PositionD, _PositionI
from .bounds import Bounds, BoundsD, BoundsI, _BoundsI
from .angle import Angle, AngleUnit, _Angle, radians, degrees, hours, arcmin, arcsec
from .shear import Shear, _Shear
from .wcs import BaseWCS, PixelScale
from .image import Image, _Image, ImageF, ImageD, ImageI, ImageS, ImageCF, ImageCD
from .gsobject import GSObject
from .profiles import Gaussian, Exponential, Sersic, DeVaucouleurs, Moffat, Kolmogorov, Airy
from .box import Box, Pixel
from .interpolant import (Interpolant, Delta, Nearest, SincInterpolant, Linear, Cubic, Quintic,
                          Lanczos, convert_interpolant)
from .interpolatedimage import InterpolatedImage
from .noise import BaseDeviate, BaseNoise, GaussianNoise, PoissonNoise, CCDNoise, VariableGaussianNoise, DeviateNoise
from .random import UniformDeviate, GaussianDeviate, PoissonDeviate, WeibullDeviate, GammaDeviate, Chi2Deviate, BinomialDeviate, DistDeviate
from . import fits
from .fits import FitsHeader
from .compound import Convolve, Convolution, Add, Sum, Transform, Transformation, _Transform
from .batch import draw_batch, draw_batches, plan_batch, run_batch, StampBatch
from .table import LookupTable, _LookupTable, trapz
from .sed import SED
from .bandpass import Bandpass
from . import integ, dcr
from .chromatic import (ChromaticObject, ChromaticTransformation, SimpleChromaticTransformation,
                        ChromaticAtmosphere, ChromaticAiry, ChromaticSum, ChromaticConvolution)
from ._lib import set_device
from . import autodiff
from . import config
from .config import draw_config

__version__ = '0.1.0'

"""ORACLE / CPU BASELINE: the reference's own C++ drawing arithmetic, driven from Python.

TEST INFRASTRUCTURE ONLY (tests/ and bench.py's reference arm).  libgsref.so is built by
`make -C oracle ref` from the reference's src/*.cpp (with the FP64 FFTW-API shim
oracle/ref_build/fftw3_fp64_shim.c, since libfftw3 is not installed).  The orchestration
below is drawFFT (galsim/gsobject.py:1927-2045) restated over the oracle's tree classes:
every leaf is drawn by the reference's SBProfile::drawK, shifted transforms by its
ApplyKImagePhases, then its wrapImage and irfft; stepK / maxK of the leaves come from the
reference's C++ and are composed with the reference's Python rules.
"""
import ctypes
import math
import os

import numpy as np

import galsim_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, '_ref', 'libgsref.so')
GAUSS, EXPO, SERSIC, MOFFAT, KOLMO, AIRY, BOX = range(7)
_lib = None


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        L.gsref_profile_info.argtypes = [ctypes.c_int, dp, ctypes.c_double, dp, dp]
        L.gsref_draw_k.argtypes = [ctypes.c_int, dp, ctypes.c_double, dp, dp, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_double, dp]
        L.gsref_apply_phases.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.gsref_wrap.argtypes = [dp] + [ctypes.c_int] * 10
        L.gsref_irfft.argtypes = [dp, ctypes.c_int, ctypes.c_int, dp]
        L.gsref_good_fft_size.argtypes = [ctypes.c_int]
        L.gsref_last_error.restype = ctypes.c_char_p
        ip = ctypes.POINTER(ctypes.c_int)
        L.gsref_ii_create.restype = ctypes.c_void_p
        L.gsref_ii_create.argtypes = [dp, ctypes.c_int, ip, ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, dp]
        L.gsref_ii_destroy.argtypes = [ctypes.c_void_p]
        L.gsref_ii_maxk.argtypes = [ctypes.c_void_p, ctypes.c_double, dp]
        L.gsref_ii_draw_k.argtypes = [ctypes.c_void_p, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_double, dp]
        L.gsref_size_containing_flux.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_double, dp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


GSP = np.array([128, 8192, 5e-3, 5, 1e-3, 1e-5, 1e-5, 1, 1e-4, 1e-6, 1e-6, 1e-8, 1e-5], dtype=np.float64)


def _leaf_args(o):
    if isinstance(o, O.OGaussian):
        return GAUSS, [o.sigma]
    if isinstance(o, O.OExponential):
        return EXPO, [o.r0]
    if isinstance(o, O.OSersic):
        return SERSIC, [o.n, o.r0, 0.]
    if isinstance(o, O.OMoffat):
        return MOFFAT, [o.beta, o.r0, 0.]
    if isinstance(o, O.OKolmogorov):
        return KOLMO, [o.lor0]
    if isinstance(o, O.OAiry):
        return AIRY, [o.lod, o.obs]
    if isinstance(o, O.OBox):
        return BOX, [o.w, o.h]
    raise TypeError(o)


INTERP_CODES = {'delta': 0, 'nearest': 1, 'linear': 2, 'cubic': 3, 'quintic': 4}


class RIILeaf(object):
    """The reference's SBInterpolatedImage (image units) over a padded image."""

    def __init__(self, xim, ib, nb, xcode, kcode, stepk_img):
        N = xim.shape[0]
        self.xim = np.ascontiguousarray(xim, dtype=np.float64)
        ibv = (ctypes.c_int * 4)(*ib)
        nbv = (ctypes.c_int * 4)(*nb)
        self.h = lib().gsref_ii_create(_p(self.xim), N, ibv, nbv, xcode, kcode, stepk_img, 0., _p(GSP))
        if not self.h:
            raise RuntimeError(lib().gsref_last_error().decode())

    def maxk(self, max_maxk=0.):
        out = np.zeros(1)
        if lib().gsref_ii_maxk(self.h, max_maxk, _p(out)):
            raise RuntimeError(lib().gsref_last_error().decode())
        return float(out[0])

    def __del__(self):
        if getattr(self, 'h', None):
            lib().gsref_ii_destroy(self.h)


class RInterpolatedImage(O.OObj):
    """InterpolatedImage(image, scale=...) on the reference's C++ (interpolatedimage.py:303-685):
    CalculateSizeContainingFlux and calculateMaxK for the sizes, SBInterpolatedImage::drawK for
    the k-values; the frame and the world transform follow the reference's Python."""

    def __init__(self, array, scale, x_interp='quintic', k_interp='quintic', pad_factor=4.):
        arr = np.ascontiguousarray(array, dtype=np.float64)
        ny, nx = arr.shape
        x0, y0 = -(nx // 2), -(ny // 2)
        dx = -0.5 if nx % 2 == 0 else 0.
        dy = -0.5 if ny % 2 == 0 else 0.
        pad = max(nx, ny)
        if pad_factor > 1.:
            pad = int(math.ceil(pad_factor * pad))
        N = lib().gsref_good_fft_size(pad)
        xim = np.zeros((N, N))
        xim[y0 + N // 2:y0 + N // 2 + ny, x0 + N // 2:x0 + N // 2 + nx] = arr
        b = (x0, x0 + nx - 1, y0, y0 + ny - 1)
        image_flux = float(np.sum(arr, dtype=np.float64))
        out = np.zeros(1)
        if lib().gsref_size_containing_flux(_p(arr), b[0], b[1], b[2], b[3], (1. - GSP[2]) * image_flux, _p(out)):
            raise RuntimeError(lib().gsref_last_error().decode())
        R = math.hypot(float(out[0]), O.INTERP_XRANGE[x_interp])
        self.stepk = math.pi / (R * scale)
        self.leaf = RIILeaf(xim, b, b, INTERP_CODES[x_interp], INTERP_CODES[k_interp], self.stepk * scale)
        self.maxk = self.leaf.maxk() / scale
        prof = self.leaf
        if dx != 0. or dy != 0.:
            prof = O.OTransform(prof, offset=(-dx, -dy))
        jac = None if scale == 1. else [[scale, 0.], [0., scale]]
        self.inner = O.OTransform(prof, jac=jac, flux_ratio=(1. / scale) ** 2)


def stepk_maxk(o):
    """Leaf sizes from the reference C++; composition by the reference Python rules."""
    if isinstance(o, RInterpolatedImage):
        return o.stepk, o.maxk
    if isinstance(o, O.OConvolve):
        s = [stepk_maxk(x) for x in o.objs]
        inv = 0
        for sk, _ in s:
            inv = inv + sk ** (-2)
        return inv ** (-0.5), min(mk for _, mk in s)
    if isinstance(o, O.OSum):
        s = [stepk_maxk(x) for x in o.objs]
        return min(sk for sk, _ in s), max(mk for _, mk in s)
    if isinstance(o, O.OTransform):
        sk, mk = stepk_maxk(o.original)
        if o.jac is None:
            major = minor = 1.
        else:
            j = o.jac
            h1 = math.hypot(j[0, 0] + j[1, 1], j[0, 1] - j[1, 0])
            h2 = math.hypot(j[0, 0] - j[1, 1], j[0, 1] + j[1, 0])
            major, minor = 0.5 * abs(h1 + h2), 0.5 * abs(h1 - h2)
        sk = sk / major
        if o.dx != 0. or o.dy != 0.:
            sk = math.pi / (math.pi / sk + math.hypot(o.dx, o.dy))
        return sk, mk / minor
    t, p = _leaf_args(o)
    out = np.zeros(2)
    pa = np.array(p, dtype=np.float64)
    rc = lib().gsref_profile_info(t, _p(pa), o.flux, _p(GSP), _p(out))
    if rc:
        raise RuntimeError(lib().gsref_last_error().decode())
    if t == GAUSS:          # gaussian.py:148-155 overrides the C++ value
        return O.OGaussian.stepk_maxk(o)
    if t == EXPO:
        return out[0], 1e-3 ** (-1. / 3.) / o.r0
    if t == KOLMO:
        return out[0], (-math.log(1e-5)) ** 0.6 * o.k0
    if t == AIRY:
        return out[0], 2. * math.pi / o.lod
    if t == BOX:
        return math.pi / max(o.w, o.h), 2. / (1e-3 * min(o.w, o.h))
    return out[0], out[1]


def draw_k(o, kim, xmin, ymin, dk, jac):
    """_drawKImage tree walk with the reference's C++ for the leaves and phases."""
    n, m = kim.shape
    if isinstance(o, RInterpolatedImage):
        draw_k(o.inner, kim, xmin, ymin, dk, jac)
        return
    if isinstance(o, RIILeaf):
        j = None if jac is None else np.ascontiguousarray(jac, dtype=np.float64)
        if lib().gsref_ii_draw_k(o.h, _p(kim.view(np.float64)), xmin, xmin + m - 1, ymin, ymin + n - 1,
                                 dk, _p(j)):
            raise RuntimeError(lib().gsref_last_error().decode())
        return
    if isinstance(o, (O.OConvolve, O.OSum)):
        draw_k(o.objs[0], kim, xmin, ymin, dk, jac)
        tmp = np.empty_like(kim)
        for x in o.objs[1:]:
            draw_k(x, tmp, xmin, ymin, dk, jac)
            if isinstance(o, O.OConvolve):
                kim *= tmp
            else:
                kim += tmp
        return
    if isinstance(o, O.OTransform):
        jac1 = o.jac if jac is None else jac if o.jac is None else jac.dot(o.jac)
        draw_k(o.original, kim, xmin, ymin, dk, jac1)
        fs = abs(o.det()) * o.flux_ratio
        if o.dx != 0. or o.dy != 0.:
            j = None if jac is None else np.ascontiguousarray(jac, dtype=np.float64)
            lib().gsref_apply_phases(_p(kim.view(np.float64)), xmin, xmin + m - 1, ymin, ymin + n - 1,
                                     dk, _p(j), o.dx, o.dy, fs)
        elif abs(fs - 1.) > 1e-5:
            kim *= fs
        return
    t, p = _leaf_args(o)
    pa = np.array(p, dtype=np.float64)
    j = None if jac is None else np.ascontiguousarray(jac, dtype=np.float64)
    rc = lib().gsref_draw_k(t, _p(pa), o.flux, _p(GSP), _p(kim.view(np.float64)), xmin, xmin + m - 1,
                            ymin, ymin + n - 1, dk, _p(j))
    if rc:
        raise RuntimeError(lib().gsref_last_error().decode())


class RSersic(O.OSersic):
    """A Sersic leaf whose scale radius comes from the reference's SersicHLR (C++), without
    building the oracle's own FT table."""

    def __init__(self, n, hlr, flux=1.):
        lib().gsref_sersic_hlr.restype = ctypes.c_double
        lib().gsref_sersic_hlr.argtypes = [ctypes.c_double, ctypes.c_double]
        self.n, self.flux = float(n), float(flux)
        self.r0 = float(hlr) / lib().gsref_sersic_hlr(self.n, 1.0)


def c2_profile(n, hlr, flux, g1, g2, fwhm, scale):
    """Sersic.shear x Kolmogorov x Pixel, the batched-forward workload's stamp."""
    return O.OConvolve(RSersic(n, hlr, flux).shear(g1, g2), O.OKolmogorov(fwhm=fwhm), O.OBox(scale))


def draw_image(prof, nx, ny, scale, offset=(0., 0.), pixel=True):
    """drawImage(nx, ny, scale, method='fft' | 'no_pixel' (pixel=False)) through the reference
    C++ (FP64); nx = ny = None sizes the image automatically (getGoodImageSize,
    gsobject.py:1900-1925)."""
    auto = nx is None
    dx = float(offset[0]) - (0.5 if auto or nx % 2 == 0 else 0.)
    dy = float(offset[1]) - (0.5 if auto or ny % 2 == 0 else 0.)
    inv = 1. / scale
    img = O.OTransform(prof, jac=[[inv, 0.], [0., inv]], offset=(dx, dy), flux_ratio=scale ** 2)
    if pixel:
        img = O.OConvolve(img, O.OBox(1.0))
    if auto:
        sk, _ = stepk_maxk(img)
        nn = int(math.ceil(2. * math.pi / sk * (1. - 1.e-12)))
        nx = ny = 2 * ((nn + 1) // 2)
    cx, cy = 1 + nx // 2, 1 + ny // 2
    xmin, xmax, ymin, ymax = 1 - cx, nx - cx, 1 - cy, ny - cy
    stepk, maxk = stepk_maxk(img)
    Nd = 2. * math.pi / stepk
    N = int(math.ceil(Nd * (1. - 1.e-12)))
    N = 2 * ((N + 1) // 2)
    N = max(N, max(abs(xmin), abs(xmax), abs(ymin), abs(ymax)) * 2, max(nx, ny))
    N = lib().gsref_good_fft_size(N)
    N = max(N, 128)
    dk = 2. * math.pi / N
    Nk = N if N * dk / 2 > maxk else int(np.ceil(maxk / dk)) * 2
    kim = np.zeros((Nk + 1, Nk // 2 + 1), dtype=np.complex128)
    draw_k(img, kim, 0, -Nk // 2, dk, None)
    lib().gsref_wrap(_p(kim.view(np.float64)), 0, Nk // 2, -Nk // 2, Nk // 2, 0, N // 2, -N // 2, N // 2 - 1, 1, 0)
    row0 = (Nk - N) // 2
    sub = kim[row0:]
    real = np.zeros((N, N + 2), dtype=np.float64)
    lib().gsref_irfft(_p(sub.view(np.float64)), Nk // 2 + 1, N, _p(real))
    stamp = real[ymin + N // 2:ymax + N // 2 + 1, xmin + N // 2:xmax + N // 2 + 1]
    return stamp.copy(), float(stamp.sum()), N, Nk

"""The oracle's FFTW3 stand-in (oracle/ref_build/fftw3_fp64_shim.c, linked into
oracle/_ref/libgsref.so with the reference C++) against numpy.fft (pocketfft, FP64): the
c2c, r2c and c2r plans the reference's image code makes (src/Image.cpp:796, 907, 983), with
FFTW's sign and layout conventions, at the lengths GalSim's goodFFTSize picks (2^a, 3 * 2^a)
and at lengths with other prime factors.  CPU only; skipped when libgsref.so is not built."""
import ctypes
import os

import numpy as np
import pytest

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle', '_ref', 'libgsref.so')
pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason='oracle/_ref/libgsref.so not built')

FFTW_FORWARD, FFTW_BACKWARD, FFTW_ESTIMATE = -1, 1, 1 << 6


@pytest.fixture(scope='module')
def fftw():
    L = ctypes.CDLL(LIB)
    vp = ctypes.c_void_p
    L.fftw_plan_dft_2d.restype = vp
    L.fftw_plan_dft_2d.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_uint]
    L.fftw_plan_dft_r2c_2d.restype = vp
    L.fftw_plan_dft_r2c_2d.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_uint]
    L.fftw_plan_dft_c2r_2d.restype = vp
    L.fftw_plan_dft_c2r_2d.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_uint]
    L.fftw_execute.argtypes = [vp]
    L.fftw_destroy_plan.argtypes = [vp]
    return L


def _run(L, plan):
    L.fftw_execute(plan)
    L.fftw_destroy_plan(plan)


SHAPES = [(8, 8), (12, 16), (128, 128), (192, 96), (6, 10), (15, 21), (7, 5), (256, 384)]


@pytest.mark.parametrize('shape', SHAPES)
@pytest.mark.parametrize('sign', [FFTW_FORWARD, FFTW_BACKWARD])
def test_c2c(fftw, shape, sign):
    rng = np.random.default_rng(1)
    a = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    out = np.zeros_like(a)
    _run(fftw, fftw.fftw_plan_dft_2d(shape[0], shape[1], a.ctypes.data, out.ctypes.data, sign, FFTW_ESTIMATE))
    ref = np.fft.fft2(a) if sign < 0 else np.fft.ifft2(a) * a.size
    assert np.abs(out - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize('shape', SHAPES)
def test_r2c_c2r(fftw, shape):
    n0, n1 = shape
    h1 = n1 // 2 + 1
    rng = np.random.default_rng(2)
    x = rng.normal(size=shape)
    k = np.zeros((n0, h1), complex)
    _run(fftw, fftw.fftw_plan_dft_r2c_2d(n0, n1, x.ctypes.data, k.ctypes.data, FFTW_ESTIMATE))
    ref = np.fft.rfft2(x)
    assert np.abs(k - ref).max() <= 1e-13 * np.abs(ref).max()
    # c2r, out of place: unnormalised inverse of a Hermitian half plane
    kin = ref.copy()
    y = np.zeros(shape)
    _run(fftw, fftw.fftw_plan_dft_c2r_2d(n0, n1, kin.ctypes.data, y.ctypes.data, FFTW_ESTIMATE))
    assert np.abs(y / x.size - x).max() <= 1e-13 * np.abs(x).max()
    # c2r in place: real rows padded to 2 * (n1 / 2 + 1) doubles (the reference's irfft)
    buf = np.zeros((n0, h1), complex)
    buf[:] = ref
    _run(fftw, fftw.fftw_plan_dft_c2r_2d(n0, n1, buf.ctypes.data, buf.ctypes.data, FFTW_ESTIMATE))
    y2 = buf.view(np.float64).reshape(n0, 2 * h1)[:, :n1]
    assert np.abs(y2 / x.size - x).max() <= 1e-13 * np.abs(x).max()

"""The reference's own drawFFT sequence (galsim/gsobject.py:2014-2045 and drawFFT_finish,
:1975-2012), step by step, with each compiled step it calls in _galsim replaced by this
library's standalone entry point through galsim_b200.refbinding -- the drop-in at the
reference's boundary for a caller that keeps the reference's orchestration:

    kimage, N = drawFFT_makeKImage(image)         sizing (here: the library's, equal to the reference's)
    prof._drawKImage(kimage)                      -> refbinding.drawK          (gsb_draw_k)
    kimage._wrap(bwrap, hermx=True)               -> refbinding.wrapImage      (gsb_wrap_image)
    _galsim.irfft(kwrap, real, True, True)        -> refbinding.irfft          (gsb_irfft)
    real.subImage(image.bounds), sum              numpy

on every drawImage fixture the reference drew (tests/golden/reference_draws.npz), for the
profile in image coordinates that drawImage hands to drawFFT (gsobject.py:1736-1764).
Tolerances: float64 images 1e-9 x peak and 1e-10 in flux; float32 images (complex64
k-images, FP32 k-values) 1e-5 x peak and 1e-6 in flux.
"""
import os

import numpy as np
import pytest

import galsim_b200 as galsim
from galsim_b200 import box, refbinding
from galsim_b200.compound import Convolve, _Transform
import make_golden as MG

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'reference_draws.npz'))


def _image_profile(prof, nx, ny, scale, off):
    """drawImage's world-to-image profile: offset (true centre of even sizes at -0.5),
    Jacobian diag(1/scale), flux x scale^2, convolved with Pixel(1)."""
    dx, dy = float(off[0]), float(off[1])
    if nx % 2 == 0:
        dx -= 0.5
    if ny % 2 == 0:
        dy -= 0.5
    inv = 1. / scale
    t = _Transform(prof, np.array([[inv, 0.], [0., inv]]), flux_ratio=scale ** 2,
                   offset=(np.array([dx]), np.array([dy])))
    return Convolve(t, box.Pixel(scale=1.0))


@pytest.mark.parametrize('case', MG.DRAW_CASES, ids=[c[0] for c in MG.DRAW_CASES])
def test_reference_drawfft_sequence_through_standalone_steps(case):
    name, spec, nx, ny, scale, dt, off = case
    prof = MG.profile(galsim, spec)
    # drawFFT_makeKImage's sizes for this image (the batched path's sizing, which equals the
    # reference's on these fixtures: test_gpu_parity.py)
    st = galsim.draw_batch(prof, nx=nx, ny=ny, scale=scale, dtype=np.float64, offset=off)
    N, Nk = int(st.N[0]), int(st.Nk[0])
    ctype = np.complex128 if dt == 'f8' else np.complex64
    kb = (0, Nk // 2, -Nk // 2, Nk // 2)
    kimage = np.zeros((Nk + 1, Nk // 2 + 1), dtype=ctype)
    refbinding.drawK(_image_profile(prof, nx, ny, scale, off), kimage, kb, 2. * np.pi / N)
    bwrap = (0, N // 2, -N // 2, N // 2 - 1)
    refbinding.wrapImage(kimage, kb, bwrap, True, False)
    kwrap = kimage[bwrap[2] - kb[2]:bwrap[3] - kb[2] + 1, 0:N // 2 + 1]
    breal = (-N // 2, N // 2 + 1, -N // 2, N // 2 - 1)
    real = np.zeros((N, N + 2))
    refbinding.irfft(kwrap, bwrap, real, breal, True, True)
    # the image's bounds relative to its centre (image.setCenter(0, 0), gsobject.py:1776)
    cx, cy = 1 + nx // 2, 1 + ny // 2
    x0, y0 = 1 - cx, 1 - cy
    sub = real[y0 + N // 2:y0 + N // 2 + ny, x0 + N // 2:x0 + N // 2 + nx].astype(np.dtype(dt))
    added = float(sub.sum(dtype=float))
    ref = GOLD['draw_' + name]
    fref = float(GOLD['draw_' + name + '_flux'])
    ptol, ftol = (1e-9, 1e-10) if dt == 'f8' else (1e-5, 1e-6)
    assert np.abs(sub.astype(float) - ref).max() <= ptol * np.abs(ref).max(), name
    assert abs(added - fref) <= ftol * abs(fref), (name, added, fref)


def test_refbinding_irfft_bound_errors():
    """The reference's irfft bound checks (src/Image.cpp:818-840) with its messages."""
    k = np.zeros((8, 5), np.complex128)
    out = np.zeros((8, 10))
    with pytest.raises(galsim.GalSimError, match='inverse_fft requires bounds'):
        refbinding.irfft(k, (1, 5, -4, 3), out, (-4, 5, -4, 3), True, True)
    with pytest.raises(galsim.GalSimError, match='out.bounds'):
        refbinding.irfft(k, (0, 4, -4, 3), np.zeros((8, 9)), (-4, 4, -4, 3), True, True)

"""GPU tests of the standalone entry points that mirror the reference's compiled hot-path
steps (_galsim.SBProfile.drawK, ApplyKImagePhases, wrapImage, irfft), called through the C ABI
on device images and compared with the reference's own outputs on the same inputs
(tests/golden/reference_standalone.npz and the wrap / irfft cases of reference_draws.npz).

Tolerances: FP64 results to 1e-12 of the image's largest value (the reference computes in
FP64 too; only the order of operations differs) except drawK, whose profile evaluation is
held to the same 1e-9 x peak as the drawKImage parity tests; complex64 outputs to 2e-6.
"""
import ctypes
import os

import numpy as np
import pytest

import galsim_b200 as galsim
from galsim_b200 import _lib
from galsim_b200.program import Program
import make_golden as MG

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
STD = np.load(os.path.join(HERE, 'golden', 'reference_standalone.npz'))
GOLD = np.load(os.path.join(HERE, 'golden', 'reference_draws.npz'))


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(_lib.Device.torch_device())


def _c(t):
    return ctypes.c_void_p(t.data_ptr())


def _dp(arr):
    return arr.ctypes.data_as(ctypes.c_void_p) if arr is not None else None


@pytest.mark.parametrize('case', MG.STANDALONE_DRAWK, ids=[c[0] for c in MG.STANDALONE_DRAWK])
def test_draw_k_vs_reference(case):
    import torch
    name, spec, dk, b, jac, dt = case
    prog = Program(MG.profile(galsim, spec))
    prog.prepare()
    nx, ny = b[1] - b[0] + 1, b[3] - b[2] + 1
    f64 = dt == 'c16'
    out = torch.zeros(nx * ny * 2, dtype=torch.float64 if f64 else torch.float32, device=_lib.Device.torch_device())
    ph = _lib.to_device(np.stack(prog.bld.phases, axis=1)) if prog.bld.phases else None
    sc = _lib.to_device(np.stack(prog.bld.scales, axis=1)) if prog.bld.scales else None
    j = None if jac is None else np.array(jac, dtype=np.float64)
    _lib.check(_lib.lib().gsb_draw_k(ctypes.byref(prog.tpl), 1, ctypes.byref(prog.gsp_c), _lib.ptr(prog.d_leaves),
                                     _c(ph) if ph is not None else None, _c(sc) if sc is not None else None,
                                     prog.tables.handle if prog.tables else None, float(dk), _dp(j),
                                     b[0], b[2], nx, ny, _c(out), _lib.F64 if f64 else _lib.F32,
                                     _lib.Device.stream()))
    a = out.cpu().numpy().reshape(ny, nx, 2)
    got = a[..., 0] + 1j * a[..., 1]
    ref = STD['drawk_' + name]
    tol = 1e-9 if f64 else 2e-6
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (name, np.abs(got - ref).max() / np.abs(ref).max())


@pytest.mark.parametrize('tag', ['jac', 'nojac'])
@pytest.mark.parametrize('f64', [True, False])
def test_apply_kimage_phases_vs_reference(tag, f64):
    a = STD['phase_in_' + tag]
    dt = np.complex128 if f64 else np.complex64
    img = _dev(a.astype(dt).view(np.float64 if f64 else np.float32))
    jac = None if tag == 'nojac' else np.array((0.9, 0.3, -0.2, 1.1))
    _lib.check(_lib.lib().gsb_apply_kimage_phases(_c(img), _lib.F64 if f64 else _lib.F32, 0, -10, a.shape[1],
                                                  a.shape[0], a.shape[1], 0.3, _dp(jac), 0.37, -0.61, 1.7,
                                                  _lib.Device.stream()))
    got = img.cpu().numpy().view(dt)
    ref = STD['phase_out_' + tag]
    tol = 1e-12 if f64 else 2e-6
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()


def _wrap(a, cplx, b_in, b_out, hermx, f64=True):
    import torch
    xmin, xmax, ymin, ymax = b_in
    bx0, bx1, by0, by1 = b_out
    mw, nw = bx1 - bx0 + 1, by1 - by0 + 1
    if cplx:
        dt = np.complex128 if f64 else np.complex64
        d_in = _dev(a.astype(dt).view(np.float64 if f64 else np.float32))
        out = torch.zeros(mw * nw * 2, dtype=torch.float64 if f64 else torch.float32, device=d_in.device)
    else:
        d_in = _dev(a.astype(np.float64 if f64 else np.float32))
        out = torch.zeros(mw * nw, dtype=d_in.dtype, device=d_in.device)
    _lib.check(_lib.lib().gsb_wrap_image(_c(d_in), _lib.F64 if f64 else _lib.F32, int(cplx), xmin, xmax, ymin,
                                         ymax, a.shape[1], bx0, bx1, by0, by1, int(hermx), 0, _c(out), mw,
                                         _lib.Device.stream()))
    o = out.cpu().numpy()
    if cplx:
        o = o.view(np.complex128 if f64 else np.complex64)
    return o.reshape(nw, mw)


@pytest.mark.parametrize('Nk,N', [(16, 8), (20, 8), (12, 12), (24, 12)])
@pytest.mark.parametrize('f64', [True, False])
def test_wrap_hermx_vs_reference(Nk, N, f64):
    """kimage.wrap(BoundsI(0, N/2, -N/2, N/2-1), hermitian='x') of a random (non-Hermitian)
    complex k-image with bounds (0, Nk/2, -Nk/2, Nk/2), as drawFFT wraps (image.py:789-796)."""
    a = GOLD['wrap_in_%d_%d' % (Nk, N)]
    got = _wrap(a, True, (0, Nk // 2, -Nk // 2, Nk // 2), (0, N // 2, -N // 2, N // 2 - 1), True, f64)
    ref = GOLD['wrap_out_%d_%d' % (Nk, N)]
    assert np.abs(got - ref).max() <= (1e-12 if f64 else 2e-6) * np.abs(ref).max()


def test_wrap_real_and_complex_vs_reference():
    got = _wrap(STD['wrapr_in'], False, (-7, 9, -5, 12), (-2, 3, -1, 4), False)
    assert np.abs(got - STD['wrapr_out']).max() <= 1e-12 * np.abs(STD['wrapr_out']).max()
    got = _wrap(STD['wrapc_in'], True, (-4, 7, -6, 8), (-1, 4, -3, 2), False)
    assert np.abs(got - STD['wrapc_out']).max() <= 1e-12 * np.abs(STD['wrapc_out']).max()


def _irfft(k, Nx, Ny, si, so, f64=True):
    import torch
    dt = np.complex128 if f64 else np.complex64
    d_in = _dev(k.astype(dt).view(np.float64 if f64 else np.float32))
    dev = d_in.device
    out = torch.full((Ny * (Nx + 2),), float('nan'), dtype=torch.float64, device=dev)
    wbytes = int(_lib.lib().gsb_irfft_workspace_size(Nx, Ny))
    work = torch.empty(wbytes, dtype=torch.uint8, device=dev)
    _lib.check(_lib.lib().gsb_irfft(_c(d_in), _lib.F64 if f64 else _lib.F32, Nx, Ny, Nx // 2 + 1, _c(out), Nx + 2,
                                    si, so, _c(work), ctypes.c_size_t(wbytes), _lib.Device.stream()))
    return out.cpu().numpy().reshape(Ny, Nx + 2)[:, :Nx]


@pytest.mark.parametrize('Nx,Ny', MG.STANDALONE_IRFFT)
@pytest.mark.parametrize('si', [0, 1])
@pytest.mark.parametrize('so', [0, 1])
def test_irfft_vs_reference(Nx, Ny, si, so):
    got = _irfft(STD['irfft_in_%d_%d' % (Nx, Ny)], Nx, Ny, si, so)
    ref = STD['irfft_out_%d_%d_%d%d' % (Nx, Ny, si, so)]
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize('Nk,N', [(16, 8), (20, 8), (12, 12), (24, 12)])
def test_wrap_then_irfft_as_drawfft(Nk, N):
    """drawFFT's two steps chained on the device: the reference's wrap + irfft(True, True)."""
    w = _wrap(GOLD['wrap_in_%d_%d' % (Nk, N)], True, (0, Nk // 2, -Nk // 2, Nk // 2),
              (0, N // 2, -N // 2, N // 2 - 1), True)
    got = _irfft(w, N, N, 1, 1)
    ref = GOLD['irfft_out_%d_%d' % (Nk, N)]
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_irfft_large_against_numpy():
    """A 3072 x 4096 transform (the block-wide FFT with radix-3 and radix-2 passes)."""
    Nx, Ny = 3072, 4096
    rng = np.random.default_rng(5)
    k = rng.normal(size=(Ny, Nx // 2 + 1)) + 1j * rng.normal(size=(Ny, Nx // 2 + 1))
    got = _irfft(k, Nx, Ny, 1, 1)
    K = np.concatenate([k[Ny // 2:], k[:Ny // 2]], axis=0)
    K = K * np.where((np.arange(Ny)[:, None] + np.arange(Nx // 2 + 1)[None, :]) % 2 == 0, 1., -1.)
    ref = np.fft.irfft2(K, s=(Ny, Nx))
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_standalone_argument_errors():
    import torch
    L = _lib.lib()
    d = torch.zeros(64, dtype=torch.float64, device=_lib.Device.torch_device())
    # irfft: sizes with a factor 5 are not built; odd sizes are invalid
    assert L.gsb_irfft(_c(d), _lib.F64, 10, 8, 6, _c(d), 12, 1, 1, _c(d), 512, None) == -3
    assert L.gsb_irfft(_c(d), _lib.F64, 7, 8, 6, _c(d), 12, 1, 1, _c(d), 512, None) == -1
    # wrap: hermitian x needs xmin == 0
    assert L.gsb_wrap_image(_c(d), _lib.F64, 1, -1, 4, -3, 3, 6, 0, 2, -2, 1, 1, 0, _c(d), 3, None) == -1
    assert L.gsb_wrap_image(_c(d), _lib.F64, 1, 0, 4, -3, 3, 5, 0, 2, -2, 1, 0, 1, _c(d), 3, None) == -3

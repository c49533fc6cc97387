"""GPU test of gsb_draw_images_noalloc, the drawing entry point that allocates nothing.

Some callers of this library cannot allocate device memory while they draw: an application
that hands the GPU a fixed memory budget up front, or a plugin that lives inside another
program's memory pool.  For them gsb_draw_images_noalloc takes its scratch from an array
compiled into the library instead of from a caller-provided workspace.  This test calls it
through the C ABI and checks its images and fluxes against gsb_draw_images (which uses a
workspace) on two calls in a row:
  * FFT sizes whose wrapped k-image does not fit in shared memory (so the scratch array is
    really used), FP32 and FP64;
  * more stamps than the array has slabs for (N = 1024: 7 FP32 / 3 FP64 slabs), so that the
    reduced grid's CTAs each draw several stamps through one slab;
  * a program with an InterpolatedImage leaf (an image PSF);
and that a stamp whose FFT size differs from the N argument, or an N beyond the limit, is
refused with an error.  The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _psf_image():
    y, x = np.mgrid[-12:12, -12:12] + 0.5
    return np.exp(-0.5 * (x * x + 1.3 * y * y + 0.4 * x * y) / 4.) + 0.02 * np.exp(-0.5 * (x * x + y * y) / 40.)


def _setup(N_img, B=5, image_psf=False, dtype=np.float32):
    import galsim_b200 as galsim
    from galsim_b200 import _lib
    from galsim_b200.program import fft_sizes
    sig = np.linspace(0.4, 0.6, B)
    gal = galsim.Gaussian(sigma=sig, flux=100.).shear(g1=0.1, g2=-0.05)
    psf = (galsim.InterpolatedImage(galsim.Image(_psf_image(), scale=0.2)) if image_psf
           else galsim.Kolmogorov(fwhm=0.7))
    plan = galsim.plan_batch(galsim.Convolve(gal, psf), nx=N_img, ny=N_img, scale=0.2, dtype=dtype)
    prog = plan.prog
    prog.compute_leaves()
    stepk, maxk = prog.stepk_maxk()
    xmin = np.full(B, -(N_img // 2))
    N, Nk = fft_sizes(stepk, maxk, xmin, xmin + N_img - 1, xmin, xmin + N_img - 1, prog.gsparams)
    assert len(set(N)) == 1
    stamps = np.zeros(B, dtype=_lib.STAMP_DTYPE)
    stamps['N'] = N
    stamps['Nk'] = Nk
    stamps['xmin'] = xmin
    stamps['ymin'] = xmin
    stamps['nx'] = N_img
    stamps['ny'] = N_img
    stamps['out_offset'] = np.arange(B) * N_img * N_img
    d_st = _lib.to_device(stamps)
    d_ph = _lib.to_device(np.stack(prog.bld.phases, axis=1)) if prog.bld.phases else None
    d_sc = _lib.to_device(np.stack(prog.bld.scales, axis=1)) if prog.bld.scales else None
    return prog, int(N[0]), B, stamps, d_st, d_ph, d_sc


def _noalloc():
    from galsim_b200 import _lib
    f = _lib.lib().gsb_draw_images_noalloc
    vp = ctypes.c_void_p
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(_lib.TemplateC), ctypes.c_int, ctypes.POINTER(_lib.GSParamsC), vp, vp, vp,
                  vp, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, vp]
    return f


def _opt(t):
    from galsim_b200 import _lib
    return _lib.ptr(t) if t is not None else None


def _compare_with_workspace_entry_point(N_img, f64, B=5, image_psf=False, min_N=256):
    import torch
    from galsim_b200 import _lib
    prog, N, B, _, d_st, d_ph, d_sc = _setup(N_img, B, image_psf)
    assert N >= min_N        # the wrapped k-image lives in scratch, not shared memory
    lib = _lib.lib()
    f = _noalloc()
    dev = _lib.Device.torch_device()
    prec = _lib.F64 if f64 else _lib.F32
    stream = _lib.Device.stream()
    tables = prog.tables.handle if prog.tables else None
    # the existing entry point, with a caller-provided workspace
    ref = torch.zeros(B * N_img * N_img, dtype=torch.float32, device=dev)
    ref_flux = torch.zeros(B, dtype=torch.float64, device=dev)
    wbytes = lib.gsb_draw_workspace_size(N, B, prec)
    work = torch.empty(max(int(wbytes), 8), dtype=torch.uint8, device=dev)
    _lib.check(lib.gsb_draw_images(ctypes.byref(prog.tpl), B, ctypes.byref(prog.gsp_c), _lib.ptr(prog.d_leaves),
                                   _opt(d_ph), _opt(d_sc), _lib.ptr(d_st), tables,
                                   _lib.ptr(ref), _lib.F32, 0, _lib.ptr(ref_flux), prec, _lib.ptr(work),
                                   ctypes.c_size_t(int(wbytes)), stream))
    torch.cuda.synchronize(dev)
    peak = float(ref.abs().max())
    for call in range(2):
        out = torch.full((B * N_img * N_img,), float('nan'), dtype=torch.float32, device=dev)
        flux = torch.zeros(B, dtype=torch.float64, device=dev)
        _lib.check(f(ctypes.byref(prog.tpl), B, ctypes.byref(prog.gsp_c), _lib.ptr(prog.d_leaves),
                     _opt(d_ph), _opt(d_sc), _lib.ptr(d_st), tables, N,
                     _lib.ptr(out), _lib.F32, 0, _lib.ptr(flux), prec, stream))
        torch.cuda.synchronize(dev)
        assert bool(torch.isfinite(out).all()), call
        assert float((out - ref).abs().max()) <= 1e-5 * peak, call
        assert np.allclose(flux.cpu().numpy(), ref_flux.cpu().numpy(), rtol=1e-6, atol=0), call
    return N


@pytest.mark.parametrize('N_img,f64', [(200, False), (400, False), (200, True)])
def test_noalloc_matches_workspace_entry_point(N_img, f64):
    _compare_with_workspace_entry_point(N_img, f64)


@pytest.mark.parametrize('f64,B', [(False, 9), (True, 8)])
def test_noalloc_more_stamps_than_scratch_slabs(f64, B):
    """N = 1024: the 32 MiB array holds 7 FP32 (3 FP64) wrapped k-image slabs, fewer than the
    stamps, so the grid is reduced and each CTA draws several stamps through its slab."""
    N = _compare_with_workspace_entry_point(800, f64, B=B, min_N=1024)
    assert N == 1024


def test_noalloc_image_psf():
    """A Gaussian galaxy convolved with an InterpolatedImage PSF."""
    _compare_with_workspace_entry_point(200, False, image_psf=True)


def test_noalloc_rejects_stamps_of_another_size():
    import torch
    from galsim_b200 import _lib
    prog, N, B, stamps, d_st, d_ph, d_sc = _setup(200)
    dev = _lib.Device.torch_device()
    # one stamp of the batch claims another FFT size than the call's N
    bad = stamps.copy()
    bad['N'][2] = 2 * N
    d_bad = _lib.to_device(bad)
    out = torch.zeros(B * 200 * 200, dtype=torch.float32, device=dev)
    rc = _noalloc()(ctypes.byref(prog.tpl), B, ctypes.byref(prog.gsp_c), _lib.ptr(prog.d_leaves),
                    _opt(d_ph), _opt(d_sc), _lib.ptr(d_bad), prog.tables.handle if prog.tables else None, N,
                    _lib.ptr(out), _lib.F32, 0, None, _lib.F32, _lib.Device.stream())
    assert rc == -1
    assert b'differs' in _lib.lib().gsb_last_error()
    assert float(out.abs().max()) == 0.          # nothing was drawn


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch
    from galsim_b200 import _lib
    prog, N, B, _, d_st, d_ph, d_sc = _setup(200)
    dev = _lib.Device.torch_device()
    out = torch.zeros(B * 200 * 200, dtype=torch.float32, device=dev)
    rc = _noalloc()(ctypes.byref(prog.tpl), B, ctypes.byref(prog.gsp_c), _lib.ptr(prog.d_leaves),
                    _opt(d_ph), _opt(d_sc), _lib.ptr(d_st), None, 2048, _lib.ptr(out), _lib.F32, 0, None,
                    _lib.F32, _lib.Device.stream())
    assert rc == -3
    assert b'1024' in _lib.lib().gsb_last_error()

"""GPU test of gsb_draw_images_noalloc, the drawing entry point that allocates nothing.

Some callers of this library cannot allocate device memory while they draw: an application
that hands the GPU a fixed memory budget up front, or a plugin that lives inside another
program's memory pool.  For them gsb_draw_images_noalloc takes its scratch from an array
compiled into the library instead of from a caller-provided workspace.  This test calls it
through the C ABI and checks its images and fluxes against gsb_draw_images (which uses a
workspace) on two calls in a row, for FFT sizes whose wrapped k-image does not fit in shared
memory (so the scratch array is really used).  The file is named so that pytest collects it
last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(N_img, precision_f64):
    import torch
    import galsim_b200 as galsim
    from galsim_b200 import _lib
    from galsim_b200.program import fft_sizes
    sig = np.array([0.4, 0.5, 0.6, 0.45, 0.55])
    obj = galsim.Convolve(galsim.Gaussian(sigma=sig, flux=100.).shear(g1=0.1, g2=-0.05),
                          galsim.Kolmogorov(fwhm=0.7))
    plan = galsim.plan_batch(obj, nx=N_img, ny=N_img, scale=0.2, dtype=np.float32)
    prog = plan.prog
    prog.compute_leaves()
    stepk, maxk = prog.stepk_maxk()
    B = prog.B
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
    return prog, int(N[0]), B, d_st, d_ph, d_sc


@pytest.mark.parametrize('N_img,f64', [(200, False), (400, False), (200, True)])
def test_noalloc_matches_workspace_entry_point(N_img, f64):
    import torch
    from galsim_b200 import _lib
    prog, N, B, d_st, d_ph, d_sc = _setup(N_img, f64)
    assert N >= 256          # the wrapped k-image lives in scratch, not shared memory
    lib = _lib.lib()
    f = lib.gsb_draw_images_noalloc
    vp = ctypes.c_void_p
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(_lib.TemplateC), ctypes.c_int, ctypes.POINTER(_lib.GSParamsC), vp, vp, vp,
                  vp, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, vp]
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
                                   _lib.ptr(d_ph) if d_ph is not None else None,
                                   _lib.ptr(d_sc) if d_sc is not None else None, _lib.ptr(d_st), tables,
                                   _lib.ptr(ref), _lib.F32, 0, _lib.ptr(ref_flux), prec, _lib.ptr(work),
                                   ctypes.c_size_t(int(wbytes)), stream))
    torch.cuda.synchronize(dev)
    peak = float(ref.abs().max())
    for call in range(2):
        out = torch.full((B * N_img * N_img,), float('nan'), dtype=torch.float32, device=dev)
        flux = torch.zeros(B, dtype=torch.float64, device=dev)
        _lib.check(f(ctypes.byref(prog.tpl), B, ctypes.byref(prog.gsp_c), _lib.ptr(prog.d_leaves),
                     _lib.ptr(d_ph) if d_ph is not None else None,
                     _lib.ptr(d_sc) if d_sc is not None else None, _lib.ptr(d_st), tables, N,
                     _lib.ptr(out), _lib.F32, 0, _lib.ptr(flux), prec, stream))
        torch.cuda.synchronize(dev)
        assert bool(torch.isfinite(out).all()), call
        assert float((out - ref).abs().max()) <= 1e-5 * peak, call
        assert np.allclose(flux.cpu().numpy(), ref_flux.cpu().numpy(), rtol=1e-6, atol=0), call


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch
    from galsim_b200 import _lib
    prog, N, B, d_st, d_ph, d_sc = _setup(200, False)
    lib = _lib.lib()
    f = lib.gsb_draw_images_noalloc
    vp = ctypes.c_void_p
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(_lib.TemplateC), ctypes.c_int, ctypes.POINTER(_lib.GSParamsC), vp, vp, vp,
                  vp, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, vp]
    dev = _lib.Device.torch_device()
    out = torch.zeros(B * 200 * 200, dtype=torch.float32, device=dev)
    rc = f(ctypes.byref(prog.tpl), B, ctypes.byref(prog.gsp_c), _lib.ptr(prog.d_leaves),
           _lib.ptr(d_ph) if d_ph is not None else None, _lib.ptr(d_sc) if d_sc is not None else None,
           _lib.ptr(d_st), None, 2048, _lib.ptr(out), _lib.F32, 0, None, _lib.F32, _lib.Device.stream())
    assert rc == -3
    assert b'1024' in lib.gsb_last_error()

"""Host-array adapters with the call shapes of the reference's compiled hot-path functions.

The reference's Python drives its FFT path through four functions of its pybind11 module
``_galsim``, each taking ImageView objects (pysrc/Image.cpp:25-37 builds them from a numpy
array's data pointer, strides and bounds):

    SBProfile.drawK(image, dk, jac_ptr)                            pysrc/SBProfile.cpp:35-40
    ApplyKImagePhases(image, dk, jac_ptr, cenx, ceny, flux_scaling) pysrc/SBTransform.cpp:27-40
    wrapImage(image, bounds, hermx, hermy)                         pysrc/Image.cpp:60-61
    irfft(in_image, out_image, shift_in, shift_out)                pysrc/Image.cpp:53-57

The functions here take the same arguments with each ImageView given as its numpy array and
bounds (xmin, xmax, ymin, ymax), and run the step on the GPU through the C ABI
(gsb_draw_k, gsb_apply_kimage_phases, gsb_wrap_image, gsb_irfft): the array is copied to the
device, the step runs there, and the result is copied back into the array, in place, as the
reference's functions write into their ImageView.  A reference maintainer who keeps
GSObject.drawFFT (galsim/gsobject.py:2014-2045) and replaces only these calls binds them as
INTEGRATION.md shows.  (The batched path, draw_batch, never leaves the device between steps.)
"""
import ctypes

import numpy as np

from . import _lib
from .errors import GalSimError, GalSimValueError

__all__ = ['drawK', 'ApplyKImagePhases', 'wrapImage', 'irfft']


def _torch():
    import torch
    return torch


def _to_dev(a):
    """A device copy of a C-contiguous numpy array, as a flat tensor of its real components."""
    torch = _torch()
    a = np.ascontiguousarray(a)
    if np.iscomplexobj(a):
        a = a.view(np.float64 if a.dtype == np.complex128 else np.float32)
    return torch.from_numpy(a.reshape(-1)).to(_lib.Device.torch_device())


def _back(t, arr):
    """Copy a device tensor back into the numpy array arr (same layout)."""
    h = t.cpu().numpy()
    if np.iscomplexobj(arr):
        h = h.view(arr.dtype)
    arr[...] = h.reshape(arr.shape)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _jac_arg(jac):
    if jac is None:
        return None, None
    j = np.ascontiguousarray(np.asarray(jac, dtype=np.float64).reshape(4))
    return j, j.ctypes.data_as(ctypes.c_void_p)


def _check_shape(array, bounds):
    xmin, xmax, ymin, ymax = bounds
    if array.shape != (ymax - ymin + 1, xmax - xmin + 1):
        raise GalSimValueError("array shape does not match bounds", (array.shape, bounds))


def drawK(prof, array, bounds, dk, jac=None):
    """SBProfile.drawK: draw the profile's k-values on the grid k = (i dk, j dk) of the
    complex array with the given bounds (complex64 or complex128), with the optional 2x2
    Jacobian jac (row-major) composed as Transformation._drawKImage does.  prof is a
    galsim_b200 GSObject (one profile)."""
    from .program import Program
    _check_shape(array, bounds)
    if array.dtype not in (np.complex64, np.complex128):
        raise GalSimValueError("drawK draws into a complex image", array.dtype)
    torch = _torch()
    prog = Program(prof)
    prog.prepare()
    ph = _lib.to_device(np.stack(prog.bld.phases, axis=1)) if prog.bld.phases else None
    sc = _lib.to_device(np.stack(prog.bld.scales, axis=1)) if prog.bld.scales else None
    xmin, xmax, ymin, ymax = bounds
    f64 = array.dtype == np.complex128
    out = torch.empty(array.size * 2, dtype=torch.float64 if f64 else torch.float32,
                      device=_lib.Device.torch_device())
    j, jp = _jac_arg(jac)
    _lib.check(_lib.lib().gsb_draw_k(
        ctypes.byref(prog.tpl), 1, ctypes.byref(prog.gsp_c), _lib.ptr(prog.d_leaves),
        _lib.ptr(ph) if ph is not None else None, _lib.ptr(sc) if sc is not None else None,
        prog.tables.handle if prog.tables else None, float(dk), jp, xmin, ymin, xmax - xmin + 1,
        ymax - ymin + 1, _ptr(out), _lib.F64 if f64 else _lib.F32, _lib.Device.stream()))
    _back(out, array)


def ApplyKImagePhases(array, bounds, dk, jac, cenx, ceny, flux_scaling):
    """ApplyKImagePhases: array *= flux_scaling exp(-i (kx' cenx + ky' ceny)) in place."""
    _check_shape(array, bounds)
    if array.dtype not in (np.complex64, np.complex128):
        raise GalSimValueError("ApplyKImagePhases needs a complex image", array.dtype)
    xmin, xmax, ymin, ymax = bounds
    d = _to_dev(array)
    j, jp = _jac_arg(jac)
    _lib.check(_lib.lib().gsb_apply_kimage_phases(
        _ptr(d), _lib.F64 if array.dtype == np.complex128 else _lib.F32, xmin, ymin, xmax - xmin + 1,
        ymax - ymin + 1, xmax - xmin + 1, float(dk), jp, float(cenx), float(ceny), float(flux_scaling),
        _lib.Device.stream()))
    _back(d, array)


def wrapImage(array, bounds, wrap_bounds, hermx, hermy):
    """wrapImage: fold the image onto wrap_bounds and write the result into that subimage of
    the array (the rest of the array is left as it was; the reference leaves partial sums
    there, which its callers do not read)."""
    _check_shape(array, bounds)
    xmin, xmax, ymin, ymax = bounds
    bx0, bx1, by0, by1 = wrap_bounds
    torch = _torch()
    cplx = np.iscomplexobj(array)
    f64 = array.dtype in (np.float64, np.complex128)
    if array.dtype not in (np.float32, np.float64, np.complex64, np.complex128):
        raise GalSimValueError("wrapImage supports float and complex images", array.dtype)
    d = _to_dev(array)
    mw, nw = bx1 - bx0 + 1, by1 - by0 + 1
    out = torch.empty(mw * nw * (2 if cplx else 1), dtype=d.dtype, device=d.device)
    _lib.check(_lib.lib().gsb_wrap_image(
        _ptr(d), _lib.F64 if f64 else _lib.F32, int(cplx), xmin, xmax, ymin, ymax, xmax - xmin + 1,
        bx0, bx1, by0, by1, int(bool(hermx)), int(bool(hermy)), _ptr(out), mw, _lib.Device.stream()))
    sub = np.empty((nw, mw), dtype=array.dtype)
    _back(out, sub)
    array[by0 - ymin:by1 - ymin + 1, bx0 - xmin:bx1 - xmin + 1] = sub


def irfft(in_array, in_bounds, out_array, out_bounds, shift_in, shift_out):
    """irfft: the inverse real FFT of the half plane in_array (bounds (0, Nx/2, -Ny/2,
    Ny/2-1)) into the float64 out_array (bounds (-Nx/2, Nx/2+1, -Ny/2, Ny/2-1)); the same
    bound checks and errors as the reference (src/Image.cpp:818-840)."""
    _check_shape(in_array, in_bounds)
    _check_shape(out_array, out_bounds)
    xmin, xmax, ymin, ymax = in_bounds
    if xmin != 0:
        raise GalSimError("inverse_fft requires bounds to be (0, Nx/2, -Ny/2, Ny/2-1)")
    Nxo2, Nyo2 = xmax, ymax + 1
    Nx, Ny = 2 * Nxo2, 2 * Nyo2
    if ymin != -Nyo2:
        raise GalSimError("inverse_fft requires bounds to be (0, N/2, -N/2, N/2-1)")
    if tuple(out_bounds) != (-Nxo2, Nxo2 + 1, -Nyo2, Nyo2 - 1):
        raise GalSimError("inverse_fft requires out.bounds to be (-Nx/2, Nx/2+1, -Ny/2, Ny/2-1)")
    if out_array.dtype != np.float64:
        raise GalSimValueError("irfft writes a float64 image", out_array.dtype)
    if in_array.dtype not in (np.complex64, np.complex128):
        raise GalSimValueError("irfft reads a complex image", in_array.dtype)
    torch = _torch()
    d_in = _to_dev(in_array)
    d_out = torch.empty(out_array.size, dtype=torch.float64, device=d_in.device)
    wbytes = int(_lib.lib().gsb_irfft_workspace_size(Nx, Ny))
    work = torch.empty(max(wbytes, 8), dtype=torch.uint8, device=d_in.device)
    _lib.check(_lib.lib().gsb_irfft(
        _ptr(d_in), _lib.F64 if in_array.dtype == np.complex128 else _lib.F32, Nx, Ny, Nxo2 + 1,
        _ptr(d_out), Nx + 2, int(bool(shift_in)), int(bool(shift_out)), _ptr(work), ctypes.c_size_t(wbytes),
        _lib.Device.stream()))
    h = d_out.cpu().numpy().reshape(Ny, Nx + 2)
    out_array[:, :Nx] = h[:, :Nx]

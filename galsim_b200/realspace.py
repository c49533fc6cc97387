"""Real-space drawing (drawReal, gsobject.py:1846-1898) of profiles that are analytic in real
space: sums and affine transformations of Gaussian, Exponential, Sersic, Moffat, Kolmogorov,
Airy and Box leaves and InterpolatedImages (their x interpolant over the image's pixels,
SBInterpolatedImage::xValue).

The reference draws such a profile (method 'no_pixel' or 'sb', gsobject.py:1810-1811) by
walking the tree with _drawReal -- each Transformation composes its Jacobian, offset and flux
scaling into the arguments (transform.py:571-583), a Sum draws each member (sum.py:304-310) --
and drawing each leaf with SBProfile::draw.  Here the walk is done once on the host into one
gsb_xleaf record per (stamp, leaf), and one kernel (gsb_draw_real) evaluates every stamp's
leaves at every pixel on the device.
"""
import ctypes

import numpy as np

from . import _lib
from .errors import GalSimNotImplementedError

__all__ = ['xleaf_records', 'draw_real_stamps']


def _collect(obj, jac, dx, dy, fs, out):
    from .compound import Transformation, Sum
    from .profiles import _Leaf
    from .interpolatedimage import InterpolatedImage, _ImageLeaf
    if isinstance(obj, InterpolatedImage):
        _collect(obj._inner, jac, dx, dy, fs, out)
        return
    if isinstance(obj, Transformation):
        if np.any(obj._has_offset):
            if jac is not None:
                x1 = jac[..., 0, 0] * obj._dx + jac[..., 0, 1] * obj._dy
                y1 = jac[..., 1, 0] * obj._dx + jac[..., 1, 1] * obj._dy
            else:
                x1, y1 = obj._dx, obj._dy
            dx = dx + x1
            dy = dy + y1
        fs = fs * obj._flux_scaling
        if jac is None:
            jac = obj._jac
        elif obj._jac is not None:
            jac = np.matmul(jac, obj._jac)
        _collect(obj._original, jac, dx, dy, fs, out)
    elif isinstance(obj, Sum):
        for o in obj.obj_list:
            _collect(o, jac, dx, dy, fs, out)
    elif isinstance(obj, (_Leaf, _ImageLeaf)):
        out.append((obj, jac, dx, dy, fs))
    else:
        raise GalSimNotImplementedError("real-space drawing of %s is not built" % type(obj).__name__)


def _leaf_params(leaf):
    from .profiles import Sersic
    if isinstance(leaf, Sersic):
        return (leaf.n, leaf.scale_radius, leaf.trunc)
    p = leaf._params()
    return tuple(p) + (0.,) * (3 - len(p))


def _image_leaf(arr, l, leaf, B, keep):
    """An InterpolatedImage leaf: its sources' nonzero regions in one device buffer (kept alive
    in `keep`), each stamp pointing at its own source's region."""
    import torch
    from .interpolant import Delta, Lanczos
    xi = leaf._x_interpolant
    if xi._code is None or isinstance(xi, Delta):
        raise GalSimNotImplementedError("real-space drawing of an InterpolatedImage with x interpolant "
                                        "%s is not built" % (xi,))
    srcs = leaf._sources
    flat = np.concatenate([np.ascontiguousarray(s.region, dtype=np.float64).ravel() for s in srcs])
    d = torch.from_numpy(flat).to(_lib.Device.torch_device())
    keep.append(d)
    offs = np.concatenate([[0], np.cumsum([s.region.size for s in srcs])[:-1]]).astype(np.int64)
    idx = np.arange(B) % len(srcs) if len(srcs) > 1 else np.zeros(B, np.int64)
    arr['type'][:, l] = _lib.INTERPOLATED
    arr['flux'][:, l] = 1.
    arr['p'][:, l, 0] = float(xi._code)
    arr['region'][:, l] = d.data_ptr() + 8 * offs[idx]
    arr['rx0'][:, l] = [srcs[i].x0 for i in idx]
    arr['ry0'][:, l] = [srcs[i].y0 for i in idx]
    arr['rnx'][:, l] = [srcs[i].region.shape[1] for i in idx]
    arr['rny'][:, l] = [srcs[i].region.shape[0] for i in idx]
    if isinstance(xi, Lanczos):
        kt = xi._table.kdevice()
        keep.append(kt)
        arr['ktab'][:, l] = kt.data_ptr()


def xleaf_records(prof, B, keep=None):
    """The (B, L) gsb_xleaf records of profile `prof` (batch size B); device buffers the records
    point at are appended to `keep`."""
    from .interpolatedimage import _ImageLeaf
    recs = []
    _collect(prof, None, 0., 0., 1., recs)
    if len(recs) > _lib.MAX_LEAVES:
        from .errors import GalSimError
        raise GalSimError("profile tree has more than %d leaves" % _lib.MAX_LEAVES)
    keep = [] if keep is None else keep
    arr = np.zeros((B, len(recs)), dtype=_lib.XLEAF_DTYPE)
    for l, (leaf, jac, dx, dy, fs) in enumerate(recs):
        if isinstance(leaf, _ImageLeaf):
            _image_leaf(arr, l, leaf, B, keep)
        else:
            arr['type'][:, l] = leaf._type
            arr['flux'][:, l] = np.broadcast_to(np.asarray(leaf.flux, float), (B,))
            for k, v in enumerate(_leaf_params(leaf)):
                arr['p'][:, l, k] = np.broadcast_to(np.asarray(v, float), (B,))
        arr['xoff'][:, l] = np.broadcast_to(np.asarray(dx, float), (B,))
        arr['yoff'][:, l] = np.broadcast_to(np.asarray(dy, float), (B,))
        arr['flux_ratio'][:, l] = np.broadcast_to(np.asarray(fs, float), (B,))
        if jac is not None:
            j = np.broadcast_to(np.asarray(jac, float), (B, 2, 2))
            arr['jac'][:, l] = j.reshape(B, 4)
            arr['flags'][:, l] = _lib.XLEAF_JAC
    return arr


def draw_real_stamps(prof, B, gsparams, xmin, ymin, nx, ny, dtype, init=None):
    """Draw the B stamps of `prof` in real space: stamp s covers image positions
    xmin[s] .. xmin[s] + nx[s] - 1 (and likewise y) around the profile origin.  Returns the flat
    device output (stamps packed row-major), the offsets and the per-stamp drawn fluxes (device).
    init: optional flat device tensor to add to (add_to_image)."""
    import torch
    keep = []
    rec = xleaf_records(prof, B, keep)
    dev = _lib.Device.torch_device()
    nx = np.broadcast_to(np.asarray(nx, np.int64), (B,))
    ny = np.broadcast_to(np.asarray(ny, np.int64), (B,))
    sizes = nx * ny
    offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    stamps = np.zeros(B, dtype=_lib.STAMP_DTYPE)
    stamps['xmin'] = np.broadcast_to(np.asarray(xmin), (B,))
    stamps['ymin'] = np.broadcast_to(np.asarray(ymin), (B,))
    stamps['nx'] = nx
    stamps['ny'] = ny
    stamps['out_offset'] = offsets
    f64 = np.dtype(dtype) == np.float64
    tdt = torch.float64 if f64 else torch.float32
    if init is not None:
        out = init
        add = 1
    else:
        out = torch.empty(int(sizes.sum()), dtype=tdt, device=dev)
        add = 0
    flux = torch.zeros(B, dtype=torch.float64, device=dev)
    d_rec = _lib.to_device(np.ascontiguousarray(rec))
    d_st = _lib.to_device(stamps)
    _lib.check(_lib.lib().gsb_draw_real(rec.shape[1], B, ctypes.byref(_lib.gsparams_c(gsparams)),
                                        _lib.ptr(d_rec), _lib.ptr(d_st), _lib.ptr(out),
                                        _lib.F64 if f64 else _lib.F32, add, _lib.ptr(flux),
                                        _lib.Device.stream()))
    return out, offsets, flux

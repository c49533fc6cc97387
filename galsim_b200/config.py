"""Config-driven batched drawing: a GalSim config dict (the `gal`, `psf`, `image` and `stamp`
fields of galsim/config) turned into ONE batched GSObject for all objects and drawn with
draw_batch, instead of the reference's per-object BuildStamp -> drawImage loop
(galsim/config/stamp.py:244-558, run one process per core by config/util.py:672).

Supported (the FFT-path subset of the reference's config):
* object types Gaussian, Exponential, Sersic, DeVaucouleurs, Moffat, Kolmogorov, Airy, Box,
  Pixel, Sum / Add, Convolve / Convolution, with `flux` and the transformations of
  config/gsobject.py:515-549 in the reference's order: dilate/dilation, ellip, rotate/rotation,
  scale_flux, lens, shear, magnify/magnification, shift;
* values: constants, strings with a unit for angles ('30 deg'), and the types List, Sequence,
  Sum, Catalog (columns of the `catalog` argument instead of an input file), G1G2, E1E2,
  EtaBeta-free shears GBeta / EBeta / QBeta, XY, Radians, Degrees;
* stamps: gal convolved with psf (config/stamp.py:860-886), size from stamp.size / xsize /
  ysize or image.stamp_size / image.size / xsize / ysize, image.pixel_scale, stamp.offset,
  stamp.draw_method (default 'auto').
Random value types, input files, noise and output are not part of the FFT path and raise
GalSimConfigError.
"""
import math

import numpy as np

from .errors import GalSimConfigError, GalSimConfigValueError


class _Ctx(object):
    def __init__(self, nobj, catalog):
        self.nobj = nobj
        self.catalog = catalog
        self.index = np.arange(nobj)


def _vec(ctx, v):
    a = np.asarray(v, dtype=np.float64)
    return np.broadcast_to(a, (ctx.nobj,)) if a.ndim == 0 else a


def _angle(ctx, v):
    """Radians per object."""
    from .angle import Angle, AngleUnit
    if isinstance(v, Angle):
        return _vec(ctx, v.rad)
    if isinstance(v, str):
        parts = v.split()
        if len(parts) != 2:
            raise GalSimConfigValueError("Cannot parse angle", v)
        return _vec(ctx, float(parts[0]) * AngleUnit.from_name(parts[1]).value)
    if isinstance(v, dict):
        t = v.get('type')
        if t == 'Radians':
            return _float(ctx, v['theta'])
        if t == 'Degrees':
            return _float(ctx, v['theta']) * (math.pi / 180.)
        if t == 'List':
            return _list(ctx, v, _angle)
        raise GalSimConfigError("Unsupported Angle value type %r" % t)
    raise GalSimConfigValueError("Invalid angle value", v)


def _list(ctx, v, parse):
    items = [parse(ctx, it) for it in v['items']]
    idx = _float(ctx, v['index']).astype(np.int64) if 'index' in v else ctx.index
    stacked = np.stack([np.broadcast_to(it, (ctx.nobj,)) for it in items])
    return stacked[idx % len(items), np.arange(ctx.nobj)]


def _float(ctx, v):
    if isinstance(v, (int, float, np.integer, np.floating)) and not isinstance(v, bool):
        return _vec(ctx, float(v))
    if isinstance(v, np.ndarray):
        return _vec(ctx, v)
    if isinstance(v, dict):
        t = v.get('type')
        if t == 'List':
            return _list(ctx, v, _float)
        if t == 'Sequence':
            # config/value.py _GenerateFromSequence: first + step * (index // repeat), wrapping
            # at nitems (or at last)
            first = float(v.get('first', 0))
            step = float(v.get('step', 1))
            repeat = int(v.get('repeat', 1))
            k = ctx.index // repeat
            if 'nitems' in v:
                k = k % int(v['nitems'])
            elif 'last' in v:
                k = k % (int(round((float(v['last']) - first) / step)) + 1)
            return first + step * k
        if t == 'Sum':
            return sum(_float(ctx, it) for it in v['items'])
        if t == 'Catalog':
            if ctx.catalog is None:
                raise GalSimConfigError("Catalog values need the catalog argument")
            col = np.asarray(ctx.catalog[v['col']], dtype=np.float64)
            if len(col) < ctx.nobj:
                raise GalSimConfigError("Catalog column %r has fewer than %d rows" % (v['col'], ctx.nobj))
            return col[:ctx.nobj]
        raise GalSimConfigError("Unsupported float value type %r" % t)
    raise GalSimConfigValueError("Invalid float value", v)


def _shear(ctx, v):
    """(g1, g2) per object."""
    from .shear import _e2g
    if not isinstance(v, dict):
        raise GalSimConfigValueError("Invalid shear value", v)
    t = v.get('type')
    if t == 'G1G2':
        return _float(ctx, v.get('g1', 0.)), _float(ctx, v.get('g2', 0.))
    if t == 'E1E2':
        e1, e2 = _float(ctx, v.get('e1', 0.)), _float(ctx, v.get('e2', 0.))
        f = _e2g(e1 * e1 + e2 * e2)
        return e1 * f, e2 * f
    if t in ('GBeta', 'EBeta', 'QBeta'):
        beta = _angle(ctx, v['beta'])
        if t == 'GBeta':
            g = _float(ctx, v['g'])
        elif t == 'EBeta':
            e = _float(ctx, v['e'])
            g = e * _e2g(e * e)
        else:
            q = _float(ctx, v['q'])
            g = (1. - q) / (1. + q)
        return g * np.cos(2. * beta), g * np.sin(2. * beta)
    if t == 'List':
        pairs = [_shear(ctx, it) for it in v['items']]
        idx = _float(ctx, v['index']).astype(np.int64) if 'index' in v else ctx.index
        g1 = np.stack([np.broadcast_to(p[0], (ctx.nobj,)) for p in pairs])
        g2 = np.stack([np.broadcast_to(p[1], (ctx.nobj,)) for p in pairs])
        sel = idx % len(pairs), np.arange(ctx.nobj)
        return g1[sel], g2[sel]
    raise GalSimConfigError("Unsupported Shear value type %r" % t)


def _position(ctx, v):
    if isinstance(v, dict) and v.get('type') == 'XY':
        return _float(ctx, v.get('x', 0.)), _float(ctx, v.get('y', 0.))
    raise GalSimConfigError("Unsupported PositionD value %r" % (v,))


_SIMPLE = {
    'Gaussian': ('sigma', 'fwhm', 'half_light_radius', 'flux'),
    'Exponential': ('half_light_radius', 'scale_radius', 'flux'),
    'Sersic': ('n', 'half_light_radius', 'scale_radius', 'flux', 'trunc'),
    'DeVaucouleurs': ('half_light_radius', 'scale_radius', 'flux', 'trunc'),
    'Moffat': ('beta', 'scale_radius', 'half_light_radius', 'fwhm', 'trunc', 'flux'),
    'Kolmogorov': ('lam_over_r0', 'fwhm', 'half_light_radius', 'flux'),
    'Airy': ('lam_over_diam', 'obscuration', 'flux'),
    'Box': ('width', 'height', 'flux'),
    'Pixel': ('scale', 'flux'),
}
_TRANSFORM_KEYS = ('dilate', 'dilation', 'ellip', 'rotate', 'rotation', 'scale_flux', 'lens',
                   'shear', 'magnify', 'magnification', 'shift')
_OTHER_KEYS = ('type', 'items', 'gsparams') + _TRANSFORM_KEYS


def build_object(ctx, cfg, gsparams=None):
    """The batched GSObject of one config object section (config/gsobject.py BuildGSObject)."""
    from . import compound, profiles, box
    if not isinstance(cfg, dict) or 'type' not in cfg:
        raise GalSimConfigError("object section needs a type: %r" % (cfg,))
    t = cfg['type']
    if t in _SIMPLE:
        unknown = set(cfg) - set(_SIMPLE[t]) - set(_OTHER_KEYS)
        if unknown:
            raise GalSimConfigError("Unexpected %s parameters %s" % (t, sorted(unknown)))
        kw = {k: _float(ctx, cfg[k]) for k in _SIMPLE[t] if k in cfg}
        cls = {'Gaussian': profiles.Gaussian, 'Exponential': profiles.Exponential,
               'Sersic': profiles.Sersic, 'DeVaucouleurs': profiles.DeVaucouleurs,
               'Moffat': profiles.Moffat, 'Kolmogorov': profiles.Kolmogorov, 'Airy': profiles.Airy,
               'Box': box.Box, 'Pixel': box.Pixel}[t]
        obj = cls(gsparams=gsparams, **kw)
    elif t in ('Sum', 'Add', 'Convolve', 'Convolution'):
        items = [build_object(ctx, it, gsparams) for it in cfg['items']]
        obj = (compound.Add if t in ('Sum', 'Add') else compound.Convolve)(items, gsparams=gsparams)
        if 'flux' in cfg:
            obj = obj.withFlux(_float(ctx, cfg['flux']))
    else:
        raise GalSimConfigError("Unsupported object type %r" % t)
    return transform_object(ctx, obj, cfg)


def transform_object(ctx, obj, cfg):
    """The transformations of config/gsobject.py:515-549, in that order."""
    from .shear import Shear
    for key in _TRANSFORM_KEYS:
        if key not in cfg:
            continue
        v = cfg[key]
        if key in ('dilate', 'dilation'):
            obj = obj.dilate(_float(ctx, v))
        elif key in ('ellip', 'shear'):
            g1, g2 = _shear(ctx, v)
            obj = obj.shear(Shear(g1=g1, g2=g2))
        elif key in ('rotate', 'rotation'):
            th = _angle(ctx, v)
            c, s = np.cos(th), np.sin(th)
            obj = obj.transform(c, -s, s, c)
        elif key == 'scale_flux':
            obj = obj * _float(ctx, v)
        elif key == 'lens':
            obj = obj.lens(_float(ctx, v['g1']), _float(ctx, v['g2']), _float(ctx, v['mu']))
        elif key in ('magnify', 'magnification'):
            obj = obj.magnify(_float(ctx, v))
        elif key == 'shift':
            dx, dy = _position(ctx, v)
            obj = obj.shift(dx, dy)
    return obj


def _size(config):
    st = config.get('stamp', {})
    im = config.get('image', {})
    for sec, keys in ((st, ('size', 'xsize', 'ysize')), (im, ('stamp_size', 'size', 'xsize', 'ysize'))):
        if any(k in sec for k in keys):
            sz = sec.get('size', sec.get('stamp_size'))
            nx = int(sec.get('xsize', sz)) if sec.get('xsize', sz) is not None else None
            ny = int(sec.get('ysize', sz)) if sec.get('ysize', sz) is not None else None
            return nx, ny
    return None, None


def build_batch(config, nobjects=None, catalog=None):
    """The batched profile that config's stamps draw (gal convolved with psf) and the number of
    objects."""
    im = config.get('image', {})
    if nobjects is None:
        nobjects = im.get('nobjects')
    if nobjects is None and catalog is not None:
        first = next(iter(catalog.values())) if isinstance(catalog, dict) else catalog[catalog.dtype.names[0]]
        nobjects = len(first)
    if nobjects is None:
        raise GalSimConfigError("number of objects unknown: give nobjects, image.nobjects or a catalog")
    ctx = _Ctx(int(nobjects), catalog)
    gal = build_object(ctx, config['gal']) if 'gal' in config else None
    psf = build_object(ctx, config['psf']) if 'psf' in config else None
    if gal is None and psf is None:
        raise GalSimConfigError("config has neither gal nor psf")
    from .compound import Convolve
    prof = Convolve(gal, psf) if gal is not None and psf is not None else (gal if gal is not None else psf)
    return prof, ctx


def draw_config(config, nobjects=None, catalog=None, dtype=np.float32, precision='fp32'):
    """Draw every stamp of `config` as one batch on the GPU; returns a StampBatch whose stamp i is
    the reference's BuildStamp for object i (FFT and no_pixel methods)."""
    from .batch import draw_batch
    prof, ctx = build_batch(config, nobjects, catalog)
    im = config.get('image', {})
    st = config.get('stamp', {})
    scale = im.get('pixel_scale', 1.0)
    method = st.get('draw_method', im.get('draw_method', 'auto'))
    if method not in ('auto', 'fft', 'no_pixel'):
        raise GalSimConfigValueError("draw_method on the FFT path", method, ('auto', 'fft', 'no_pixel'))
    offset = None
    if 'offset' in st:
        dx, dy = _position(ctx, st['offset'])
        offset = np.stack([dx, dy], -1)
    nx, ny = _size(config)
    return draw_batch(prof, nx=nx, ny=ny, scale=float(scale), dtype=dtype, method=method, offset=offset,
                      precision=precision)


__all__ = ['draw_config', 'build_batch', 'build_object']

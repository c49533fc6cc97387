"""Composite profiles: Convolution, Sum and Transformation (convolve.py, sum.py, transform.py).

On the GPU a composite is a sequence of program ops: a Convolution multiplies its members'
k-values (convolve.py:420-426), a Sum adds them (sum.py:341-347), and a Transformation
composes its Jacobian into its leaves and then applies its shift phase or flux factor
(transform.py:592-602).  Their stepk / maxk follow the reference's rules exactly.
"""
import math

import numpy as np

from . import _lib
from .errors import GalSimError, GalSimIncompatibleValuesError, galsim_warn
from .gsobject import GSObject, _as_param, _plen
from .gsparams import GSParams
from .position import Position, PositionD


def _compose(a, b):
    """jac a . jac b with None meaning identity (transform.py:593)."""
    if a is None:
        return b
    if b is None:
        return a
    return np.matmul(a, b)


def _batch_of(objs):
    n = 1
    for o in objs:
        if o._batch != 1:
            if n != 1 and n != o._batch:
                raise GalSimIncompatibleValuesError("batched members have different batch sizes")
            n = o._batch
    return n


def Convolve(*args, **kwargs):
    """Convolve 2 or more GSObjects (convolve.py:32-68)."""
    if len(args) == 0:
        raise TypeError("At least one ChromaticObject or GSObject must be provided.")
    elif len(args) == 1:
        from .chromatic import ChromaticObject
        if isinstance(args[0], (GSObject, ChromaticObject)):
            args = [args[0]]
        elif isinstance(args[0], (list, tuple)):
            args = args[0]
        else:
            raise TypeError("Single input argument must be a GSObject, ChromaticObject, "
                            "or a (possibly mixed) list of them.")
    from .chromatic import ChromaticObject, ChromaticConvolution
    if any(isinstance(a, ChromaticObject) for a in args):
        return ChromaticConvolution(*args, **kwargs)
    return Convolution(*args, **kwargs)


class Convolution(GSObject):
    """Convolution of several GSObjects; drawn by multiplying their FTs (convolve.py:71-436)."""

    def __init__(self, *args, **kwargs):
        if len(args) == 0:
            raise TypeError("At least one GSObject must be provided.")
        elif len(args) == 1:
            if isinstance(args[0], GSObject):
                args = [args[0]]
            elif isinstance(args[0], (list, tuple)):
                args = args[0]
            else:
                raise TypeError("Single input argument must be a GSObject or list of them.")
        real_space = kwargs.pop("real_space", None)
        gsparams = kwargs.pop("gsparams", None)
        self._propagate_gsparams = kwargs.pop('propagate_gsparams', True)
        if kwargs:
            raise TypeError("Convolution constructor got unexpected keyword argument(s): %s" %
                            kwargs.keys())
        hard_edge = True
        for obj in args:
            if not isinstance(obj, GSObject):
                raise TypeError("Arguments to Convolution must be GSObjects, not %s" % obj)
            if not obj.has_hard_edges:
                hard_edge = False
        if real_space is None:
            real_space = hard_edge if len(args) <= 2 else False
        elif bool(real_space) != real_space:
            raise TypeError("real_space must be a boolean")
        if not real_space and hard_edge:
            if len(args) == 2:
                galsim_warn("Doing convolution of 2 objects, both with hard edges. "
                            "This might be more accurate and/or faster using real_space=True")
            else:
                galsim_warn("Doing convolution where all objects have hard edges. "
                            "There might be some inaccuracies due to ringing in k-space.")
        if real_space:
            if len(args) > 2:
                galsim_warn("Real-space convolution of more than 2 objects is not implemented. "
                            "Switching to DFT method.")
                real_space = False
            else:
                for obj in args:
                    if not obj.is_analytic_x:
                        galsim_warn("A component to be convolved is not analytic in real space. "
                                    "Cannot use real space convolution. Switching to DFT method.")
                        real_space = False
                        break
        self._real_space = bool(real_space)
        if gsparams is None:
            self._gsparams = GSParams.combine([obj.gsparams for obj in args])
        else:
            self._gsparams = GSParams.check(gsparams)
        if self._propagate_gsparams:
            self._obj_list = [obj.withGSParams(self._gsparams) for obj in args]
        else:
            self._obj_list = list(args)
        self._batch = _batch_of(self._obj_list)

    obj_list = property(lambda self: self._obj_list)
    real_space = property(lambda self: self._real_space)

    @property
    def flux(self):
        f = 1.
        for obj in self._obj_list:
            f = f * obj.flux
        return f

    @property
    def _has_hard_edges(self):
        return len(self._obj_list) == 1 and self._obj_list[0].has_hard_edges

    @property
    def _is_axisymmetric(self):
        return all(obj.is_axisymmetric for obj in self._obj_list)

    @property
    def _is_analytic_x(self):
        return len(self._obj_list) == 1 and self._obj_list[0].is_analytic_x

    def withGSParams(self, gsparams=None, **kwargs):
        if gsparams == self.gsparams and not kwargs:
            return self
        import copy
        ret = copy.copy(self)
        ret._gsparams = GSParams.check(gsparams, self.gsparams, **kwargs)
        ret.__dict__.pop('_cached_sizes', None)
        if self._propagate_gsparams:
            ret._obj_list = [obj.withGSParams(ret._gsparams) for obj in self._obj_list]
        return ret

    def _flatten(self, bld, jac):
        self._obj_list[0]._flatten(bld, jac)
        for obj in self._obj_list[1:]:
            obj._flatten(bld, jac)
            bld.add_op(_lib.OP_MUL)

    def _size(self, prog, it):
        sizes = [obj._size(prog, it) for obj in self._obj_list]
        # convolve.py:296-305: min maxk; 1/stepk^2 = sum 1/stepk_i^2
        maxk = sizes[0][1]
        for s in sizes[1:]:
            maxk = np.minimum(maxk, s[1])
        inv = 0
        for s in sizes:
            inv = inv + s[0] ** (-2)
        return inv ** (-0.5), maxk

    def __eq__(self, other):
        return self is other or (isinstance(other, Convolution) and
                                 self.obj_list == other.obj_list and
                                 self.real_space == other.real_space and
                                 self.gsparams == other.gsparams)

    def __hash__(self):
        return hash(("galsim.Convolution", tuple(self.obj_list), self.real_space, self.gsparams))

    def __repr__(self):
        return 'galsim.Convolution(%r, real_space=%r, gsparams=%r)' % (
            self.obj_list, self.real_space, self.gsparams)


def Add(*args, **kwargs):
    """Sum of GSObjects (sum.py:33-60)."""
    if len(args) == 0:
        raise TypeError("At least one ChromaticObject or GSObject must be provided.")
    elif len(args) == 1:
        from .chromatic import ChromaticObject
        if isinstance(args[0], (GSObject, ChromaticObject)):
            args = [args[0]]
        elif isinstance(args[0], (list, tuple)):
            args = args[0]
        else:
            raise TypeError("Single input argument must be a GSObject or a list of them.")
    from .chromatic import ChromaticObject, ChromaticSum
    if any(isinstance(a, ChromaticObject) for a in args):
        return ChromaticSum(*args, **kwargs)
    return Sum(*args, **kwargs)


class Sum(GSObject):
    """A sum of GSObjects; drawn by adding their FTs (sum.py:63-356)."""

    def __init__(self, *args, **kwargs):
        if len(args) == 0:
            raise TypeError("At least one GSObject must be provided.")
        elif len(args) == 1:
            if isinstance(args[0], GSObject):
                args = [args[0]]
            elif isinstance(args[0], (list, tuple)):
                args = list(args[0])
            else:
                raise TypeError("Single input argument must be a GSObject or list of them.")
        gsparams = kwargs.pop("gsparams", None)
        self._propagate_gsparams = kwargs.pop('propagate_gsparams', True)
        if kwargs:
            raise TypeError("Add constructor got unexpected keyword argument(s): %s" % kwargs.keys())
        for obj in args:
            if not isinstance(obj, GSObject):
                raise TypeError("Arguments to Sum must be GSObjects, not %s" % obj)
        if gsparams is None:
            self._gsparams = GSParams.combine([obj.gsparams for obj in args])
        else:
            self._gsparams = GSParams.check(gsparams)
        if self._propagate_gsparams:
            self._obj_list = [obj.withGSParams(self._gsparams) for obj in args]
        else:
            self._obj_list = list(args)
        self._batch = _batch_of(self._obj_list)

    obj_list = property(lambda self: self._obj_list)

    @property
    def flux(self):
        f = 0.
        for obj in self._obj_list:
            f = f + obj.flux
        return f

    @property
    def _has_hard_edges(self):
        return any(obj.has_hard_edges for obj in self._obj_list)

    @property
    def _is_axisymmetric(self):
        return all(obj.is_axisymmetric for obj in self._obj_list)

    @property
    def _is_analytic_x(self):
        return all(obj.is_analytic_x for obj in self._obj_list)

    withGSParams = Convolution.withGSParams

    def _flatten(self, bld, jac):
        self._obj_list[0]._flatten(bld, jac)
        for obj in self._obj_list[1:]:
            obj._flatten(bld, jac)
            bld.add_op(_lib.OP_ADD)

    def _size(self, prog, it):
        sizes = [obj._size(prog, it) for obj in self._obj_list]
        # sum.py:243-251: max maxk, min stepk
        stepk, maxk = sizes[0]
        for s in sizes[1:]:
            stepk = np.minimum(stepk, s[0])
            maxk = np.maximum(maxk, s[1])
        return stepk, maxk

    def __eq__(self, other):
        return self is other or (isinstance(other, Sum) and self.obj_list == other.obj_list and
                                 self.gsparams == other.gsparams)

    def __hash__(self):
        return hash(("galsim.Sum", tuple(self.obj_list), self.gsparams))

    def __repr__(self):
        return 'galsim.Sum(%r, gsparams=%r)' % (self.obj_list, self.gsparams)


def _as_jac(jac):
    """A Jacobian given as None, 4 numbers, a (2,2) array or a (B,2,2) stack."""
    if jac is None:
        return None
    j = np.asarray(jac, dtype=np.float64)
    if j.shape == (4,):
        return j.reshape(2, 2)
    if j.ndim == 1 and j.size == 4:
        return j.reshape(2, 2)
    if j.shape[-2:] == (2, 2):
        return j
    if j.ndim == 2 and j.shape[0] == 4:     # four arrays (dudx, dudy, dvdx, dvdy)
        return np.moveaxis(j, 0, -1).reshape(j.shape[1], 2, 2)
    raise TypeError("Invalid jacobian shape %s" % (j.shape,))


def Transform(obj, jac=None, offset=(0., 0.), flux_ratio=1., gsparams=None, propagate_gsparams=True):
    """An affine transformation of a GSObject (transform.py:40-80)."""
    from .chromatic import ChromaticObject, _Transform as _chromatic_transform
    from .sed import SED
    if isinstance(obj, ChromaticObject) or hasattr(jac, '__call__') or hasattr(offset, '__call__') or \
            isinstance(flux_ratio, SED) or hasattr(flux_ratio, '__call__'):
        return _chromatic_transform(obj, jac, offset, flux_ratio, gsparams, propagate_gsparams)
    if not isinstance(obj, GSObject):
        raise TypeError("Argument to Transform must be a GSObject.")
    return Transformation(obj, jac, offset, flux_ratio, gsparams, propagate_gsparams)


class Transformation(GSObject):
    """obj transformed by jac, shifted by offset and scaled by flux_ratio (transform.py:83-604).
    jac, offset and flux_ratio may be batched (arrays over stamps)."""

    def __init__(self, obj, jac=None, offset=(0., 0.), flux_ratio=1., gsparams=None,
                 propagate_gsparams=True):
        self._jac = _as_jac(jac)
        if isinstance(offset, Position):
            dx, dy = offset.x, offset.y
        else:
            dx, dy = offset[0], offset[1]
        self._dx = _as_param(dx)
        self._dy = _as_param(dy)
        self._flux_ratio = _as_param(flux_ratio)
        self._gsparams = GSParams.check(gsparams, obj.gsparams)
        self._propagate_gsparams = propagate_gsparams
        if self._propagate_gsparams:
            obj = obj.withGSParams(self._gsparams)
        self._absorb(obj, jac is None)
        if np.any(np.asarray(self._det) == 0.):
            raise GalSimError("Attempt to Transform with degenerate matrix")

    def _absorb(self, obj, jac_is_none):
        if isinstance(obj, Transformation):
            if np.any(obj._has_offset):
                if jac_is_none:
                    dx1, dy1 = obj._dx, obj._dy
                else:
                    dx1, dy1 = self._fwd_normal(obj._dx, obj._dy)
                self._dx = self._dx + dx1
                self._dy = self._dy + dy1
            if jac_is_none:
                self._jac = obj._jac
            else:
                self._jac = self._jac if obj._jac is None else np.matmul(self._jac, obj._jac)
            self._flux_ratio = self._flux_ratio * obj._flux_ratio
            self._original = obj._original
        else:
            self._original = obj
        self._has_offset = (np.asarray(self._dx) != 0.) | (np.asarray(self._dy) != 0.)
        jb = 1 if self._jac is None or self._jac.ndim == 2 else self._jac.shape[0]
        self._batch = _plen(np.zeros(jb) if jb > 1 else 0., self._dx, self._dy, self._flux_ratio,
                            np.zeros(self._original._batch) if self._original._batch > 1 else 0.)

    original = property(lambda self: self._original)
    flux_ratio = property(lambda self: self._flux_ratio)

    @property
    def jac(self):
        return np.array([[1., 0.], [0., 1.]]) if self._jac is None else self._jac

    @property
    def offset(self):
        return PositionD(self._dx, self._dy) if np.ndim(self._dx) == 0 else (self._dx, self._dy)

    @property
    def _det(self):
        """transform.py:361-372."""
        j = self._jac
        if j is None:
            return 1.
        d = j[..., 0, 0] * j[..., 1, 1] - j[..., 0, 1] * j[..., 1, 0]
        diag = (j[..., 0, 1] == 0.) & (j[..., 1, 0] == 0.)
        d = np.where(diag, j[..., 0, 0] * j[..., 1, 1], d)
        return float(d) if np.ndim(d) == 0 else d

    @property
    def _flux_scaling(self):
        return np.abs(self._det) * self._flux_ratio

    @property
    def flux(self):
        return self._flux_scaling * self._original.flux

    @property
    def _has_hard_edges(self):
        return self._original.has_hard_edges

    @property
    def _is_analytic_x(self):
        return self._original.is_analytic_x

    @property
    def _is_axisymmetric(self):
        j = self._jac
        return bool(self._original.is_axisymmetric and
                    (j is None or (np.all(j[..., 0, 0] == j[..., 1, 1]) and
                                   np.all(j[..., 0, 1] == -j[..., 1, 0]))) and
                    not np.any(self._has_offset))

    def _fwd_normal(self, x, y):
        j = self._jac
        return j[..., 0, 0] * x + j[..., 0, 1] * y, j[..., 1, 0] * x + j[..., 1, 1] * y

    def _major_minor(self):
        """transform.py:496-505."""
        if self._jac is None:
            return 1., 1.
        j = self._jac
        h1 = np.hypot(j[..., 0, 0] + j[..., 1, 1], j[..., 0, 1] - j[..., 1, 0])
        h2 = np.hypot(j[..., 0, 0] - j[..., 1, 1], j[..., 0, 1] + j[..., 1, 0])
        return 0.5 * np.abs(h1 + h2), 0.5 * np.abs(h1 - h2)

    def withGSParams(self, gsparams=None, **kwargs):
        if gsparams == self.gsparams and not kwargs:
            return self
        import copy
        ret = copy.copy(self)
        ret._gsparams = GSParams.check(gsparams, self.gsparams, **kwargs)
        ret.__dict__.pop('_cached_sizes', None)
        if self._propagate_gsparams:
            ret._original = self._original.withGSParams(ret._gsparams)
        return ret

    def _flatten(self, bld, jac):
        jac_b = None if jac is None else np.asarray(jac)
        jac1 = _compose(jac_b, self._jac)
        self._original._flatten(bld, jac1)
        fs = np.asarray(self._flux_scaling, dtype=np.float64)
        kacc = self._gsparams.kvalue_accuracy
        scale_needed = np.abs(fs - 1.) > kacc
        if np.any(self._has_offset):
            fs_eff = np.where(self._has_offset | scale_needed, fs, 1.)
            bld.add_phase(jac_b, self._dx, self._dy, fs_eff)
        elif np.any(scale_needed):
            bld.add_scale(np.where(scale_needed, fs, 1.))

    def _size(self, prog, it):
        stepk, maxk = self._original._size(prog, it)
        major, minor = self._major_minor()
        stepk = stepk / major
        if np.any(self._has_offset):
            dr = np.hypot(self._dx, self._dy)
            stepk = np.where(self._has_offset, math.pi / (math.pi / stepk + dr), stepk)
        return stepk, maxk / minor

    def __eq__(self, other):
        return self is other or (isinstance(other, Transformation) and
                                 self.original == other.original and
                                 np.array_equal(self.jac, other.jac) and
                                 np.array_equal(self._dx, other._dx) and
                                 np.array_equal(self._dy, other._dy) and
                                 np.array_equal(self.flux_ratio, other.flux_ratio) and
                                 self.gsparams == other.gsparams)

    def __hash__(self):
        return hash(("galsim.Transformation", self.original, str(self.jac), str(self._dx),
                     str(self._dy), str(self.flux_ratio), self.gsparams))

    def __repr__(self):
        return 'galsim.Transformation(%r, jac=%r, offset=(%r, %r), flux_ratio=%r, gsparams=%r)' % (
            self.original, None if self._jac is None else self._jac.tolist(), self._dx, self._dy,
            self.flux_ratio, self.gsparams)


def _Transform(obj, jac=None, offset=(0., 0.), flux_ratio=1.):
    """Transform without gsparams handling (transform.py:606-643)."""
    ret = Transformation.__new__(Transformation)
    ret._gsparams = obj.gsparams
    ret._propagate_gsparams = True
    ret._jac = _as_jac(jac)
    ret._dx = _as_param(offset[0])
    ret._dy = _as_param(offset[1])
    ret._flux_ratio = _as_param(flux_ratio)
    ret._absorb(obj, jac is None)
    return ret


__all__ = ['Convolve', 'Convolution', 'Add', 'Sum', 'Transform', 'Transformation', '_Transform']

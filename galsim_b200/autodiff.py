"""Differentiable FFT drawing: the adjoint kernels (gsb_adjoint_images) behind torch.autograd.

GalSim itself has no derivatives; this module adds them for the FFT drawing path.  The
gradient of a loss with respect to the drawn stamps is pushed back through the forward-sign
FFTs, the Hermitian wrap, the k-space program and each profile's analytic dkValue/dparameter
by one fused kernel per FFT-size bucket.  Derivatives are taken on each stamp's fixed grid
(N, Nk, dk): the sizing rules are piecewise constant in the parameters.

Two levels:

* draw_records(plan, ...) -- a torch.autograd.Function over the numeric records of any
  flattened profile tree (leaf flux, Jacobian, size, Sersic index; phase centre, flux scaling,
  Jacobian; scale factors).  RecordPlan flattens a batched GSObject drawn into fixed-size
  stamps (drawImage's world-to-image transform, pixel and centring included).
* GalaxyModel -- a galaxy model Convolve(Sersic(n, hlr, flux).shear(g1, g2).shift(dx, dy), psf)
  whose seven parameters per stamp are a (B, 7) tensor; the chain from those parameters to
  the records (shear matrix, centroid) is ordinary torch code.
"""
import numpy as np

from . import _lib
from .errors import GalSimError, GalSimValueError

# p index of each leaf type's size parameter (Box: width, height = p[0], p[1])
# (InterpolatedImage leaves have no size record: their p holds the interpolant codes, and
# the adjoint gives them no gradient entries.)
_SIZE_INDEX = {_lib.GAUSSIAN: 0, _lib.EXPONENTIAL: 0, _lib.SERSIC: 1, _lib.MOFFAT: 1,
               _lib.KOLMOGOROV: 0, _lib.AIRY: 0, _lib.BOX: 0, _lib.INTERPOLATED: None}

RECORD_FIELDS = ('leaf_flux', 'leaf_jac', 'leaf_size', 'leaf_n', 'phase_cen', 'phase_fs',
                 'phase_jac', 'scales')


class RecordPlan(object):
    """A batched GSObject flattened for fixed-size stamps (nx x ny, pixel scale `scale`), whose
    numeric records can be replaced from tensors before each draw."""

    def __init__(self, obj, nx, ny, scale, dtype=np.float32, precision='fp32', offset=None,
                 use_true_center=True, tables=None):
        from .batch import plan_batch
        if nx is None or ny is None:
            raise GalSimValueError("differentiable drawing needs fixed stamp sizes nx, ny", (nx, ny))
        self.batch_plan = plan_batch(obj, nx, ny, scale, dtype, offset=offset,
                                     use_true_center=use_true_center, precision=precision,
                                     tables=tables)
        self.prog = self.batch_plan.prog
        for l, t in enumerate(self.prog.bld.leaf_types):
            if t == _lib.MOFFAT and np.any(self.prog.bld.leaves[l]['p'][:, 2] > 0.):
                # its table depends on trunc / scale_radius, so the size derivative at fixed
                # trunc is not the derivative at a fixed table that the adjoint computes
                from .errors import GalSimNotImplementedError
                raise GalSimNotImplementedError("gradients of truncated Moffat profiles are not built")
        self.prog.need_dn = True
        self.B = self.prog.B
        self.L = self.prog.L
        self.P = len(self.prog.bld.phases)
        self.S = len(self.prog.bld.scales)
        self.types = list(self.prog.bld.leaf_types)
        self.dtype = np.dtype(dtype)
        self.precision = _lib.F64 if precision == 'fp64' else _lib.F32
        self.nx, self.ny = int(nx), int(ny)
        self.last = None
        self._rec_dev = {}
        # records whose gradients the adjoint computes (leaf l: bit l, phase p: bit 8 + p,
        # scale q: bit 16 + q); the others get zero gradients
        self.want = _lib.WANT_ALL

    # -- records <-> tensors ----------------------------------------------------------------
    def records(self):
        """The current records as FP64 device tensors (detached)."""
        import torch
        dev = _lib.Device.torch_device()
        B, L, P, S = self.B, self.L, self.P, self.S
        bld = self.prog.bld
        lv = np.stack(bld.leaves, axis=1) if L else np.zeros((B, 0), _lib.LEAF_DTYPE)
        size = np.zeros((B, L, 2))
        nval = np.zeros((B, L))
        for l, t in enumerate(self.types):
            i = _SIZE_INDEX[t]
            if i is None:
                continue
            size[:, l, 0] = lv['p'][:, l, i]
            if t == _lib.BOX:
                size[:, l, 1] = lv['p'][:, l, 1]
            if t == _lib.SERSIC:
                nval[:, l] = lv['p'][:, l, 0]
        out = dict(leaf_flux=lv['flux'], leaf_jac=lv['jac'].reshape(B, L, 4), leaf_size=size,
                   leaf_n=nval)
        if P:
            ph = np.stack(bld.phases, axis=1)
            out['phase_cen'] = np.stack([ph['cenx'], ph['ceny']], axis=-1)
            out['phase_fs'] = ph['flux_scaling']
            out['phase_jac'] = ph['jac'].reshape(B, P, 4)
        else:
            out['phase_cen'] = np.zeros((B, 0, 2))
            out['phase_fs'] = np.zeros((B, 0))
            out['phase_jac'] = np.zeros((B, 0, 4))
        out['scales'] = np.stack(bld.scales, axis=1) if S else np.zeros((B, 0))
        # one host-to-device copy for all fields
        flat = np.concatenate([np.ascontiguousarray(out[k], dtype=np.float64).ravel() for k in RECORD_FIELDS])
        dflat = torch.as_tensor(flat, device=dev)
        res, o = {}, 0
        for k in RECORD_FIELDS:
            n = out[k].size
            res[k] = dflat[o:o + n].view(out[k].shape)
            o += n
        return res

    def set_records(self, rec):
        """Write record tensors (any subset of RECORD_FIELDS) into the host records."""
        import torch
        bld = self.prog.bld
        keys = [k for k in RECORD_FIELDS if k in rec]
        vals = [rec[k].detach().to(torch.float64) for k in keys]
        self._rec_dev = {k: v for k, v in zip(keys, vals)}
        flat = torch.cat([v.reshape(-1) for v in vals]).cpu().numpy() if vals else np.zeros(0)
        host, o = {}, 0
        for k, v in zip(keys, vals):
            n = v.numel()
            host[k] = flat[o:o + n].reshape(tuple(v.shape))
            o += n
        for l, t in enumerate(self.types):
            r = bld.leaves[l]
            if 'leaf_flux' in host:
                r['flux'] = host['leaf_flux'][:, l]
            if 'leaf_jac' in host:
                j = host['leaf_jac'][:, l]
                r['jac'] = j
                general = (j[:, 1] != 0.) | (j[:, 2] != 0.)
                r['flags'] = (r['flags'] & ~_lib.LEAF_JAC_GENERAL) | np.where(general, _lib.LEAF_JAC_GENERAL, 0)
            if 'leaf_size' in host and _SIZE_INDEX[t] is not None:
                r['p'][:, _SIZE_INDEX[t]] = host['leaf_size'][:, l, 0]
                if t == _lib.BOX:
                    r['p'][:, 1] = host['leaf_size'][:, l, 1]
            if 'leaf_n' in host and t == _lib.SERSIC:
                r['p'][:, 0] = host['leaf_n'][:, l]
        for i in range(self.P):
            r = bld.phases[i]
            if 'phase_cen' in host:
                r['cenx'] = host['phase_cen'][:, i, 0]
                r['ceny'] = host['phase_cen'][:, i, 1]
            if 'phase_fs' in host:
                r['flux_scaling'] = host['phase_fs'][:, i]
            if 'phase_jac' in host:
                r['jac'] = host['phase_jac'][:, i]
        if 'scales' in host:
            for i in range(self.S):
                bld.scales[i] = np.ascontiguousarray(host['scales'][:, i])
        self.prog.reset_records()

    # -- forward / adjoint -------------------------------------------------------------------
    def draw(self):
        """Size and draw every stamp; returns the (B, ny, nx) device tensor."""
        from .batch import run_batch
        sb = run_batch(self.batch_plan)
        self.last = sb
        self.draw_count = getattr(self, 'draw_count', 0) + 1
        t = self.prog.tables
        self._tables_gen = (t, t.generation) if t is not None else None
        return sb.stack()

    def adjoint(self, cot):
        """Record gradients (dict of FP64 device tensors) for the cotangent of the last draw."""
        import torch
        if self.last is None:
            raise GalSimError("RecordPlan.adjoint needs a preceding draw")
        B, L, P, S = self.B, self.L, self.P, self.S
        if self._tables_gen is not None and self._tables_gen[0].generation != self._tables_gen[1]:
            # a shared table set was rebuilt for another draw since ours: rebuild our slots
            # and prepare the leaves again (they hold the image slots' device addresses)
            self.prog.need_dn = True
            self.prog.compute_leaves()
            self._tables_gen = (self.prog.tables, self.prog.tables.generation)
        dt = _lib.F32 if self.dtype == np.float32 else _lib.F64
        tdt = torch.float32 if dt == _lib.F32 else torch.float64
        c = cot.to(dtype=tdt).contiguous().reshape(-1)
        g = self.prog.adjoint_stamps(c, dt, self.precision, self.want)
        gl = g[:, :_lib.GRAD_PER_LEAF * L].reshape(B, L, _lib.GRAD_PER_LEAF)
        gp = g[:, _lib.GRAD_PER_LEAF * L:_lib.GRAD_PER_LEAF * L + _lib.GRAD_PER_PHASE * P].reshape(
            B, P, _lib.GRAD_PER_PHASE)
        gs = g[:, _lib.GRAD_PER_LEAF * L + _lib.GRAD_PER_PHASE * P:]
        rec = self._rec_dev if all(k in self._rec_dev for k in ('leaf_jac', 'leaf_size')) else self.records()
        jac = rec['leaf_jac']
        gjac = gl[..., 1:5]
        size = rec['leaf_size']
        gsize = torch.zeros_like(size)
        for l, t in enumerate(self.types):
            if t == _lib.INTERPOLATED:
                continue
            if t == _lib.BOX:
                gsize[:, l, 0] = (jac[:, l, 0] * gjac[:, l, 0] + jac[:, l, 2] * gjac[:, l, 2]) / size[:, l, 0]
                gsize[:, l, 1] = (jac[:, l, 1] * gjac[:, l, 1] + jac[:, l, 3] * gjac[:, l, 3]) / size[:, l, 1]
            else:
                gsize[:, l, 0] = (jac[:, l] * gjac[:, l]).sum(-1) / size[:, l, 0]
        return dict(leaf_flux=gl[..., 0], leaf_jac=gjac, leaf_size=gsize, leaf_n=gl[..., 5],
                    phase_cen=gp[..., 0:2], phase_fs=gp[..., 2], phase_jac=gp[..., 3:7], scales=gs)


def _function():
    import torch

    class RecordDraw(torch.autograd.Function):
        """Images of a RecordPlan as a function of its record tensors."""

        @staticmethod
        def forward(ctx, plan, *tensors):
            plan.set_records(dict(zip(RECORD_FIELDS, tensors)))
            img = plan.draw()
            ctx.plan = plan
            ctx.dtypes = [t.dtype for t in tensors]
            ctx.records = [t.detach() for t in tensors]
            ctx.draw_id = plan.draw_count
            return img.clone()

        @staticmethod
        def backward(ctx, gout):
            plan = ctx.plan
            if plan.draw_count != ctx.draw_id:
                # the plan drew other records since this forward (a reused plan): draw this
                # forward's records again so that the adjoint sees its stamps and geometry
                plan.set_records(dict(zip(RECORD_FIELDS, ctx.records)))
                plan.draw()
            g = plan.adjoint(gout)
            return (None,) + tuple(g[k].to(dt) for k, dt in zip(RECORD_FIELDS, ctx.dtypes))

    return RecordDraw


_RecordDraw = None


def draw_records(plan, leaf_flux, leaf_jac, leaf_size, leaf_n, phase_cen, phase_fs, phase_jac,
                 scales):
    """Draw `plan` with the given records; differentiable with respect to every record tensor.
    Shapes: leaf_flux (B, L), leaf_jac (B, L, 4), leaf_size (B, L, 2), leaf_n (B, L),
    phase_cen (B, P, 2), phase_fs (B, P), phase_jac (B, P, 4), scales (B, S)."""
    global _RecordDraw
    if _RecordDraw is None:
        _RecordDraw = _function()
    return _RecordDraw.apply(plan, leaf_flux, leaf_jac, leaf_size, leaf_n, phase_cen, phase_fs,
                             phase_jac, scales)


def shear_matrix(g1, g2):
    """[[1+g1, g2], [g2, 1-g1]] / sqrt(1-g^2) (galsim/shear.py:365-386), batched, in torch."""
    import torch
    f = 1. / torch.sqrt(1. - (g1 * g1 + g2 * g2))
    return torch.stack([torch.stack([(1. + g1) * f, g2 * f], -1),
                        torch.stack([g2 * f, (1. - g1) * f], -1)], -2)


class GalaxyModel(object):
    """Differentiable batched drawImage(nx, ny, scale, method='fft') of
    Convolve(Sersic(n, half_light_radius=hlr, flux=flux).shear(g1=g1, g2=g2).shift(dx, dy), psf).

    Call with a (B, 7) tensor of (flux, hlr, n, g1, g2, dx, dy) per stamp (dx, dy in arcsec, i.e.
    world units of the pixel scale); returns the (B, ny, nx) stamps.  Gradients flow to all seven
    columns through the adjoint kernels."""

    PARAMS = ('flux', 'hlr', 'n', 'g1', 'g2', 'dx', 'dy')

    def __init__(self, psf, nx, ny, scale, dtype=np.float32, precision='fp32', gsparams=None):
        self.psf = psf
        self.nx, self.ny, self.scale = int(nx), int(ny), float(scale)
        self.dtype = dtype
        self.precision = precision
        self.gsparams = gsparams
        self.plan = None
        self.tables = None        # device Sersic tables, rebuilt in place on every call

    def build(self, p):
        """The batched GSObject for parameters p ((B, 7) numpy)."""
        from .compound import Convolve
        from .profiles import Sersic
        flux, hlr, n, g1, g2, dx, dy = [np.ascontiguousarray(c) for c in p.T]
        if not np.any((dx != 0.) | (dy != 0.)):
            # keep the shift in the program so that its gradient exists: a 1e-300 arcsec shift
            # has a phase factor of exactly 1
            dx = np.full_like(dx, 1e-300)
        gal = Sersic(n=n, half_light_radius=hlr, flux=flux, gsparams=self.gsparams)
        return Convolve(gal.shear(g1=g1, g2=g2).shift(dx, dy), self.psf)

    def __call__(self, params):
        import torch
        B = int(params.shape[0])
        if self.plan is None or self.plan.B != B:
            # The program's layout (galaxy leaf, its shift, the PSF's leaves) depends only on the
            # batch size: built once, then every call overwrites the galaxy's records.
            p = params.detach().to('cpu', torch.float64).numpy()
            if self.tables is None:
                self.tables = _lib.Tables()
            plan = RecordPlan(self.build(p), self.nx, self.ny, self.scale, self.dtype, self.precision,
                              tables=self.tables)
            if plan.types[0] != _lib.SERSIC or plan.P < 1:
                raise GalSimError("unexpected program layout for GalaxyModel")
            plan.want = 1 | (1 << 8)          # the galaxy leaf and its shift
            rec = plan.records()
            g1, g2 = torch.as_tensor(p[:, 3], device=rec['leaf_jac'].device), \
                torch.as_tensor(p[:, 4], device=rec['leaf_jac'].device)
            S = shear_matrix(g1, g2)
            # the galaxy leaf's Jacobian without its shear: the world-to-image transform
            self._jpre = rec['leaf_jac'][:, 0].reshape(B, 2, 2) @ torch.linalg.inv(S)
            self._rec0 = rec
            self.plan = plan
        plan, rec = self.plan, self._rec0
        pr = params.to(torch.float64)
        flux, hlr, n, g1, g2, dx, dy = pr.unbind(-1)
        S = shear_matrix(g1, g2)
        leaf_flux = rec['leaf_flux'].clone()
        leaf_flux[:, 0] = flux
        leaf_jac = rec['leaf_jac'].clone()
        leaf_jac[:, 0] = (self._jpre @ S).reshape(B, 4)
        leaf_size = rec['leaf_size'].clone()
        leaf_size[:, 0, 0] = hlr
        leaf_n = rec['leaf_n'].clone()
        leaf_n[:, 0] = n
        phase_cen = rec['phase_cen'].clone()
        phase_cen[:, 0] = torch.stack([dx, dy], -1)     # the program keeps its shift op (see build)
        phase_fs = rec['phase_fs'].clone()
        phase_fs[:, 0] = torch.abs(torch.linalg.det(S))
        return draw_records(plan, leaf_flux, leaf_jac, leaf_size, leaf_n, phase_cen, phase_fs,
                            rec['phase_jac'], rec['scales'])


__all__ = ['RecordPlan', 'draw_records', 'shear_matrix', 'GalaxyModel', 'RECORD_FIELDS']

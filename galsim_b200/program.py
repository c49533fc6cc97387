"""Flattening of GSObject trees into device programs, GalSim-exact FFT sizing, and the calls
into libgsb that draw them.

A *program* is the profile tree of every stamp of a batch written as a postfix op list
(LEAF / MUL / ADD / PHASE / SCALE, see include/gsb.h) plus per-stamp numeric records.  All
stamps of a batch share the topology; parameters may differ per stamp.  This replaces the
reference's Python tree walk of _drawKImage (convolve.py:420-426, sum.py:341-347,
transform.py:592-602), which issues one C++ call per leaf and one numpy pass per node.

Sizing (stepk / maxk -> N, Nk) follows the reference exactly: the leaf stepK()/maxK() values
are computed in FP64 on the GPU (gsb_prepare_leaves), and the composition rules
(convolve.py:296-305, sum.py:243-251, transform.py:490-516) and the integer sizing of
drawFFT_makeKImage (gsobject.py:1900-1963) run here in vectorised FP64 numpy, in the same
order of operations as the reference's Python.
"""
import ctypes
import math

import numpy as np

from . import _lib
from .errors import GalSimError, galsim_warn_fft


def unique_pairs(a, b):
    """np.unique of the rows (a_i, b_i) with return_inverse (lexicographic order), through a
    complex key: numpy's row-wise unique (axis=0) is ~10x slower on thousands of rows."""
    u, inv = np.unique(np.asarray(a, np.float64) + 1j * np.asarray(b, np.float64), return_inverse=True)
    return u.real.copy(), u.imag.copy(), np.asarray(inv).reshape(-1)


def stack_records(recs):
    """np.stack(recs, axis=1) of equal-length 1-d structured record arrays, copied as raw
    bytes (numpy's structured stack copies record by record)."""
    B = len(recs[0])
    dt = recs[0].dtype
    raw = np.stack([np.ascontiguousarray(r).view(np.uint8).reshape(B, dt.itemsize) for r in recs], axis=1)
    return raw.view(dt).reshape(B, len(recs))


class Builder(object):
    def __init__(self, B, gsparams):
        self.B = B
        self.gsparams = gsparams
        self.ops = []
        self.leaf_types = []
        self.leaves = []
        self.phases = []
        self.scales = []
        self.image_sources = {}   # InterpolatedImage leaf -> its _ImageSource list (1 or B)
        self.image_kinterp = {}   # InterpolatedImage leaf -> its Lanczos k interpolant (or None)

    def _bcast(self, v):
        a = np.asarray(v, dtype=np.float64)
        return np.broadcast_to(a, (self.B,)) if a.ndim == 0 else a.reshape(self.B)

    def _bjac(self, jac):
        if jac is None:
            return None
        j = np.asarray(jac, dtype=np.float64)
        return np.broadcast_to(j, (self.B, 2, 2))

    def add_leaf(self, ltype, jac, flux, params, flags=0):
        if len(self.leaves) >= _lib.MAX_LEAVES:
            raise GalSimError("profile tree has more than %d leaves" % _lib.MAX_LEAVES)
        # the record as 17 float64 words (jac 0-3, flux 4, p 5-7, d 8-15, flags / table in 16),
        # filled column by column with broadcasting, then viewed as LEAF_DTYPE
        B = self.B
        w = np.empty((B, 17), dtype=np.float64)
        iw = w.view(np.int32)                      # (B, 34): flags at 32, table at 33
        if jac is None:
            w[:, 0:4] = (1., 0., 0., 1.)
            general = 0
        else:
            j = np.asarray(jac, dtype=np.float64)
            if j.ndim == 2:
                w[:, 0:4] = j.reshape(4)
                general = _lib.LEAF_JAC_GENERAL if (j[0, 1] != 0. or j[1, 0] != 0.) else 0
            else:
                j = j.reshape(B, 4)
                w[:, 0:4] = j
                general = np.where((j[:, 1] != 0.) | (j[:, 2] != 0.), _lib.LEAF_JAC_GENERAL, 0)
        w[:, 4] = flux
        w[:, 5:8] = 0.
        for i, p in enumerate(params):
            w[:, 5 + i] = np.asarray(p, dtype=np.float64).reshape(-1) if np.ndim(p) else p
        w[:, 8:16] = 0.
        iw[:, 32] = np.bitwise_or(general, flags)
        iw[:, 33] = 0
        rec = w.view(_lib.LEAF_DTYPE).reshape(B)
        self.ops.append((_lib.OP_LEAF, len(self.leaves)))
        self.leaf_types.append(ltype)
        self.leaves.append(rec)

    def add_op(self, code):
        self.ops.append((code, 0))

    def add_phase(self, jac, cx, cy, fs):
        if len(self.phases) >= _lib.MAX_PHASES:
            raise GalSimError("profile tree has more than %d shifted transformations" % _lib.MAX_PHASES)
        rec = np.zeros(self.B, dtype=_lib.PHASE_DTYPE)
        j = self._bjac(jac)
        rec['jac'] = (1., 0., 0., 1.) if j is None else j.reshape(self.B, 4)
        rec['cenx'] = self._bcast(cx)
        rec['ceny'] = self._bcast(cy)
        rec['flux_scaling'] = self._bcast(fs)
        self.ops.append((_lib.OP_PHASE, len(self.phases)))
        self.phases.append(rec)

    def add_scale(self, s):
        if len(self.scales) >= _lib.MAX_SCALES:
            raise GalSimError("profile tree has more than %d flux scalings" % _lib.MAX_SCALES)
        self.ops.append((_lib.OP_SCALE, len(self.scales)))
        self.scales.append(self._bcast(s))

    def template(self):
        if len(self.ops) > _lib.MAX_OPS:
            raise GalSimError("profile tree needs more than %d program ops" % _lib.MAX_OPS)
        t = _lib.TemplateC()
        t.n_ops = len(self.ops)
        t.n_leaves = len(self.leaves)
        t.n_phases = len(self.phases)
        t.n_scales = len(self.scales)
        for i, (c, a) in enumerate(self.ops):
            t.op_code[i] = c
            t.op_arg[i] = a
        for i, lt in enumerate(self.leaf_types):
            t.leaf_type[i] = lt
        return t


def batch_size(obj):
    return obj._batch


class Program(object):
    """A flattened batch of profile trees resident on the device, ready to size and draw."""

    def __init__(self, obj, gsparams=None, tables=None):
        self.obj = obj
        self.tables = tables      # a _lib.Tables to (re)build into; one is made when needed
        self.B = batch_size(obj)
        self.gsparams = gsparams if gsparams is not None else obj.gsparams
        bld = Builder(self.B, self.gsparams)
        obj._flatten(bld, None)
        self.bld = bld
        self.tpl = bld.template()
        self.L = len(bld.leaves)
        self.gsp_c = _lib.gsparams_c(self.gsparams)
        self._prepared = False
        self.need_dn = False      # build the Sersic d/dn tables (for the adjoint)

    # -- device preparation ------------------------------------------------------------------
    def upload(self):
        """Pack the leaf records, assign Sersic table slots and copy the leaves to the device."""
        if getattr(self, 'd_leaves', None) is not None:
            return
        import torch
        B, L = self.B, self.L
        leaves = stack_records(self.bld.leaves)               # (B, L)
        self.sersic_n = None
        self.sersic_trunc = None
        sersic = [l for l in range(L) if self.bld.leaf_types[l] == _lib.SERSIC]
        if sersic:
            # one table per distinct (n, trunc / r0); truncated leaves carry r0 in p[1]
            nvals = np.concatenate([leaves[:, l]['p'][:, 0] for l in sersic])
            tvals = np.concatenate([np.where(leaves[:, l]['p'][:, 2] > 0.,
                                             leaves[:, l]['p'][:, 2] / leaves[:, l]['p'][:, 1], 0.)
                                    for l in sersic])
            un, ut, inv = unique_pairs(nvals, tvals)
            self.sersic_n = np.ascontiguousarray(un)
            self.sersic_trunc = np.ascontiguousarray(ut) if np.any(ut > 0.) else None
            inv = np.asarray(inv).reshape(len(sersic), B)
            for k, l in enumerate(sersic):
                leaves['table'][:, l] = inv[k]
        self.moffat_beta = None
        self.moffat_trunc = None
        moffat = [l for l in range(L) if self.bld.leaf_types[l] == _lib.MOFFAT]
        if moffat:
            # one table per distinct (beta, trunc / rD) of the truncated Moffat leaves
            bvals = np.concatenate([leaves[:, l]['p'][:, 0] for l in moffat])
            tvals = np.concatenate([leaves[:, l]['p'][:, 2] / leaves[:, l]['p'][:, 1] for l in moffat])
            cut = tvals > 0.
            if np.any(cut):
                ub, ut, inv = unique_pairs(bvals[cut], tvals[cut])
                uniq = np.stack([ub, ut], -1)
                slot = np.full(len(bvals), -1, dtype=np.int32)
                slot[cut] = inv
                slot = slot.reshape(len(moffat), B)
                for k, l in enumerate(moffat):
                    leaves['table'][:, l] = slot[k]
                self.moffat_beta = np.ascontiguousarray(uniq[:, 0])
                self.moffat_trunc = np.ascontiguousarray(uniq[:, 1])
        self.image_order = []
        image_leaves = [l for l in range(L) if self.bld.leaf_types[l] == _lib.INTERPOLATED]
        if image_leaves:
            slot_of = {}
            for l in image_leaves:
                slots = []
                for src in self.bld.image_sources[l]:
                    if id(src) not in slot_of:
                        slot_of[id(src)] = len(self.image_order)
                        self.image_order.append(src)
                    slots.append(slot_of[id(src)])
                leaves['table'][:, l] = np.broadcast_to(np.array(slots, dtype=np.int32), (B,))
                ki = self.bld.image_kinterp.get(l)
                if ki is not None:
                    # the coefficient block's device address, as the bits of p[2]
                    addr = np.array([ki._table.kdevice().data_ptr()], dtype=np.uint64).view(np.float64)[0]
                    leaves['p'][:, l, 2] = addr
        self.d_leaves = _lib.to_device(leaves)
        self.d_info = torch.empty(B * L * 2, dtype=torch.float64, device=_lib.Device.torch_device())
        if self.sersic_n is None and not self.image_order and self.moffat_beta is None:
            self.tables = None
        elif getattr(self, 'tables', None) is None:
            self.tables = _lib.TablePool.acquire()
            self._pooled_tables = True

    def compute_leaves(self):
        """FP64 on the GPU: build the Sersic and truncated-Moffat FT tables, then every leaf's
        derived constants, stepk and maxk; copy stepk / maxk back for the host-side composition."""
        self.upload()
        B, L = self.B, self.L
        if self.tables is not None and self.sersic_n is not None:
            self.tables.build_sersic(self.sersic_n, self.gsparams, with_dn=self.need_dn,
                                     trunc_over_r0=self.sersic_trunc)
        if self.tables is not None and self.moffat_beta is not None:
            self.tables.build_moffat(self.moffat_beta, self.moffat_trunc, self.gsparams)
        if self.image_order:
            self._build_images()
        _lib.check(_lib.lib().gsb_prepare_leaves(
            ctypes.byref(self.tpl), B, ctypes.byref(self.gsp_c), _lib.ptr(self.d_leaves),
            self.tables.handle if self.tables else None, _lib.ptr(self.d_info), _lib.Device.stream()))
        info = self.d_info.cpu().numpy().reshape(B, L, 2)
        self.leaf_stepk = info[:, :, 0]
        self.leaf_maxk = info[:, :, 1]
        self._prepared = True

    def _build_images(self):
        """The k-images and size scans of the InterpolatedImage sources, on the GPU.  A table
        set that already holds the same sources (kept alive by it) for the same GSParams is
        not rebuilt."""
        import torch
        key = (tuple(id(src) for src in self.image_order), self.gsparams)
        if getattr(self.tables, '_image_key', None) == key:
            return
        offsets = np.cumsum([0] + [src.region.size for src in self.image_order])
        desc = np.array([src.desc(off) for src, off in zip(self.image_order, offsets[:-1])],
                        dtype=_lib.IMAGE_DESC_DTYPE)
        pix = np.concatenate([src.region.ravel() for src in self.image_order])
        d_pix = torch.from_numpy(pix).to(_lib.Device.torch_device())
        self.tables.build_images(desc, d_pix, self.gsparams)
        self.tables._image_key = key
        self.tables._image_sources = list(self.image_order)

    def prepare(self):
        if self._prepared:
            return
        self.upload()
        self.compute_leaves()

    def stepk_maxk(self):
        """Composite stepk / maxk per stamp, by the reference's composition rules."""
        self.prepare()
        it = iter(range(self.L))
        return self.obj._size(self, it)

    def leaf_size(self, l):
        return self.leaf_stepk[:, l], self.leaf_maxk[:, l]

    # -- drawing ---------------------------------------------------------------------------
    def __del__(self):
        # graphs hold the table pointers; drop them before the tables go back to the pool
        self._graph_state = None
        if getattr(self, '_pooled_tables', False):
            try:
                _lib.TablePool.release(self.tables)
            except Exception:      # interpreter shutdown
                pass
            self.tables = None

    def reset_records(self):
        """Forget the device copy and sizing after the host records (bld.leaves / phases /
        scales) were changed in place."""
        self.d_leaves = None
        self._prepared = False
        self._geom = None
        self._graph_state = None

    def _stamp_geometry(self, N, Nk, xmin, ymin, nx, ny):
        """Device stamp records sorted by FFT size, with the bucket boundaries; kept for the
        adjoint of the same draw."""
        import torch
        B, L = self.B, self.L
        dev = _lib.Device.torch_device()
        N = np.asarray(N, np.int64)
        order = np.argsort(N, kind='stable')
        nx = np.broadcast_to(np.asarray(nx, np.int64), (B,))
        ny = np.broadcast_to(np.asarray(ny, np.int64), (B,))
        sizes = nx * ny
        offsets = np.zeros(B, np.int64)
        offsets[1:] = np.cumsum(sizes)[:-1]
        stamps = np.zeros(B, dtype=_lib.STAMP_DTYPE)
        stamps['N'] = N
        stamps['Nk'] = Nk
        stamps['xmin'] = xmin
        stamps['ymin'] = ymin
        stamps['nx'] = nx
        stamps['ny'] = ny
        stamps['out_offset'] = offsets
        perm = torch.from_numpy(order).to(dev)
        lv = torch.empty(B * L * _lib.LEAF_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        _lib.permute_records(lv, self.d_leaves, perm)
        ph = (_lib.to_device(stack_records(self.bld.phases)[order]) if self.bld.phases else None)
        sc = (_lib.to_device(np.stack(self.bld.scales, axis=1)[order]) if self.bld.scales else None)
        st = _lib.to_device(stamps[order])
        Ns = N[order]
        bounds = np.flatnonzero(np.diff(Ns)) + 1
        starts = np.concatenate([[0], bounds]).astype(np.int64)
        ends = np.concatenate([bounds, [B]]).astype(np.int64)
        self._geom = dict(order=order, perm=perm, lv=lv, ph=ph, sc=sc, st=st, Ns=Ns, starts=starts,
                          ends=ends, offsets=offsets, total=int(sizes.sum()))
        return self._geom

    def _bucket_ptrs(self, g, s0):
        L, P, S = self.L, len(self.bld.phases), len(self.bld.scales)
        return (ctypes.c_void_p(g['lv'].data_ptr() + int(s0) * L * _lib.LEAF_DTYPE.itemsize),
                ctypes.c_void_p(g['ph'].data_ptr() + int(s0) * P * _lib.PHASE_DTYPE.itemsize) if P else None,
                ctypes.c_void_p(g['sc'].data_ptr() + int(s0) * S * 8) if S else None,
                ctypes.c_void_p(g['st'].data_ptr() + int(s0) * _lib.STAMP_DTYPE.itemsize))

    def _launch_buckets(self, g, out, flux, flux_sorted, works, dtype, add, precision):
        """Draw every FFT-size bucket of geometry g (one stream per bucket, largest N first: the
        few long-running stamps of the big-N buckets take their SMs first and overlap the large
        small-N buckets).  The workspaces are allocated by the caller on the current stream
        before the fork and outlive the join, so the caching allocator cannot hand them out
        while a bucket runs."""
        import torch
        lib = _lib.lib()
        dev = _lib.Device.torch_device()
        main = torch.cuda.current_stream(dev)
        streams = _lib.Device.side_streams(len(g['buckets']))
        for (s0, s1), (wbytes, work), st in zip(g['buckets'], works, streams):
            st.wait_stream(main)
            lvp, php, scp, stp = self._bucket_ptrs(g, s0)
            _lib.check(lib.gsb_draw_bucket(
                ctypes.byref(self.tpl), int(s1 - s0), ctypes.byref(self.gsp_c), lvp, php, scp, stp,
                self.tables.handle if self.tables else None, int(g['Ns'][s0]),
                _lib.ptr(out), dtype, add,
                ctypes.c_void_p(flux_sorted.data_ptr() + int(s0) * 8),
                precision, _lib.ptr(work), ctypes.c_size_t(wbytes), ctypes.c_void_p(st.cuda_stream)))
        for st in streams:
            main.wait_stream(st)
        _lib.permute_records(flux, flux_sorted, g['perm'], scatter=True)

    def _workspaces(self, g, precision):
        import torch
        lib = _lib.lib()
        dev = _lib.Device.torch_device()
        works = []
        for s0, s1 in g['buckets']:
            wbytes = int(lib.gsb_draw_workspace_size(int(g['Ns'][s0]), int(s1 - s0), precision))
            works.append((wbytes, torch.empty(max(wbytes, 8), dtype=torch.uint8, device=dev) if wbytes else None))
        return works

    def draw_stamps(self, N, Nk, xmin, ymin, nx, ny, dtype, add_to=None, precision=_lib.F32,
                    graph=False):
        """Run the fused kernels for every stamp.  Arrays are per stamp.  Returns the device
        output buffer (flat), per-stamp offsets and the device added-flux array.

        graph=True: the draw stage of a repeated geometry (same N, Nk, bounds, dtype and
        precision as the previous call) is captured once as a CUDA graph, on the second such
        call, and replayed from then on, with the current leaf / phase / scale records copied
        into its input buffers first.  The returned buffers are copies."""
        import torch
        self.prepare()
        B = self.B
        dev = _lib.Device.torch_device()
        tdt = torch.float32 if dtype == _lib.F32 else torch.float64
        key = None
        if graph and add_to is None:
            # the captured launches hold the table pointers: the same Sersic indices keep them
            key = tuple(np.asarray(v, np.int64).tobytes() for v in (N, Nk, xmin, ymin, nx, ny)) + \
                (dtype, precision, b'' if self.sersic_n is None else self.sersic_n.tobytes(),
                 b'' if self.sersic_trunc is None else self.sersic_trunc.tobytes(),
                 b'' if self.moffat_beta is None else self.moffat_beta.tobytes() + self.moffat_trunc.tobytes())
            gs = getattr(self, '_graph_state', None)
            if gs is not None and gs['key'] == key:
                g = gs['geom']
                # refresh the inputs in place (the records may have changed since)
                _lib.permute_records(g['lv'], self.d_leaves, g['perm'])
                if g['ph'] is not None:
                    g['ph'].copy_(_lib.to_device(stack_records(self.bld.phases)[g['order']]))
                if g['sc'] is not None:
                    g['sc'].copy_(_lib.to_device(np.stack(self.bld.scales, axis=1)[g['order']]))
                if gs['graph'] is None:
                    cg = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(cg, capture_error_mode='thread_local'):
                        self._launch_buckets(g, gs['out'], gs['flux'], gs['flux_sorted'], gs['works'],
                                             dtype, 0, precision)
                    gs['graph'] = cg
                gs['graph'].replay()
                self._geom = g
                return gs['out'].clone(), g['offsets'], gs['flux'].clone()
        g = self._stamp_geometry(N, Nk, xmin, ymin, nx, ny)
        g['buckets'] = sorted(zip(g['starts'], g['ends']), key=lambda se: -int(g['Ns'][se[0]]))
        out = add_to if add_to is not None else torch.empty(max(g['total'], 1), dtype=tdt, device=dev)
        flux = torch.empty(B, dtype=torch.float64, device=dev)
        flux_sorted = torch.empty(B, dtype=torch.float64, device=dev)
        works = self._workspaces(g, precision)
        self._launch_buckets(g, out, flux, flux_sorted, works, dtype, 1 if add_to is not None else 0, precision)
        if key is not None:
            self._graph_state = dict(key=key, geom=g, out=out, flux=flux, flux_sorted=flux_sorted,
                                     works=works, graph=None)
            return out.clone(), g['offsets'], flux.clone()
        return out, g['offsets'], flux

    def grad_count(self):
        return _lib.lib().gsb_adjoint_grad_count(ctypes.byref(self.tpl))

    def adjoint_stamps(self, cot, cot_dtype, precision=_lib.F32, want=_lib.WANT_ALL):
        """Reverse mode of the last draw_stamps call: cot is the flat device cotangent in the
        output's layout.  Returns the (B, grad_count) FP64 device tensor of record gradients
        (see gsb_adjoint_grad_count for the entry order); records outside the `want` bit mask
        (leaf l: bit l, phase p: bit 8 + p, scale q: bit 16 + q) get zeros."""
        import torch
        g = self._geom
        if g is None:
            raise GalSimError("adjoint_stamps needs a preceding draw_stamps")
        B = self.B
        dev = _lib.Device.torch_device()
        ng = self.grad_count()
        grad_sorted = torch.empty((B, ng), dtype=torch.float64, device=dev)
        stream = _lib.Device.stream()
        lib = _lib.lib()
        for s0, s1 in zip(g['starts'], g['ends']):
            n = int(s1 - s0)
            NN = int(g['Ns'][s0])
            wbytes = lib.gsb_adjoint_workspace_size(NN, n, precision)
            work = torch.empty(max(int(wbytes), 8), dtype=torch.uint8, device=dev) if wbytes else None
            lvp, php, scp, stp = self._bucket_ptrs(g, s0)
            _lib.check(lib.gsb_adjoint_images(
                ctypes.byref(self.tpl), n, ctypes.byref(self.gsp_c), lvp, php, scp, stp,
                self.tables.handle if self.tables else None, NN,
                _lib.ptr(cot), cot_dtype, ctypes.c_void_p(grad_sorted.data_ptr() + int(s0) * ng * 8),
                ctypes.c_uint(int(want) & 0xffffffff), precision, _lib.ptr(work),
                ctypes.c_size_t(int(wbytes)), stream))
        grad = torch.empty_like(grad_sorted)
        _lib.permute_records(grad, grad_sorted, g['perm'], scatter=True, stream=stream)
        return grad

    def draw_kimage(self, dk, kxmin, kymin, nkx, nky, dtype):
        """Evaluate the program on a k grid; returns a host complex array (B, nky, nkx)."""
        import torch
        self.prepare()
        dev = _lib.Device.torch_device()
        tdt = torch.float32 if dtype == _lib.F32 else torch.float64
        out = torch.empty(self.B * nkx * nky * 2, dtype=tdt, device=dev)
        ph = _lib.to_device(stack_records(self.bld.phases)) if self.bld.phases else None
        sc = _lib.to_device(np.stack(self.bld.scales, axis=1)) if self.bld.scales else None
        _lib.check(_lib.lib().gsb_draw_kimages(
            ctypes.byref(self.tpl), self.B, ctypes.byref(self.gsp_c), _lib.ptr(self.d_leaves),
            _lib.ptr(ph) if ph is not None else None, _lib.ptr(sc) if sc is not None else None,
            self.tables.handle if self.tables else None, float(dk), int(kxmin), int(kymin),
            int(nkx), int(nky), _lib.ptr(out), dtype, _lib.Device.stream()))
        a = out.cpu().numpy().reshape(self.B, nky, nkx, 2)
        cdt = np.complex64 if dtype == _lib.F32 else np.complex128
        return (a[..., 0] + 1j * a[..., 1]).astype(cdt)


# ---- GalSim-exact sizing helpers (gsobject.py:1900-1963) -------------------------------------
_GOOD_SIZES = np.array(sorted(set([2 ** a for a in range(1, 31)] + [3 * 2 ** a for a in range(1, 30)])),
                       dtype=np.float64)


def good_fft_size_array(n):
    """goodFFTSize (src/Image.cpp:1141-1153) vectorised: the smallest 2^a or 3*2^a (>= 6) that is
    >= (1 - 1e-5) n, and 2 for n <= 2."""
    n = np.asarray(n, np.int64)
    insize = (1. - 1.e-5) * n.astype(np.float64)
    idx = np.searchsorted(_GOOD_SIZES, insize, side='left')
    out = _GOOD_SIZES[np.minimum(idx, len(_GOOD_SIZES) - 1)].astype(np.int64)
    return np.where(n <= 2, 2, out)


def good_image_size(stepk, pixel_scale):
    """getGoodImageSize (gsobject.py:1900-1925), per stamp."""
    stepk = np.atleast_1d(np.asarray(stepk, np.float64))
    Nd = 2. * math.pi / (pixel_scale * stepk)
    N = np.ceil(Nd * (1. - 1.e-12)).astype(np.int64)
    return 2 * ((N + 1) // 2)


def fft_sizes(stepk, maxk, xmin, xmax, ymin, ymax, gsparams, scale=1.0):
    """(N, Nk) per stamp as in drawFFT_makeKImage (gsobject.py:1927-1963).  (xmin..ymax) are
    the bounds of each stamp's centred image view."""
    stepk = np.atleast_1d(np.asarray(stepk, np.float64))
    maxk = np.atleast_1d(np.asarray(maxk, np.float64))
    xmin, xmax, ymin, ymax = [np.broadcast_to(np.asarray(v, np.int64), stepk.shape)
                              for v in (xmin, xmax, ymin, ymax)]
    N = good_image_size(stepk, scale)
    absmax = np.max(np.abs(np.stack([xmin, xmax, ymin, ymax])), axis=0)
    image_N = np.maximum(absmax * 2, np.maximum(ymax - ymin + 1, xmax - xmin + 1))
    N = np.maximum(N, image_N)
    N = good_fft_size_array(N)
    N = np.maximum(N, gsparams.minimum_fft_size)
    dk = 2. * np.pi / (N * scale)
    Nk = np.where(N * dk / 2 > maxk, N, np.ceil(maxk / dk).astype(np.int64) * 2)
    big = Nk > gsparams.maximum_fft_size
    if np.any(big):
        galsim_warn_fft("drawFFT requires a very large FFT.", int(Nk[big].max()))
    return N.astype(np.int64), Nk.astype(np.int64)

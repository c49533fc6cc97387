"""Batched drawing: many stamps of one profile-tree topology in one set of kernel launches.

    >>> gal = galsim_b200.Sersic(n=n_arr, half_light_radius=hlr_arr, flux=flux_arr)
    >>> obj = galsim_b200.Convolve(gal.shear(g1=g1_arr, g2=g2_arr), psf)
    >>> stamps = galsim_b200.draw_batch(obj, scale=0.2, dtype=np.float32)

This is drawImage(method='fft') (gsobject.py:1283-1844) applied to every element of a
batched GSObject: each stamp gets the reference's world-to-image transform, pixel
convolution, automatic or fixed size, centring and flux bookkeeping; the FP64 sizing runs on
the GPU once for the whole batch and the stamps are drawn by FFT-size bucket.
"""
import numpy as np

from . import _lib
from .errors import GalSimIncompatibleValuesError, GalSimValueError
from .gsparams import GSParams
from .position import _PositionD


_PINNED = {}          # page-locked read-back buffers: host() pixels
_PINNED_FITS = {}     # and FITS file images
_PINNED_ASYNC = {}    # host_async: two alternating buffers per size
_COPY_STREAMS = {}


def _copy_stream(dev):
    import torch
    s = _COPY_STREAMS.get(dev.index)
    if s is None:
        s = torch.cuda.Stream(device=dev)
        _COPY_STREAMS[dev.index] = s
    return s


class HostRead(object):
    """A read of a StampBatch's pixels and drawn fluxes to the host in flight on a copy stream
    (StampBatch.host_async); result() waits for it and returns the flat host array,
    added_flux() the per-stamp fluxes."""

    def __init__(self, buf, fbuf, done, flux_scale):
        self._buf = buf
        self._fbuf = fbuf
        self._done = done
        self._flux_scale = flux_scale

    def done(self):
        return self._done.query()

    def result(self):
        self._done.synchronize()
        return self._buf.numpy()

    def added_flux(self):
        self._done.synchronize()
        return self._fbuf.numpy() / self._flux_scale


class StampBatch(object):
    """The drawn stamps: a flat device buffer plus per-stamp geometry.

    Attributes: ``flat`` (torch tensor on the device), ``offsets``, ``nx``, ``ny``, ``xmin``,
    ``ymin`` (numpy, per stamp, bounds relative to each stamp's centre), ``N``, ``Nk`` (FFT
    sizes), ``added_flux`` (numpy), ``dtype``."""

    def __init__(self, flat, offsets, nx, ny, xmin, ymin, N, Nk, flux_dev, dtype, scale, bounds,
                 flux_scale=1.):
        self.flat = flat
        self._flux_dev = flux_dev
        self._flux_scale = flux_scale
        self.offsets = offsets
        self.nx = nx
        self.ny = ny
        self.xmin = xmin
        self.ymin = ymin
        self.N = N
        self.Nk = Nk
        self.dtype = dtype
        self.scale = scale
        self.bounds = bounds

    @property
    def added_flux(self):
        """Per-stamp drawn flux / flux_scale (image.added_flux, gsobject.py:1840)."""
        return self._flux_dev.cpu().numpy() / self._flux_scale

    def __len__(self):
        return len(self.offsets)

    def addNoise(self, noise, seeds, skips=None):
        """Add noise to every stamp on the device, stamp i with its own stream
        BaseDeviate(seeds[i]) (positioned skips[i] raw draws in): the noise each stamp would get
        from ``image.addNoise(noise.copy(rng=galsim.BaseDeviate(seeds[i])))`` in the reference
        (noise.py:31-39), as its config layer seeds each object.  Returns the draws used per
        stamp (seeding included), to continue the streams."""
        return noise._apply_batch(self, seeds, skips)

    def array(self, i):
        """Stamp i as a host numpy array (ny, nx)."""
        n = int(self.nx[i] * self.ny[i])
        o = int(self.offsets[i])
        return self.flat[o:o + n].cpu().numpy().reshape(int(self.ny[i]), int(self.nx[i]))

    def host(self, copy=True):
        """All pixels as one flat host numpy array, read through page-locked memory (a buffer
        reused by calls of the same size).  copy=False returns a view of that buffer, valid
        until the next host() call of the same size."""
        import torch
        n = self.flat.numel()
        buf = _PINNED.get((n, self.flat.dtype))
        if buf is None:
            buf = torch.empty(n, dtype=self.flat.dtype, pin_memory=True)
            _PINNED.clear()
            _PINNED[(n, self.flat.dtype)] = buf
        buf.copy_(self.flat, non_blocking=True)
        torch.cuda.current_stream(self.flat.device).synchronize()
        return buf.numpy().copy() if copy else buf.numpy()

    def host_async(self):
        """Start reading all pixels and the drawn fluxes to the host on a copy stream, so that
        the read overlaps whatever is launched next on the drawing stream (the next batch's
        tables and draws) and the host need not wait for this batch's draws before preparing
        the next.  Returns a HostRead; its result() is a view of one of two page-locked buffers
        that alternate between calls of the same size, valid until the call after next."""
        import torch
        dev = self.flat.device
        key = (self.flat.numel(), self.flat.dtype, self._flux_dev.numel())
        slot = _PINNED_ASYNC.get(key)
        if slot is None:
            slot = [[(torch.empty(key[0], dtype=key[1], pin_memory=True),
                      torch.empty(key[2], dtype=self._flux_dev.dtype, pin_memory=True))
                     for _ in range(2)], 0]
            _PINNED_ASYNC.clear()
            _PINNED_ASYNC[key] = slot
        buf, fbuf = slot[0][slot[1]]
        slot[1] ^= 1
        cs = _copy_stream(dev)
        ready = torch.cuda.Event()
        ready.record(torch.cuda.current_stream(dev))
        cs.wait_event(ready)
        with torch.cuda.stream(cs):
            buf.copy_(self.flat, non_blocking=True)
            fbuf.copy_(self._flux_dev, non_blocking=True)
            done = torch.cuda.Event()
            done.record(cs)
        self.flat.record_stream(cs)
        self._flux_dev.record_stream(cs)
        return HostRead(buf, fbuf, done, self._flux_scale)

    def arrays(self):
        host = self.host()
        return [host[o:o + int(x * y)].reshape(int(y), int(x))
                for o, x, y in zip(self.offsets, self.nx, self.ny)]

    def stack(self):
        """All stamps as one (B, ny, nx) device tensor (they must share a size)."""
        if len(set(self.nx)) != 1 or len(set(self.ny)) != 1:
            raise GalSimValueError("stamps have different sizes", (set(self.nx), set(self.ny)))
        return self.flat[:len(self) * int(self.nx[0] * self.ny[0])].view(
            len(self), int(self.ny[0]), int(self.nx[0]))

    def fits_bytes(self, cube=False):
        """The FITS file image of every stamp, assembled on the device and read back once:
        one HDU per stamp (writeMulti; the first is the primary HDU) or one data cube
        (writeCube; the stamps must share a size).  Each header carries the stamp's BITPIX,
        NAXISn, GS_XMIN / GS_YMIN and its PixelScale WCS, as fits.py writes them."""
        return self._fits_image(cube).tobytes()

    def _fits_image(self, cube=False):
        """fits_bytes as a uint8 view of a reused page-locked buffer (valid until the next call
        of the same size)."""
        import ctypes
        import torch
        from . import fits
        from .bounds import _BoundsI
        from .wcs import PixelScale
        B = len(self)
        if B == 0:
            raise GalSimValueError("no stamps to write", B)
        dt = np.dtype(np.float32) if self.flat.dtype == torch.float32 else np.dtype(np.float64)
        esz = dt.itemsize
        wcs = PixelScale(self.scale)
        nx = np.asarray(self.nx, np.int64)
        ny = np.asarray(self.ny, np.int64)
        offsets = np.asarray(self.offsets, np.int64)
        bnd = np.asarray(self.bounds, np.int64).reshape(B, 4)
        hdrs = []

        def header(shape, primary, b):
            cls = fits.PrimaryHDU if primary else fits.ImageHDU
            hdu = cls(np.empty(shape, dt), fits.image_header_cards(_BoundsI(*(int(v) for v in b)), wcs))
            off = sum(len(h) for h in hdrs)
            hdrs.append(np.frombuffer(hdu.header_bytes(), np.uint8))
            return off, len(hdrs[-1])

        if cube:
            if np.any(nx != nx[0]) or np.any(ny != ny[0]):
                raise GalSimValueError("In writeCube: the stamps have different sizes",
                                       (sorted(set(nx.tolist())), sorted(set(ny.tolist()))))
            n1 = int(nx[0] * ny[0])
            if not np.array_equal(offsets, np.arange(B, dtype=np.int64) * n1):
                raise GalSimValueError("In writeCube: the stamps are not stored back to back", offsets)
            hs, hl = header((B, int(ny[0]), int(nx[0])), True, bnd[0])
            rec = np.zeros(1, dtype=_lib.FITS_HDU_DTYPE)
            rec['header_src'], rec['header_len'], rec['data_src'], rec['n_elem'] = hs, hl, offsets[0], B * n1
        else:
            # one extension header per distinct (shape, origin); the first stamp's as the primary
            keys = np.stack([ny, nx, bnd[:, 0], bnd[:, 2]], axis=1)
            uniq, inv = np.unique(keys, axis=0, return_inverse=True)
            inv = inv.reshape(-1)
            hsrc = np.zeros(len(uniq), np.int64)
            hlen = np.zeros(len(uniq), np.int64)
            for u, k in enumerate(uniq):
                b = (k[2], k[2] + k[1] - 1, k[3], k[3] + k[0] - 1)
                hsrc[u], hlen[u] = header((int(k[0]), int(k[1])), False, b)
            rec = np.zeros(B, dtype=_lib.FITS_HDU_DTYPE)
            rec['header_src'] = hsrc[inv]
            rec['header_len'] = hlen[inv]
            p0, l0 = header((int(ny[0]), int(nx[0])), True, bnd[0])
            rec['header_src'][0], rec['header_len'][0] = p0, l0
            rec['data_src'] = offsets
            rec['n_elem'] = nx * ny
        dbytes = (rec['n_elem'] * esz + fits.BLOCK - 1) // fits.BLOCK * fits.BLOCK
        sizes = rec['header_len'] + dbytes
        rec['dst'][1:] = np.cumsum(sizes)[:-1]
        total = int(sizes.sum())
        dev = self.flat.device
        d_hdr = torch.from_numpy(np.concatenate(hdrs)).to(dev)
        out = torch.empty(total, dtype=torch.uint8, device=dev)
        _lib.check(_lib.lib().gsb_fits_pack(
            rec.ctypes.data_as(ctypes.c_void_p), len(rec), _lib.ptr(d_hdr), d_hdr.numel(),
            _lib.ptr(self.flat), self.flat.numel(), _lib.F32 if esz == 4 else _lib.F64,
            _lib.ptr(out), total, _lib.Device.stream()))
        buf = _PINNED_FITS.get(total)
        if buf is None:
            buf = torch.empty(total, dtype=torch.uint8, pin_memory=True)
            _PINNED_FITS.clear()
            _PINNED_FITS[total] = buf
        buf.copy_(out, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        return buf.numpy()

    def writeMulti(self, file_name, dir=None, clobber=True, compression='auto'):
        """galsim.fits.writeMulti of every stamp (fits.py:445-527), the file image made on the
        device (fits_bytes)."""
        from . import fits
        file_compress, tile = fits._parse_compression(compression, file_name)
        fits._no_tiles(tile)
        fits._write_bytes(file_name, dir, self._fits_image(cube=False), clobber, file_compress)

    def writeCube(self, file_name, dir=None, clobber=True, compression='auto'):
        """galsim.fits.writeCube of the stamps (fits.py:529-648), made on the device."""
        from . import fits
        file_compress, tile = fits._parse_compression(compression, file_name)
        fits._no_tiles(tile)
        fits._write_bytes(file_name, dir, self._fits_image(cube=True), clobber, file_compress)

    def images(self):
        from .image import Image
        from .wcs import PixelScale
        out = []
        for i, a in enumerate(self.arrays()):
            b = self.bounds[i]
            im = Image(a, xmin=b[0], ymin=b[2], wcs=PixelScale(self.scale))
            im.added_flux = float(self.added_flux[i])
            out.append(im)
        return out


class BatchPlan(object):
    """A flattened batch ready to be drawn (see draw_batch)."""

    def __init__(self, prog, nx, ny, fixed, flux_scale, dtype, scale, precision):
        self.prog = prog
        self.nx = nx
        self.ny = ny
        self.fixed = fixed
        self.flux_scale = flux_scale
        self.dtype = dtype
        self.scale = scale
        self.precision = precision


def plan_batch(obj, nx=None, ny=None, scale=None, dtype=np.float32, method='fft', area=1.,
               exptime=1., gain=1., offset=None, use_true_center=True, precision='fp32',
               tables=None):
    """Host set-up of draw_batch: drawImage's argument handling and world-to-image transform
    (gsobject.py:1647-1764) applied to the batched object, flattened into a device program.
    `tables` (a galsim_b200._lib.Tables) is reused for the Sersic tables when given."""
    from . import box, compound
    from .compound import _Transform
    from .program import Program
    if method not in ('fft', 'auto', 'no_pixel', 'sb'):
        raise GalSimValueError("draw_batch supports the FFT path only", method,
                               ('fft', 'auto', 'no_pixel', 'sb'))
    if scale is None or not scale > 0:
        raise GalSimValueError("draw_batch needs a pixel scale > 0", scale)
    if (nx is None) != (ny is None):
        raise GalSimIncompatibleValuesError("Must set either both or neither of nx, ny", nx=nx, ny=ny)
    B = obj._batch
    flux_scale = area * exptime
    if method == 'sb':
        flux_scale /= scale ** 2
    if gain != 1:
        flux_scale /= gain
    off = np.zeros((B, 2)) if offset is None else np.broadcast_to(np.asarray(offset, float), (B, 2))
    off = off.copy()
    if use_true_center:
        # _adjust_offset (gsobject.py:1234-1253); automatically sized images are even.
        if nx is None or nx % 2 == 0:
            off[:, 0] -= 0.5
        if ny is None or ny % 2 == 0:
            off[:, 1] -= 0.5
    inv = 1. / scale
    jac = None if scale == 1. else np.array(((inv, 0.), (0., inv)))
    prof = _Transform(obj, jac, flux_ratio=scale ** 2 * flux_scale, offset=(off[:, 0], off[:, 1]))
    if method in ('fft', 'auto'):
        prof = compound.Convolve(prof, box.Pixel(scale=1.0, gsparams=obj.gsparams),
                                 real_space=False, gsparams=obj.gsparams)
    prog = Program(prof, tables=tables)
    prog.upload()
    plan = BatchPlan(prog, nx, ny, nx is not None, flux_scale, dtype, scale, precision)
    # 'no_pixel' / 'sb' on a profile analytic in real space is drawn in real space, as
    # drawImage does (gsobject.py:1810-1811)
    plan.real = method in ('no_pixel', 'sb') and prof.is_analytic_x
    plan.prof = prof
    return plan


def run_batch(plan, recompute=True, graph=True):
    """Device part of draw_batch: FP64 tables and leaf sizing, GalSim sizing on the host, and
    the fused draw kernels.  recompute=False reuses the leaf sizing of an earlier run.
    graph=True: when the plan is run again with the same stamp geometry, its draw stage is
    captured as one CUDA graph (on the second run) and replayed (see Program.draw_stamps)."""
    from .program import fft_sizes, good_image_size
    prog = plan.prog
    B = prog.B
    if getattr(plan, 'real', False):
        return _run_real(plan)
    if recompute or not prog._prepared:
        prog.compute_leaves()
    stepk, maxk = prog.stepk_maxk()
    if plan.fixed:
        nxs = np.full(B, int(plan.nx), np.int64)
        nys = np.full(B, int(plan.ny), np.int64)
    else:
        nxs = good_image_size(stepk, 1.0)
        nys = nxs.copy()
    # Image bounds (1..nx, 1..ny) shifted so that the centre is (0, 0)
    xmin = -(nxs // 2)
    ymin = -(nys // 2)
    N, Nk = fft_sizes(stepk, maxk, xmin, xmin + nxs - 1, ymin, ymin + nys - 1, prog.gsparams)
    dt = _lib.F32 if np.dtype(plan.dtype) == np.float32 else _lib.F64
    prec = _lib.F64 if plan.precision == 'fp64' else _lib.F32
    flat, offsets, flux = prog.draw_stamps(N, Nk, xmin, ymin, nxs, nys, dt, precision=prec, graph=graph)
    bounds = [(1, int(x), 1, int(y)) for x, y in zip(nxs, nys)]
    return StampBatch(flat, offsets, nxs, nys, xmin, ymin, N, Nk, flux, plan.dtype, plan.scale,
                      bounds, plan.flux_scale)


def _run_real(plan):
    """run_batch for a real-space plan: GalSim's automatic image size where needed (from the
    FP64 stepk), then one gsb_draw_real over all stamps."""
    from .program import good_image_size
    from .realspace import draw_real_stamps
    prog = plan.prog
    B = prog.B
    if plan.fixed:
        nxs = np.full(B, int(plan.nx), np.int64)
        nys = np.full(B, int(plan.ny), np.int64)
    else:
        prog.compute_leaves()
        stepk, _ = prog.stepk_maxk()
        nxs = good_image_size(stepk, 1.0)
        nys = nxs.copy()
    xmin = -(nxs // 2)
    ymin = -(nys // 2)
    flat, offsets, flux = draw_real_stamps(plan.prof, B, prog.gsparams, xmin, ymin, nxs, nys, plan.dtype)
    bounds = [(1, int(x), 1, int(y)) for x, y in zip(nxs, nys)]
    zero = np.zeros(B, np.int64)
    return StampBatch(flat, offsets, nxs, nys, xmin, ymin, zero, zero, flux, plan.dtype, plan.scale,
                      bounds, plan.flux_scale)


def draw_batch(obj, nx=None, ny=None, scale=None, dtype=np.float32, method='fft', area=1.,
               exptime=1., gain=1., offset=None, use_true_center=True, precision='fp32',
               bandpass=None, integrator='quadratic'):
    """Draw every stamp of a batched GSObject.

    Each stamp is drawn like ``obj_i.drawImage(nx=nx, ny=ny, scale=scale, dtype=dtype,
    method=method, ...)``; without nx, ny every stamp gets its automatic size
    (getGoodImageSize).  ``offset`` may be a (B, 2) array.  Returns a StampBatch whose pixels
    stay on the device until read.

    A chromatic object (a batched GSObject times an SED, convolved with chromatic or achromatic
    PSFs, and sums of such terms) is drawn through ``bandpass`` like
    ``obj_i.drawImage(bandpass, nx=nx, ny=ny, ...)``; fixed nx, ny are then required, and each
    term's effective PSF is integrated once for the whole batch (see
    galsim_b200.chromatic.draw_batch_chromatic)."""
    from .chromatic import ChromaticObject, draw_batch_chromatic
    if isinstance(obj, (list, tuple)):
        obj = stack_objects(obj)
    if isinstance(obj, ChromaticObject):
        if bandpass is None:
            raise GalSimIncompatibleValuesError("a chromatic object is drawn through a bandpass",
                                                bandpass=bandpass)
        return draw_batch_chromatic(obj, bandpass, nx, ny, scale, dtype, method, area, exptime, gain,
                                    offset, use_true_center, precision, integrator)
    return run_batch(plan_batch(obj, nx, ny, scale, dtype, method, area, exptime, gain, offset,
                                use_true_center, precision))


def draw_batches(objects, nx=None, ny=None, scale=None, dtype=np.float32, method='fft', area=1.,
                 exptime=1., gain=1., offset=None, use_true_center=True, precision='fp32'):
    """Draw a sequence of batched GSObjects (a catalog in chunks), yielding per batch
    ``(stamps, pixels, fluxes)``: the StampBatch (its geometry; pixels still on the device),
    the flat host pixels and the per-stamp added fluxes.  Three stages overlap: a worker thread
    takes the next object from `objects` and builds and uploads its records (plan_batch) while
    the current batch's tables and draws run, and each batch's pixels are read back on a copy
    stream while the next batch draws.  The host arrays are views of page-locked buffers that
    alternate between batches of the same size: copy them to keep them past the next
    iteration.  The other arguments are draw_batch's."""
    from concurrent.futures import ThreadPoolExecutor
    it = iter(objects)
    kw = dict(nx=nx, ny=ny, scale=scale, dtype=dtype, method=method, area=area, exptime=exptime, gain=gain,
              offset=offset, use_true_center=use_true_center, precision=precision)
    import torch
    dev = _lib.Device.torch_device()

    def prepare():
        torch.cuda.set_device(dev)           # the worker thread's current device is its own
        try:
            obj = next(it)
        except StopIteration:
            return None
        if isinstance(obj, (list, tuple)):
            obj = stack_objects(obj)
        return plan_batch(obj, **kw)

    with ThreadPoolExecutor(max_workers=1) as pool:
        nxt = pool.submit(prepare)
        pending = None
        while True:
            plan = nxt.result()
            if plan is None:
                break
            nxt = pool.submit(prepare)          # the next batch's host set-up overlaps this one
            sb = run_batch(plan)
            read = sb.host_async()
            if pending is not None:
                psb, pread = pending
                yield psb, pread.result(), pread.added_flux()
            pending = (sb, read)
        if pending is not None:
            psb, pread = pending
            yield psb, pread.result(), pread.added_flux()


def stack_objects(objs):
    """Turn a list of scalar GSObjects with the same tree structure into one batched object."""
    raise GalSimIncompatibleValuesError(
        "draw_batch takes one GSObject with array-valued parameters; build the batch with numpy "
        "arrays for the parameters that vary")

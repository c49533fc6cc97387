"""ctypes binding of libgsb.so (include/gsb.h).

The library is built in-tree by galsim_b200/build.py.  There is no CPU implementation of the
drawing path: if the library or a CUDA device is missing, every drawing call raises.
PyTorch is used only to own device memory and to name the current CUDA stream.
"""
import ctypes
import math
import os

import numpy as np

from .errors import GSBLibraryError, GalSimError

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libgsb.so')

MAX_OPS, MAX_LEAVES, MAX_PHASES, MAX_SCALES = 32, 8, 8, 8
GAUSSIAN, EXPONENTIAL, SERSIC, MOFFAT, KOLMOGOROV, AIRY, BOX, INTERPOLATED = range(8)
INTERP_DELTA, INTERP_NEAREST, INTERP_LINEAR, INTERP_CUBIC, INTERP_QUINTIC, INTERP_LANCZOS, INTERP_SINC = range(7)
IMAGE_STEPK, IMAGE_MAXK, IMAGE_MAX_N = 1, 2, 4096
OP_LEAF, OP_MUL, OP_ADD, OP_PHASE, OP_SCALE = 1, 2, 3, 4, 5
LEAF_JAC_GENERAL, LEAF_SIZE_IS_HLR = 1, 2
PHASE_JAC_GENERAL = 1
F32, F64 = 0, 1
I16, I32, U16, U32 = 2, 3, 4, 5        # integer image types (gsb_add_noise)
TABLES_DN = 1
WANT_ALL = 0xffffffff
GRAD_PER_LEAF, GRAD_PER_PHASE = 6, 7


class GSParamsC(ctypes.Structure):
    _fields_ = [('minimum_fft_size', ctypes.c_int), ('maximum_fft_size', ctypes.c_int)] + \
               [(n, ctypes.c_double) for n in (
                   'folding_threshold', 'stepk_minimum_hlr', 'maxk_threshold', 'kvalue_accuracy',
                   'xvalue_accuracy', 'table_spacing', 'realspace_relerr', 'realspace_abserr',
                   'integration_relerr', 'integration_abserr', 'shoot_accuracy')]


class TemplateC(ctypes.Structure):
    _fields_ = [('n_ops', ctypes.c_int), ('n_leaves', ctypes.c_int), ('n_phases', ctypes.c_int),
                ('n_scales', ctypes.c_int), ('op_code', ctypes.c_int * MAX_OPS),
                ('op_arg', ctypes.c_int * MAX_OPS), ('leaf_type', ctypes.c_int * MAX_LEAVES)]


# Device record layouts (numpy structured dtypes with the C offsets).
LEAF_DTYPE = np.dtype({'names': ['jac', 'flux', 'p', 'd', 'flags', 'table'],
                       'formats': [('f8', 4), 'f8', ('f8', 3), ('f8', 8), 'i4', 'i4'],
                       'offsets': [0, 32, 40, 64, 128, 132], 'itemsize': 136})
PHASE_DTYPE = np.dtype({'names': ['jac', 'cenx', 'ceny', 'flux_scaling', 'flags', 'pad'],
                        'formats': [('f8', 4), 'f8', 'f8', 'f8', 'i4', 'i4'],
                        'offsets': [0, 32, 40, 48, 56, 60], 'itemsize': 64})
STAMP_DTYPE = np.dtype({'names': ['N', 'Nk', 'xmin', 'ymin', 'nx', 'ny', 'out_offset'],
                        'formats': ['i4', 'i4', 'i4', 'i4', 'i4', 'i4', 'i8'],
                        'offsets': [0, 4, 8, 12, 16, 20, 24], 'itemsize': 32})

XLEAF_DTYPE = np.dtype({'names': ['jac', 'xoff', 'yoff', 'flux_ratio', 'flux', 'p', 'type', 'flags',
                                  'region', 'rx0', 'ry0', 'rnx', 'rny', 'ktab'],
                        'formats': [('f8', 4), 'f8', 'f8', 'f8', 'f8', ('f8', 3), 'i4', 'i4',
                                    'u8', 'i4', 'i4', 'i4', 'i4', 'u8'],
                        'offsets': [0, 32, 40, 48, 56, 64, 88, 92, 96, 104, 108, 112, 116, 120],
                        'itemsize': 128})
XLEAF_JAC = 1

IMAGE_DESC_DTYPE = np.dtype({'names': ['N', 'nx', 'ny', 'x0', 'y0', 'bx0', 'bx1', 'by0', 'by1',
                                         'x_interp', 'flags', 'pix_offset', 'flux', 'stepk_target',
                                         'maxk_limit', 'x_table'],
                              'formats': ['i4'] * 11 + ['i8', 'f8', 'f8', 'f8', 'u8'],
                              'offsets': [0, 4, 8, 12, 16, 20, 24, 28, 32, 36, 40, 48, 56, 64, 72, 80],
                              'itemsize': 88})

# gsb_fits_hdu (include/gsb.h)
FITS_HDU_DTYPE = np.dtype({'names': ['header_src', 'header_len', 'data_src', 'n_elem', 'dst'],
                           'formats': ['i8'] * 5, 'offsets': [0, 8, 16, 24, 32], 'itemsize': 40})

SERSIC_HEADER = 18
SH_N, SH_NUSED, SH_FRONT, SH_DA, SH_KSQMIN, SH_KSQMAX, SH_KD2, SH_KD4, SH_HIGHA, SH_HIGHB, \
    SH_MAXK, SH_STEPK, SH_RE, SH_DLOGK, SH_NCAND, SH_STATUS, SH_TRUNC, SH_FLUXFRAC = range(18)

_lib = None


def lib():
    """Load libgsb.so once; raise if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GalSimError("libgsb.so is not built (run galsim_b200.build.build()); the "
                              "drawing path has no CPU implementation")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
        sig = {
            'gsb_last_error': (ctypes.c_char_p, []),
            'gsb_version': (i, []),
            'gsb_init': (i, [i]),
            'gsb_good_fft_size': (i, [i]),
            'gsb_tables_create': (i, [ctypes.POINTER(vp)]),
            'gsb_tables_destroy': (i, [vp]),
            'gsb_sersic_tables_build': (i, [vp, vp, vp, i, ctypes.POINTER(GSParamsC), vp]),
            'gsb_sersic_tables_build_ex': (i, [vp, vp, vp, i, ctypes.POINTER(GSParamsC), i, vp]),
            'gsb_sersic_tables_info': (i, [vp, vp, i, vp]),
            'gsb_sersic_truncation': (i, [i, vp, vp, vp]),
            'gsb_moffat_tables_build': (i, [vp, vp, vp, i, vp, vp]),
            'gsb_moffat_tables_info': (i, [vp, vp, i, vp]),
            'gsb_moffat_scale_radius': (i, [i, vp, vp, vp]),
            'gsb_weighted_stamp_sum': (i, [vp, i, vp, vp, i, ctypes.c_int64, vp, i, vp]),
            'gsb_draw_real': (i, [i, i, vp, vp, vp, vp, i, i, vp, vp]),
            'gsb_images_build': (i, [vp, i, vp, vp, ctypes.POINTER(GSParamsC), vp]),
            'gsb_images_info': (i, [vp, vp, i, vp]),
            'gsb_add_noise': (i, [i, vp, vp, i, i, vp, i, vp, vp, vp]),
            'gsb_fits_pack': (i, [vp, i, vp, ctypes.c_longlong, vp, ctypes.c_longlong, i, vp,
                                  ctypes.c_longlong, vp]),
            'gsb_permute_records': (i, [vp, vp, vp, ctypes.c_int64, ctypes.c_int64, i, vp]),
            'gsb_adjoint_grad_count': (i, [ctypes.POINTER(TemplateC)]),
            'gsb_adjoint_workspace_size': (sz, [i, i, i]),
            'gsb_adjoint_images': (i, [ctypes.POINTER(TemplateC), i, ctypes.POINTER(GSParamsC), vp, vp,
                                       vp, vp, vp, i, vp, i, vp, ctypes.c_uint, i, vp, sz, vp]),
            'gsb_prepare_leaves': (i, [ctypes.POINTER(TemplateC), i, ctypes.POINTER(GSParamsC), vp, vp,
                                       vp, vp]),
            'gsb_draw_workspace_size': (sz, [i, i, i]),
            'gsb_draw_images': (i, [ctypes.POINTER(TemplateC), i, ctypes.POINTER(GSParamsC), vp, vp, vp,
                                    vp, vp, vp, i, i, vp, i, vp, sz, vp]),
            'gsb_draw_bucket': (i, [ctypes.POINTER(TemplateC), i, ctypes.POINTER(GSParamsC), vp, vp, vp,
                                    vp, vp, i, vp, i, i, vp, i, vp, sz, vp]),
            'gsb_draw_set_variant': (i, [i]),
            'gsb_exp_fp64': (i, [vp, vp, i, vp]),
            'gsb_exp_fp64_ex': (i, [vp, vp, i, i, vp]),
            'gsb_draw_tune_report': (i, [ctypes.c_char_p, sz]),
            'gsb_draw_kimages': (i, [ctypes.POINTER(TemplateC), i, ctypes.POINTER(GSParamsC), vp, vp,
                                     vp, vp, d, i, i, i, i, vp, i, vp]),
            # the reference's hot-path steps one at a time (gsb_standalone.cu)
            'gsb_draw_k': (i, [ctypes.POINTER(TemplateC), i, ctypes.POINTER(GSParamsC), vp, vp, vp, vp, d,
                               vp, i, i, i, i, vp, i, vp]),
            'gsb_apply_kimage_phases': (i, [vp, i, i, i, i, i, ctypes.c_longlong, d, vp, d, d, d, vp]),
            'gsb_wrap_image': (i, [vp, i, i, i, i, i, i, ctypes.c_longlong, i, i, i, i, i, i, vp,
                                   ctypes.c_longlong, vp]),
            'gsb_irfft': (i, [vp, i, i, i, ctypes.c_longlong, vp, ctypes.c_longlong, i, i, vp, sz, vp]),
            'gsb_irfft_workspace_size': (sz, [i, i]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise GSBLibraryError(rc, lib().gsb_last_error().decode())
    return rc


def good_fft_size(n):
    """goodFFTSize (src/Image.cpp:1141-1153) through the C ABI."""
    return lib().gsb_good_fft_size(int(n))


def gsparams_c(gsp):
    g = GSParamsC()
    (g.minimum_fft_size, g.maximum_fft_size, g.folding_threshold, g.stepk_minimum_hlr,
     g.maxk_threshold, g.kvalue_accuracy, g.xvalue_accuracy, g.table_spacing, g.realspace_relerr,
     g.realspace_abserr, g.integration_relerr, g.integration_abserr, g.shoot_accuracy) = \
        gsp._getinitargs()
    return g


class Device(object):
    """The CUDA device the library draws on (cuda:0 unless set_device was called)."""
    _index = 0
    _ready = set()

    @classmethod
    def torch_device(cls):
        import torch
        if not torch.cuda.is_available():
            raise GalSimError("galsim_b200 draws on a CUDA device (B200) and none is available; "
                              "there is no CPU fallback")
        dev = torch.device('cuda', cls._index)
        if cls._index not in cls._ready:
            torch.cuda.set_device(dev)
            torch.cuda.init()
            check(lib().gsb_init(cls._index))
            cls._ready.add(cls._index)
        return dev

    @classmethod
    def stream(cls):
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream(cls.torch_device()).cuda_stream)

    _side = {}

    @classmethod
    def side_streams(cls, n):
        """n reusable side streams of the current device (for concurrent FFT-size buckets)."""
        import torch
        dev = cls.torch_device()
        lst = cls._side.setdefault(dev.index, [])
        while len(lst) < n:
            lst.append(torch.cuda.Stream(device=dev))
        return lst[:n]


def sersic_truncation(n, size, trunc, size_is_hlr, flux_untruncated):
    """(r0, flux fraction) per truncated Sersic profile, by FP64 root finding on the device
    (gsb_sersic_truncation)."""
    n, size, trunc = np.broadcast_arrays(np.atleast_1d(np.asarray(n, float)), np.asarray(size, float),
                                         np.asarray(trunc, float))
    inp = np.stack([n, size, trunc, np.full(n.shape, (1 if size_is_hlr else 0) | (2 if flux_untruncated else 0),
                                            dtype=float)], -1)
    inp = np.ascontiguousarray(inp, dtype=np.float64)
    out = np.zeros((len(n), 2))
    Device.torch_device()
    check(lib().gsb_sersic_truncation(len(n), inp.ctypes.data_as(ctypes.c_void_p),
                                      out.ctypes.data_as(ctypes.c_void_p), Device.stream()))
    return out[:, 0], out[:, 1]


MOFFAT_HEADER = 8
(MH_BETA, MH_TRUNC, MH_FLUXFACTOR, MH_DK, MH_NUSED, MH_KSQMAX, MH_MAXK, MH_STATUS) = range(8)


def moffat_scale_radius(beta, hlr, trunc):
    """Scale radius per Moffat profile from its half-light radius (trunc 0: untruncated), by
    FP64 root finding on the device for truncated profiles (gsb_moffat_scale_radius)."""
    beta, hlr, trunc = np.broadcast_arrays(np.atleast_1d(np.asarray(beta, float)), np.asarray(hlr, float),
                                           np.asarray(trunc, float))
    inp = np.ascontiguousarray(np.stack([beta, hlr, trunc], -1), dtype=np.float64)
    out = np.zeros(len(beta))
    Device.torch_device()
    check(lib().gsb_moffat_scale_radius(len(beta), inp.ctypes.data_as(ctypes.c_void_p),
                                        out.ctypes.data_as(ctypes.c_void_p), Device.stream()))
    return out


def set_draw_variant(variant):
    """0 automatic (autotuned), 1 fused kernel only, 2 split kernels where N >= 192."""
    check(lib().gsb_draw_set_variant(int(variant)))


def tune_report():
    """The autotuner's choices, one line per (device, precision, N, stamp-count class)."""
    n = lib().gsb_draw_tune_report(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib().gsb_draw_tune_report(buf, n + 1)
    return buf.value.decode()


def set_device(index):
    Device._index = int(index)


def to_device(arr):
    """Copy a numpy (structured) array to a new device buffer; returns the torch tensor."""
    import torch
    dev = Device.torch_device()
    raw = np.ascontiguousarray(arr).view(np.uint8).reshape(-1)
    if raw.size == 0:
        return torch.empty(8, dtype=torch.uint8, device=dev)
    t = torch.from_numpy(raw)
    return t.to(dev, non_blocking=False)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def permute_records(dst, src, perm, scatter=False, stream=None):
    """gsb_permute_records on device tensors: dst[i] = src[perm[i]] (gather) or
    dst[perm[i]] = src[i] (scatter), one record per leading-dimension row; perm int64 on the
    device.  Asynchronous on `stream` (default: the current stream)."""
    count = int(perm.numel())
    rec = (src.numel() * src.element_size()) // count if count else 0
    if rec == 0:
        return dst
    check(lib().gsb_permute_records(ptr(dst), ptr(src), ptr(perm), count, rec, 1 if scatter else 0,
                                    stream if stream is not None else Device.stream()))
    return dst


class Tables(object):
    """A device FT table set (gsb_tables)."""

    def __init__(self):
        Device.torch_device()
        h = ctypes.c_void_p()
        check(lib().gsb_tables_create(ctypes.byref(h)))
        self.handle = h

    def build_sersic(self, n_values, gsp, with_dn=False, trunc_over_r0=None):
        """Build one table per Sersic index (and truncation radius / r0, 0 = untruncated);
        with_dn also builds the d/dn tables that the adjoint needs (the tables themselves are
        the same either way)."""
        n = np.ascontiguousarray(n_values, dtype=np.float64)
        tr = None if trunc_over_r0 is None else np.ascontiguousarray(trunc_over_r0, dtype=np.float64)
        check(lib().gsb_sersic_tables_build_ex(self.handle, n.ctypes.data_as(ctypes.c_void_p),
                                               tr.ctypes.data_as(ctypes.c_void_p) if tr is not None else None,
                                               len(n), ctypes.byref(gsparams_c(gsp)),
                                               TABLES_DN if with_dn else 0, Device.stream()))
        self.count = len(n)
        self.with_dn = with_dn
        self.generation = getattr(self, 'generation', 0) + 1

    def build_moffat(self, beta, trunc_over_rd, gsp):
        """Build one truncated-Moffat table per (beta, trunc / scale radius) pair."""
        b = np.ascontiguousarray(beta, dtype=np.float64)
        t = np.ascontiguousarray(trunc_over_rd, dtype=np.float64)
        check(lib().gsb_moffat_tables_build(self.handle, b.ctypes.data_as(ctypes.c_void_p),
                                            t.ctypes.data_as(ctypes.c_void_p), len(b),
                                            ctypes.byref(gsparams_c(gsp)), Device.stream()))
        self.moffat_count = len(b)
        self.generation = getattr(self, 'generation', 0) + 1

    def moffat_info(self, count=None):
        count = self.moffat_count if count is None else count
        out = np.zeros((count, MOFFAT_HEADER))
        check(lib().gsb_moffat_tables_info(self.handle, out.ctypes.data_as(ctypes.c_void_p), count,
                                           Device.stream()))
        return out

    def build_images(self, desc, pixels, gsp):
        """Build the k-images (and stepk / maxk scans) of the InterpolatedImage sources:
        desc an IMAGE_DESC_DTYPE array, pixels the packed FP64 pixels (a device tensor)."""
        desc = np.ascontiguousarray(desc, dtype=IMAGE_DESC_DTYPE)
        check(lib().gsb_images_build(self.handle, len(desc), desc.ctypes.data_as(ctypes.c_void_p),
                                     ptr(pixels), ctypes.byref(gsparams_c(gsp)), Device.stream()))
        self.n_images = len(desc)
        self.generation = getattr(self, 'generation', 0) + 1

    def image_info(self, count=None):
        """(R, maxk) per image slot, image units."""
        count = self.n_images if count is None else count
        out = np.zeros((count, 2))
        check(lib().gsb_images_info(self.handle, out.ctypes.data_as(ctypes.c_void_p), count,
                                    Device.stream()))
        return out

    def sersic_info(self, count=None):
        count = self.count if count is None else count
        out = np.zeros((count, SERSIC_HEADER))
        check(lib().gsb_sersic_tables_info(self.handle, out.ctypes.data_as(ctypes.c_void_p), count,
                                           Device.stream()))
        return out

    def __del__(self):
        try:
            if self.handle:
                lib().gsb_tables_destroy(self.handle)
        except Exception:
            pass


class TablePool(object):
    """Idle table sets of the current process, reused by later programs: freeing device memory
    synchronises the device and is slow for table sets of hundreds of MB, and a new set would
    only allocate the same memory again."""
    _idle = {}

    @classmethod
    def acquire(cls):
        dev = Device.torch_device().index
        lst = cls._idle.setdefault(dev, [])
        return lst.pop() if lst else Tables()

    @classmethod
    def release(cls, t):
        if t is None:
            return
        try:
            dev = Device.torch_device().index
        except Exception:
            return
        lst = cls._idle.setdefault(dev, [])
        if len(lst) < 4:
            lst.append(t)

"""The C ABI library: it loads and exports every entry point that include/gsb.h declares.
No compute calls (CPU only)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, 'include', 'gsb.h')
LIB = os.path.join(ROOT, 'galsim_b200', 'libgsb.so')


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(gsb_[a-z0-9_]+)\s*\(', text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ('gsb_init', 'gsb_good_fft_size', 'gsb_sersic_tables_build', 'gsb_prepare_leaves',
              'gsb_draw_images', 'gsb_draw_kimages', 'gsb_last_error'):
        assert n in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        from galsim_b200.build import build
        build()
    lib = ctypes.CDLL(LIB)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_struct_layouts_match_header():
    from galsim_b200 import _lib
    assert _lib.LEAF_DTYPE.itemsize == 136
    assert _lib.PHASE_DTYPE.itemsize == 64
    assert _lib.STAMP_DTYPE.itemsize == 32
    assert ctypes.sizeof(_lib.GSParamsC) == 8 + 11 * 8
    assert ctypes.sizeof(_lib.TemplateC) == 4 * (4 + 2 * _lib.MAX_OPS + _lib.MAX_LEAVES)


def test_good_fft_size_host_function():
    """gsb_good_fft_size is host integer logic; check it and the vectorised host copy against
    the reference's values."""
    import specs
    from galsim_b200 import _lib
    from galsim_b200.program import good_fft_size_array
    gold = np.load(os.path.join(specs.HERE, 'reference_draws.npz'))
    ins, outs = gold['good_fft_in'], gold['good_fft_out']
    assert [_lib.good_fft_size(int(v)) for v in ins] == list(outs)
    assert np.array_equal(good_fft_size_array(ins), outs)


def test_permute_records_argument_checks():
    """gsb_permute_records refuses bad sizes, null and unaligned pointers and aliasing before
    any device work; a zero count is a no-op."""
    from galsim_b200 import _lib
    lib = _lib.lib()
    vp = ctypes.c_void_p
    GSB_OK, GSB_ERR_INVALID = 0, -1
    assert lib.gsb_permute_records(None, None, None, 0, 8, 0, None) == GSB_OK
    assert lib.gsb_permute_records(vp(64), vp(128), vp(256), 4, 12, 0, None) == GSB_ERR_INVALID
    assert lib.gsb_permute_records(vp(64), vp(128), vp(256), 4, 0, 0, None) == GSB_ERR_INVALID
    assert lib.gsb_permute_records(vp(64), vp(128), vp(256), -1, 8, 0, None) == GSB_ERR_INVALID
    assert lib.gsb_permute_records(vp(64), vp(128), vp(256), 4, 8, 2, None) == GSB_ERR_INVALID
    assert lib.gsb_permute_records(None, vp(128), vp(256), 4, 8, 0, None) == GSB_ERR_INVALID
    assert lib.gsb_permute_records(vp(64), vp(64), vp(256), 4, 8, 1, None) == GSB_ERR_INVALID
    assert lib.gsb_permute_records(vp(68), vp(128), vp(256), 4, 8, 0, None) == GSB_ERR_INVALID
    assert b'aligned' in lib.gsb_last_error()

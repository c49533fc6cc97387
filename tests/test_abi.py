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

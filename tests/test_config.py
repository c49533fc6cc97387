"""Config-driven batching: value parsing and object building on CPU; the GPU stamps of a
config against the reference's own galsim.config.BuildStamps (tests/golden/reference_config.npz,
made by tests/golden/make_golden.py)."""
import copy
import os

import numpy as np
import pytest

import galsim_b200 as galsim
from galsim_b200 import config as C
import make_golden as MG

HERE = os.path.dirname(os.path.abspath(__file__))


def test_value_types_follow_the_reference_rules():
    ctx = C._Ctx(7, {'a': np.arange(10.) * 2})
    assert np.array_equal(C._float(ctx, 3.5), np.full(7, 3.5))
    assert np.array_equal(C._float(ctx, {'type': 'List', 'items': [1, 2, 3]}), [1, 2, 3, 1, 2, 3, 1])
    assert np.array_equal(C._float(ctx, {'type': 'Sequence', 'first': 1, 'step': 2, 'repeat': 2}),
                          [1, 1, 3, 3, 5, 5, 7])
    assert np.array_equal(C._float(ctx, {'type': 'Sequence', 'first': 0, 'step': 1, 'nitems': 3}),
                          [0, 1, 2, 0, 1, 2, 0])
    assert np.array_equal(C._float(ctx, {'type': 'Catalog', 'col': 'a'}), np.arange(7.) * 2)
    assert np.array_equal(C._float(ctx, {'type': 'Sum', 'items': [1., {'type': 'List', 'items': [0, 1]}]}),
                          [1, 2, 1, 2, 1, 2, 1])
    th = C._angle(ctx, '90 deg')
    assert np.allclose(th, np.pi / 2)
    g1, g2 = C._shear(ctx, {'type': 'GBeta', 'g': 0.2, 'beta': '45 deg'})
    assert np.allclose(g1, 0.) and np.allclose(g2, 0.2)
    g1, g2 = C._shear(ctx, {'type': 'E1E2', 'e1': 0.3, 'e2': 0.})
    ref = galsim.Shear(e1=0.3, e2=0.)
    assert np.allclose(g1, ref.g1) and np.allclose(g2, 0.)


def test_unsupported_types_raise_config_errors():
    ctx = C._Ctx(2, None)
    with pytest.raises(galsim.GalSimConfigError):
        C._float(ctx, {'type': 'RandomGaussian', 'sigma': 1.})
    with pytest.raises(galsim.GalSimConfigError):
        C.build_object(ctx, {'type': 'InterpolatedImage', 'image': 'x.fits'})
    with pytest.raises(galsim.GalSimConfigError):
        C.build_object(ctx, {'type': 'Gaussian', 'sigma': 1., 'bogus': 2.})
    with pytest.raises(galsim.GalSimConfigError):
        C._float(ctx, {'type': 'Catalog', 'col': 'n'})


def test_config_batch_topology(monkeypatch):
    from galsim_b200 import program
    monkeypatch.setattr(program.Program, 'upload', lambda self: None)
    prof, ctx = C.build_batch(copy.deepcopy(MG.CONFIG_CASE), MG.CONFIG_NOBJ)
    prog = program.Program(prof)
    assert prog.B == MG.CONFIG_NOBJ
    assert len(prog.bld.leaves) == 3          # Sersic, Exponential, Moffat


@pytest.mark.gpu
def test_config_stamps_match_reference_buildstamps():
    gold = np.load(os.path.join(HERE, 'golden', 'reference_config.npz'))
    st = C.draw_config(copy.deepcopy(MG.CONFIG_CASE), MG.CONFIG_NOBJ)
    arrs = st.arrays()
    for i in range(MG.CONFIG_NOBJ):
        ref = gold['stamp_%d' % i]
        assert arrs[i].shape == ref.shape
        assert np.abs(arrs[i].astype(float) - ref).max() <= 1e-5 * np.abs(ref).max(), i

"""Host-side logic on the CPU: parameter parsing, tree flattening into programs, and the
GalSim sizing rules (no GPU)."""
import math

import numpy as np
import pytest

import galsim_b200 as galsim
from galsim_b200 import _lib
from galsim_b200.program import Builder, Program, fft_sizes, good_image_size
import galsim_oracle as O


def test_program_for_config1_tree():
    gal = galsim.Exponential(flux=1e4, half_light_radius=1.0).shear(g1=0.05, g2=-0.03).shift(0.13, -0.07)
    obj = galsim.Convolve(gal, galsim.Moffat(beta=3.0, fwhm=0.7), galsim.Pixel(0.2))
    p = Program(obj)
    ops = [(p.tpl.op_code[i], p.tpl.op_arg[i]) for i in range(p.tpl.n_ops)]
    assert ops == [(_lib.OP_LEAF, 0), (_lib.OP_PHASE, 0), (_lib.OP_LEAF, 1), (_lib.OP_MUL, 0),
                   (_lib.OP_LEAF, 2), (_lib.OP_MUL, 0)]
    leaf = p.bld.leaves[0]
    m = np.array([[1.05, -0.03], [-0.03, 0.95]]) / math.sqrt(1 - 0.05 ** 2 - 0.03 ** 2)
    assert np.allclose(leaf['jac'][0], m.ravel())
    assert leaf['flags'][0] & _lib.LEAF_JAC_GENERAL
    assert p.bld.leaves[1]['flags'][0] == 0
    ph = p.bld.phases[0]
    assert ph['cenx'][0] == 0.13 and ph['ceny'][0] == -0.07


def test_nested_transforms_flatten_like_reference():
    g = galsim.Gaussian(sigma=1.).shift(0.5, 0.2).shear(g1=0.1, g2=0.).dilate(2.)
    assert isinstance(g, galsim.Transformation)
    assert isinstance(g.original, galsim.Gaussian)
    o = O.OGaussian(1.).shift(0.5, 0.2).shear(0.1, 0.)
    o = O.OTransform(o, jac=[[2., 0.], [0., 2.]], flux_ratio=0.25)
    assert np.allclose(g.jac, o.jac)
    assert np.allclose([g._dx, g._dy], [o.dx, o.dy])


def test_batched_parameters_make_one_template():
    n = np.array([1., 2., 3.])
    gal = galsim.Sersic(n=n, half_light_radius=np.array([0.5, 0.6, 0.7]), flux=100.)
    obj = galsim.Convolve(gal.shear(g1=np.array([0.1, 0., -0.1]), g2=0.), galsim.Kolmogorov(fwhm=0.7))
    assert obj._batch == 3
    p = Program(obj)
    assert p.B == 3
    flags = p.bld.leaves[0]['flags']
    assert list(flags & _lib.LEAF_JAC_GENERAL) == [0, 0, 0]   # g2 = 0: diagonal jacobians
    assert list(flags & _lib.LEAF_SIZE_IS_HLR) == [2, 2, 2]


def test_sizing_matches_oracle_rules():
    rng = np.random.default_rng(5)
    sk = rng.uniform(0.05, 1.0, 50)
    mk = rng.uniform(1.0, 20.0, 50)
    N, Nk = fft_sizes(sk, mk, -32, 31, -32, 31, galsim.GSParams())
    for i in range(50):
        Nd = 2 * math.pi / sk[i]
        n0 = int(math.ceil(Nd * (1 - 1e-12)))
        n0 = 2 * ((n0 + 1) // 2)
        n1 = max(O.good_fft_size(max(n0, 64)), 128)
        dk = 2 * math.pi / n1
        nk = n1 if n1 * dk / 2 > mk[i] else int(math.ceil(mk[i] / dk)) * 2
        assert (N[i], Nk[i]) == (n1, nk)


def test_parameter_validation_matches_reference():
    with pytest.raises(galsim.GalSimRangeError):
        galsim.Sersic(n=0.2, half_light_radius=1.)
    with pytest.raises(galsim.GalSimRangeError):
        galsim.Moffat(beta=1.05, fwhm=1.)
    with pytest.raises(galsim.GalSimIncompatibleValuesError):
        galsim.Gaussian(sigma=1., fwhm=2.)
    with pytest.raises(galsim.GalSimRangeError):
        galsim.Shear(g1=0.9, g2=0.9)
    with pytest.raises(galsim.GalSimError):
        galsim.Transform(galsim.Gaussian(sigma=1.), jac=[1., 1., 1., 1.])


def test_draw_requires_gpu_without_fallback():
    """On a machine without CUDA the drawing path raises instead of computing on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    with pytest.raises(galsim.GalSimError):
        galsim.Gaussian(sigma=1.).drawImage(nx=16, ny=16, scale=0.2)


def test_adjoint_gradient_layout_from_library():
    """gsb_adjoint_grad_count is host logic: 6 entries per leaf, 7 per phase, 1 per scale."""
    import ctypes
    from galsim_b200 import _lib
    from galsim_b200.program import Program
    obj = galsim.Convolve(galsim.Sersic(n=2., half_light_radius=0.5).shear(g1=0.1, g2=0.).shift(0.1, 0.),
                          galsim.Moffat(beta=2.5, fwhm=0.8) * 2., galsim.Pixel(0.2))
    prog = Program(obj)
    L, P, S = len(prog.bld.leaves), len(prog.bld.phases), len(prog.bld.scales)
    assert (L, P, S) == (3, 1, 1)
    n = _lib.lib().gsb_adjoint_grad_count(ctypes.byref(prog.tpl))
    assert n == 6 * L + 7 * P + S
    bad = _lib.TemplateC()
    assert _lib.lib().gsb_adjoint_grad_count(ctypes.byref(bad)) < 0   # empty template


def test_torch_shear_matrix_matches_shear():
    import torch
    from galsim_b200.autodiff import shear_matrix
    g1 = np.array([0.1, -0.3, 0.0, 0.25])
    g2 = np.array([0.05, 0.2, 0.0, -0.4])
    m = shear_matrix(torch.as_tensor(g1), torch.as_tensor(g2)).numpy()
    ref = galsim.Shear(g1=g1, g2=g2).getMatrix()
    np.testing.assert_allclose(m, ref, rtol=1e-15, atol=1e-15)


def test_bench_table_launch_count_follows_the_round_size():
    """bench.py's gpu_launches claim counts one (nodes, scan) pair per round of kTableRound ln k
    nodes; the count must follow the round size the table build is compiled with."""
    import os
    import re
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = open(os.path.join(root, 'galsim_b200', 'csrc', 'gsb_tables.cu')).read()
    rnd = int(re.search(r'constexpr int kTableRound = (\d+);', src).group(1))
    sys.path.insert(0, root)
    import bench
    for n in (0.5, 1.5, 4.0, 6.2):
        kderiv6 = math.exp(math.lgamma(8. * n) - math.lgamma(2. * n)) / 2304.
        kmin = (1e-5 / kderiv6) ** (1. / 6.)
        dlogk = math.sqrt(math.sqrt(1e-6))
        stride = int((math.log(500.) - (math.log(kmin) - 0.001)) / dlogk) + 4
        assert bench.table_build_launches(np.array([n])) == 3 + 2 * ((stride + rnd - 1) // rnd)

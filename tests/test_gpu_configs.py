"""GPU parity of the batched configurations at their own settings, against stamps that the
reference's own drawImage drew one by one (tests/golden/reference_configs.npz, made by
make_golden.py --configs-only from bench.py's seeded generators):

* batched forward: the leading 256 stamps of the 4096-stamp Sersic x Kolmogorov x Pixel(0.2)
  workload (seed 1234), default GSParams, automatically sized float32 images;
* mixed bulge+disk: Sum(Sersic(n=4), Exponential) with independent shears, convolved with a
  general-beta Moffat and Pixel(0.2), GSParams(minimum_fft_size=32) -- 16 leading stamps of
  the 16384-stamp workload (seed 2468) plus three stamps of every FFT size it uses (64..512).

Each stamp is drawn inside one batch of the whole sample (the measured path) and compared on
its centred block and a strided pixel grid: FP32 kernels to max |diff| <= 1e-5 x peak and
added flux <= 1e-6 relative (the contract); FP64 kernels to 2e-7 x peak, the rounding of the
reference's own complex64 k-images for float32 images; the image shape and GalSim's FFT sizes
(N, Nk) must equal the reference's.
"""
import os

import numpy as np
import pytest

import galsim_b200 as galsim
import make_golden as MG

pytestmark = pytest.mark.gpu
CFG = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'reference_configs.npz'))


def _check(prefix, st, precision):
    shapes = CFG[prefix + '_shape']
    sizes = CFG[prefix + '_N_Nk']
    assert len(st) == len(shapes)
    bo = go = 0
    worst, worst_f = 0., 0.
    for i in range(len(st)):
        a = st.array(i)
        assert a.shape == tuple(shapes[i]), (prefix, i)
        assert (int(st.N[i]), int(st.Nk[i])) == tuple(sizes[i]), (prefix, i)
        block, grid = MG.config_sample(a)
        rb = CFG[prefix + '_block'][bo:bo + block.size].reshape(block.shape)
        rg = CFG[prefix + '_grid'][go:go + grid.size].reshape(grid.shape)
        bo += block.size
        go += grid.size
        peak = float(CFG[prefix + '_peak'][i])
        err = max(np.abs(block.astype(float) - rb).max(), np.abs(grid.astype(float) - rg).max()) / peak
        fref = float(CFG[prefix + '_flux'][i])
        ferr = abs(st.added_flux[i] - fref) / abs(fref)
        worst, worst_f = max(worst, err), max(worst_f, ferr)
    # FP64 kernels: the reference drew float32 images through complex64 k-images, so its own
    # rounding (<= 2e-7 x peak, the oracle pin for float32 fixtures) sets the bound
    ptol, ftol = (1e-5, 1e-6) if precision == 'fp32' else (2e-7, 1e-6)
    assert worst <= ptol, (prefix, precision, worst)
    assert worst_f <= ftol, (prefix, precision, worst_f)
    return worst, worst_f


@pytest.mark.parametrize('precision', ['fp32', 'fp64'])
def test_batched_forward_sample_vs_reference(precision):
    p = CFG['c2_params']
    obj = galsim.Convolve(galsim.Sersic(n=p[:, 0], half_light_radius=p[:, 1], flux=p[:, 2])
                          .shear(g1=p[:, 3], g2=p[:, 4]),
                          galsim.Kolmogorov(fwhm=p[:, 5]), galsim.Pixel(0.2))
    dt = np.float32 if precision == 'fp32' else np.float64
    st = galsim.draw_batch(obj, scale=0.2, dtype=dt, precision=precision)
    _check('c2', st, precision)


@pytest.mark.parametrize('precision', ['fp32', 'fp64'])
def test_mixed_bulge_disk_sample_vs_reference(precision):
    bench = MG.bench_module()
    m = bench.mixed_params()
    idx = CFG['c4_index']
    sub = {k: v[idx] for k, v in m.items()}
    gsp = galsim.GSParams(minimum_fft_size=32)
    dt = np.float32 if precision == 'fp32' else np.float64
    st = galsim.draw_batch(bench.mixed_object(galsim, sub, gsp), scale=0.2, dtype=dt, precision=precision)
    assert sorted(set(int(v) for v in st.N)) == sorted(set(int(v) for v in CFG['c4_pool_N']))
    _check('c4', st, precision)

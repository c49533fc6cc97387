"""GPU parity: the CUDA drawing path (through the C ABI) against fixtures made by the
reference and against the FP64 oracle.

Tolerances: max |image difference| <= 1e-5 x peak pixel and
|added_flux difference| <= 1e-6 relative for the FP32 path; the FP64 path is held to
1e-9 x peak.
"""
import numpy as np
import pytest

import galsim_b200 as galsim
import galsim_oracle as O
import make_golden as MG
import specs

pytestmark = pytest.mark.gpu
GOLD = np.load(specs.HERE + '/reference_draws.npz')


def build(spec):
    return MG.profile(galsim, spec)


@pytest.mark.parametrize('case', MG.DRAW_CASES, ids=[c[0] for c in MG.DRAW_CASES])
def test_draw_image_fp32_vs_reference(case):
    name, spec, nx, ny, scale, dt, off = case
    im = build(spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type, method='fft',
                               offset=off)
    ref = GOLD['draw_' + name]
    peak = np.abs(ref).max()
    assert im.array.dtype == ref.dtype
    err = np.abs(im.array.astype(float) - ref).max()
    assert err <= 1e-5 * peak, (name, err / peak)
    fref = float(GOLD['draw_' + name + '_flux'])
    assert abs(im.added_flux - fref) <= 1e-6 * abs(fref), (name, im.added_flux, fref)


@pytest.mark.parametrize('case', MG.DRAW_CASES[:6], ids=[c[0] for c in MG.DRAW_CASES[:6]])
def test_draw_image_fp64_vs_reference(case):
    name, spec, nx, ny, scale, dt, off = case
    if dt != 'f8':
        pytest.skip('the reference computes float32 images in complex64')
    im = build(spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.float64, method='fft',
                               offset=off, precision='fp64')
    ref = GOLD['draw_' + name]
    assert np.abs(im.array - ref).max() <= 1e-9 * np.abs(ref).max()


@pytest.mark.parametrize('case', MG.KIMAGE_CASES, ids=[c[0] for c in MG.KIMAGE_CASES])
def test_draw_kimage_vs_reference(case):
    name, spec, dk, n = case
    im = build(spec).drawKImage(nx=n, ny=n, scale=dk)
    ref = GOLD['kimg_' + name]
    assert (im.bounds.xmin, im.bounds.ymin) == tuple(GOLD['kimg_' + name + '_xmin'])
    assert np.abs(im.array - ref).max() <= 1e-9 * np.abs(ref).max(), name


def test_leaf_sizes_vs_reference():
    for spec, (sk, mk) in zip(MG.SIZE_CASES, GOLD['sizes']):
        obj = build(spec)
        # The reference's Kolmogorov stepk goes through its approximate exp
        # (include/galsim/fmath/fmath.hpp:457-478), which moves it at the 1e-7 level.
        assert abs(obj.stepk - sk) <= 5e-7 * sk, spec
        assert abs(obj.maxk - mk) <= 1e-7 * mk, spec


def test_sersic_scale_radius_vs_reference():
    n = np.array([0.5, 0.8, 1.0, 1.5, 2.5, 4.0, 6.0])
    r0 = galsim.Sersic(n=n, half_light_radius=1.).scale_radius
    assert np.allclose(r0, GOLD['sersic_r0'], rtol=1e-12, atol=0)


def test_batch_matches_oracle_per_stamp():
    """draw_batch of a config-2-like batch (Sersic x Kolmogorov x Pixel, automatic sizes)
    against the oracle stamp by stamp."""
    rng = np.random.default_rng(1234)
    B = 6
    n = rng.uniform(0.5, 4.0, B)
    hlr = np.exp(np.log(0.5) + 0.3 * rng.normal(size=B))
    flux = np.exp(np.log(1e4) + rng.normal(size=B))
    g1 = np.clip(rng.normal(0, 0.2, B), -0.5, 0.5)
    g2 = np.clip(rng.normal(0, 0.2, B), -0.5, 0.5)
    fwhm = rng.uniform(0.6, 0.9, B)
    gal = galsim.Sersic(n=n, half_light_radius=hlr, flux=flux).shear(g1=g1, g2=g2)
    obj = galsim.Convolve(gal, galsim.Kolmogorov(fwhm=fwhm), galsim.Pixel(0.2))
    st = galsim.draw_batch(obj, scale=0.2, dtype=np.float32)
    arrs = st.arrays()
    for i in range(B):
        o = O.OConvolve(O.OSersic(n[i], hlr=hlr[i], flux=flux[i]).shear(g1[i], g2[i]),
                        O.OKolmogorov(fwhm=fwhm[i]), O.OBox(0.2))
        ref, fref, N, Nk = O.draw_image(o, int(st.nx[i]), int(st.ny[i]), 0.2)
        assert (st.N[i], st.Nk[i]) == (N, Nk)
        assert np.abs(arrs[i] - ref).max() <= 1e-5 * np.abs(ref).max()
        assert abs(st.added_flux[i] - fref) <= 1e-6 * abs(fref)


def test_batch_equals_single_draws():
    """A batch draws exactly what the one-stamp path draws for each element."""
    fw = np.array([0.6, 0.7, 0.8, 0.9])
    obj = galsim.Convolve(galsim.Exponential(half_light_radius=np.array([0.3, 0.5, 0.7, 0.9]),
                                             flux=100.), galsim.Moffat(beta=2.5, fwhm=fw))
    st = galsim.draw_batch(obj, nx=40, ny=40, scale=0.2, dtype=np.float32)
    for i, a in enumerate(st.arrays()):
        single = galsim.Convolve(galsim.Exponential(half_light_radius=[0.3, 0.5, 0.7, 0.9][i], flux=100.),
                                 galsim.Moffat(beta=2.5, fwhm=fw[i]))
        im = single.drawImage(nx=40, ny=40, scale=0.2, dtype=np.float32, method='fft')
        assert np.array_equal(a, im.array)


def test_add_to_image():
    obj = galsim.Gaussian(sigma=0.5, flux=10.)
    im = obj.drawImage(nx=32, ny=32, scale=0.2, dtype=np.float64, method='fft')
    im2 = obj.drawImage(image=im.copy(), method='fft', add_to_image=True)
    assert np.allclose(im2.array, 2 * im.array, rtol=0, atol=1e-12 * im.array.max())


def test_fused_and_split_variants_agree():
    """The two kernels a bucket can run on (fused one-CTA-per-stamp, split column/row) give
    the same stamps to FP32 rounding, and the autotuner records its choice per class."""
    from galsim_b200 import _lib
    rng = np.random.default_rng(21)
    B = 24
    gal = galsim.Sersic(n=rng.uniform(1., 4., B), half_light_radius=rng.uniform(0.6, 1.5, B),
                        flux=1e4).shear(g1=rng.uniform(-0.2, 0.2, B), g2=rng.uniform(-0.2, 0.2, B))
    obj = galsim.Convolve(gal, galsim.Kolmogorov(fwhm=0.7), galsim.Pixel(0.2))
    res = {}
    try:
        for v in (1, 2, 0):
            _lib.set_draw_variant(v)
            st = galsim.draw_batch(obj, scale=0.2, dtype=np.float32)
            res[v] = (st.arrays(), st.added_flux, st.N.copy())
    finally:
        _lib.set_draw_variant(0)
    assert max(res[1][2]) >= 192
    for v in (2, 0):
        for a, b in zip(res[v][0], res[1][0]):
            assert np.abs(a.astype(float) - b).max() <= 2e-6 * np.abs(b).max()
        assert np.allclose(res[v][1], res[1][1], rtol=1e-6, atol=0)
    assert 'variant=' in _lib.tune_report()


def test_graph_replay_matches_eager_draw():
    """run_batch captures the draw stage of a repeated geometry as a CUDA graph on its second
    run and replays it afterwards: every run gives the stamps of an eager draw."""
    rng = np.random.default_rng(5)
    B = 40
    gal = galsim.Sersic(n=rng.uniform(0.8, 3.5, B), half_light_radius=rng.uniform(0.3, 1.0, B),
                        flux=1e3).shear(g1=rng.uniform(-0.2, 0.2, B), g2=rng.uniform(-0.2, 0.2, B))
    obj = galsim.Convolve(gal, galsim.Kolmogorov(fwhm=0.7), galsim.Pixel(0.2))
    eager = galsim.run_batch(galsim.plan_batch(obj, scale=0.2), graph=False)
    ref = eager.flat.cpu().numpy()
    plan = galsim.plan_batch(obj, scale=0.2)
    runs = [galsim.run_batch(plan) for _ in range(4)]
    assert plan.prog._graph_state['graph'] is not None
    for r in runs:
        assert np.array_equal(r.flat.cpu().numpy(), ref)
        assert np.array_equal(r.added_flux, eager.added_flux)
    # results of earlier runs are not overwritten by later replays
    assert np.array_equal(runs[1].flat.cpu().numpy(), ref)

"""GPU noise (gsb_add_noise through galsim_b200.Image.addNoise and StampBatch.addNoise) against
fixtures made by the reference and against the oracle.

The integer Poisson draws and the stream positions must agree exactly; the Gaussian deviates
go through CUDA's FP64 log / cos / sin, which may differ from the host's in the last bit, so
float64 results are held to 1e-13 relative and float32 results to one unit in the last place
(in practice they are bit-identical); integer images must hold the same integers."""
import numpy as np
import pytest

import galsim_b200 as galsim
import galsim_oracle as O
import make_golden as MG
import specs

pytestmark = pytest.mark.gpu
GOLD = np.load(specs.HERE + '/reference_noise.npz')
torch = pytest.importorskip('torch')


def product_noise(kind, seed, p):
    rng = galsim.BaseDeviate(seed)
    if kind == 'gauss':
        return galsim.GaussianNoise(rng, **p)
    if kind == 'poisson':
        return galsim.PoissonNoise(rng, **p)
    return galsim.CCDNoise(rng, **p)


def assert_close(got, ref):
    assert got.dtype == ref.dtype
    if np.issubdtype(ref.dtype, np.integer):
        # integer images: the same integers (casts truncate, the sky's integer part is exact)
        assert np.array_equal(got, ref), np.abs(got.astype(np.int64) - ref).max()
    elif ref.dtype == np.float32:
        ulp = np.spacing(np.abs(ref).astype(np.float32))
        assert np.all(np.abs(got.astype(np.float64) - ref) <= ulp), np.abs(got - ref).max()
    else:
        assert np.allclose(got, ref, rtol=1e-13, atol=1e-13), np.abs(got - ref).max()


@pytest.mark.parametrize('case', MG.NOISE_CASES, ids=[c[0] for c in MG.NOISE_CASES])
def test_image_add_noise_vs_reference(case):
    name, kind, src, dt, seed, p = case
    im = galsim.Image(GOLD['in_' + name].copy())
    im.addNoise(product_noise(kind, seed, p))
    assert_close(im.array, GOLD['out_' + name])


def test_stream_continues_across_uses():
    rng = galsim.BaseDeviate(4242)
    a = galsim.ImageF(9, 7, init_value=0.)
    b = galsim.ImageF(10, 5, init_value=0.)
    a.addNoise(galsim.GaussianNoise(rng, sigma=1.))
    assert rng._stream.used == 64            # 63 deviates use 32 pairs
    b.addNoise(galsim.PoissonNoise(rng, sky_level=3.5))
    assert_close(a.array, GOLD['stream_a'])
    assert_close(b.array, GOLD['stream_b'])


def test_stamp_batch_with_per_stamp_seeds_vs_reference():
    from galsim_b200.batch import StampBatch
    ins = [GOLD['batch_in_%d' % i] for i in range(len(MG.NOISE_BATCH_SEEDS))]
    dev = galsim._lib.Device.torch_device()
    flat = torch.as_tensor(np.concatenate([a.ravel() for a in ins]), device=dev)
    n = np.array([a.size for a in ins])
    offsets = np.concatenate([[0], np.cumsum(n)[:-1]])
    ny = np.array([a.shape[0] for a in ins])
    nx = np.array([a.shape[1] for a in ins])
    sb = StampBatch(flat, offsets, nx, ny, None, None, None, None, None, np.float32, 0.2, None)
    used = sb.addNoise(galsim.CCDNoise(sky_level=50., gain=1.3, read_noise=5.), seeds=MG.NOISE_BATCH_SEEDS)
    assert np.all(used > 2 * n)
    for i in range(len(ins)):
        assert_close(sb.array(i), GOLD['batch_out_%d' % i])


def test_many_blocks_and_odd_counts_vs_oracle():
    """Streams crossing many 624-draw blocks, odd pixel counts (a pair split across blocks)
    and a skipped start."""
    for seed, shape, skip in ((31, (129, 127), 0), (32, (40, 33), 623), (33, (11, 7), 1247)):
        ref = np.zeros(shape, np.float64)
        rng = O.base_deviate(seed)
        for _ in range(skip):
            rng()
        O.gaussian_noise(ref, rng, 2.5)
        r = galsim.BaseDeviate(seed)
        r.discard(skip)
        im = galsim.ImageD(np.zeros(shape))
        im.addNoise(galsim.GaussianNoise(r, sigma=2.5))
        assert np.allclose(im.array, ref, rtol=1e-13, atol=1e-13), (seed, np.abs(im.array - ref).max())
        assert r._stream.used == skip + 2 * ((ref.size + 1) // 2)


@pytest.mark.parametrize('case', MG.VARNOISE_CASES, ids=[c[0] for c in MG.VARNOISE_CASES])
def test_variable_gaussian_noise_vs_reference(case):
    name, src, dt, seed = case
    im = galsim.Image(GOLD['in_' + name].copy())
    im.addNoise(galsim.VariableGaussianNoise(galsim.BaseDeviate(seed), galsim.ImageD(GOLD['var_' + name])))
    assert_close(im.array, GOLD['out_' + name])


def test_variable_then_gaussian_stream_vs_reference():
    rng = galsim.BaseDeviate(4343)
    a = galsim.ImageF(9, 7, init_value=0.)
    b = galsim.ImageF(6, 5, init_value=1.)
    a.addNoise(galsim.VariableGaussianNoise(rng, galsim.ImageD(MG.variance_image(a.array))))
    assert rng._stream.used == 64
    b.addNoise(galsim.GaussianNoise(rng, sigma=2.))
    assert_close(a.array, GOLD['varstream_a'])
    assert_close(b.array, GOLD['varstream_b'])


def test_variable_gaussian_noise_batch_vs_oracle():
    """One variance image for every stamp of a batch, each stamp with its own seed."""
    from galsim_b200.batch import StampBatch
    var = MG.variance_image(np.zeros((24, 20)))
    B = 5
    base = np.random.default_rng(3).standard_normal((B, 24, 20)).astype(np.float32)
    dev = galsim._lib.Device.torch_device()
    flat = torch.as_tensor(base.reshape(-1).copy(), device=dev)
    nx, ny = np.full(B, 20), np.full(B, 24)
    sb = StampBatch(flat, np.arange(B) * 480, nx, ny, None, None, None, None, None, np.float32, 0.2, None)
    seeds = [71, 72, 73, 74, 75]
    used = sb.addNoise(galsim.VariableGaussianNoise(None, galsim.ImageD(var)), seeds=seeds)
    assert np.all(used == used[0])
    for i, seed in enumerate(seeds):
        ref = base[i].copy()
        O.variable_gaussian_noise(ref, O.base_deviate(seed), var)
        assert_close(sb.array(i), ref)


def test_variable_gaussian_noise_shape_mismatch():
    with pytest.raises(galsim.GalSimIncompatibleValuesError):
        galsim.ImageF(5, 4).addNoise(galsim.VariableGaussianNoise(galsim.BaseDeviate(1), galsim.ImageD(4, 5)))


def test_deviates_vs_reference():
    """UniformDeviate / GaussianDeviate / PoissonDeviate sequences and DeviateNoise: the same
    script as the reference's fixture (make_golden.deviate_sequences) run on this package."""
    mine = MG.deviate_sequences(galsim)
    for k, v in mine.items():
        ref = GOLD['dev_' + k]
        assert v.shape == ref.shape, k
        if k.startswith('devnoise'):
            assert_close(v, ref)
        elif k in ('gaussian', 'shared', 'dist'):
            assert np.allclose(v, ref, rtol=1e-13, atol=1e-13), (k, np.abs(v - ref).max())
        else:
            assert np.array_equal(v, ref), (k, v, ref)


def test_deviate_errors_and_state():
    with pytest.raises(galsim.GalSimRangeError):
        galsim.GaussianDeviate(1, sigma=-1.)
    with pytest.raises(galsim.GalSimValueError):
        galsim.PoissonDeviate(1, mean=-1.)
    with pytest.raises(galsim.GalSimValueError):
        galsim.PoissonDeviate(1).generate_from_expectation(np.array([1., -2.]))
    g = galsim.GaussianDeviate(77)
    g()
    d = g.duplicate()
    assert g() == d() and g() == d()            # the pair cache travels with the copy
    u = galsim.UniformDeviate(5)
    w = u.raw()
    assert u._stream.used > 0 and 0 <= w < 2 ** 32
    with pytest.raises(galsim.GalSimError):
        galsim.DeviateNoise(galsim.UniformDeviate(1)).getVariance()

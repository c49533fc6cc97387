"""The oracle's noise restatement against fixtures made by the reference (tests/golden/
make_golden.py main_noise): Mersenne Twister seeding, Box-Muller pairs, inversion / PTRD
Poisson draws and the Gaussian / Poisson / CCD application rules.  CPU only; the images are
small enough for the pure-Python generators."""
import numpy as np
import pytest

import galsim_oracle as O
import make_golden as MG
import specs

GOLD = np.load(specs.HERE + '/reference_noise.npz')


def oracle_apply(kind, image, seed, p):
    rng = O.base_deviate(seed)
    if kind == 'gauss':
        return O.gaussian_noise(image, rng, p['sigma'])
    if kind == 'poisson':
        return O.poisson_noise(image, rng, p.get('sky_level', 0.))
    return O.ccd_noise(image, rng, p.get('sky_level', 0.), p.get('gain', 1.), p.get('read_noise', 0.))


@pytest.mark.parametrize('case', MG.NOISE_CASES, ids=[c[0] for c in MG.NOISE_CASES])
def test_noise_matches_reference(case):
    name, kind, src, dt, seed, p = case
    img = GOLD['in_' + name].copy()
    oracle_apply(kind, img, seed, p)
    ref = GOLD['out_' + name]
    assert img.dtype == ref.dtype
    assert np.array_equal(img, ref), np.abs(img - ref).max()


def test_stream_continues_across_uses():
    rng = O.base_deviate(4242)
    a = np.zeros((7, 9), np.float32)
    b = np.zeros((5, 10), np.float32)
    O.gaussian_noise(a, rng, 1.)
    # GaussianNoise consumes 2 ceil(n / 2) draws; the PoissonNoise continues the same stream
    O.poisson_noise(b, rng, 3.5)
    assert np.array_equal(a, GOLD['stream_a'])
    assert np.array_equal(b, GOLD['stream_b'])


def test_batch_seeds():
    for i, seed in enumerate(MG.NOISE_BATCH_SEEDS):
        img = GOLD['batch_in_%d' % i].copy()
        O.ccd_noise(img, O.base_deviate(seed), 50., 1.3, 5.)
        assert np.array_equal(img, GOLD['batch_out_%d' % i])


@pytest.mark.parametrize('case', MG.VARNOISE_CASES, ids=[c[0] for c in MG.VARNOISE_CASES])
def test_variable_gaussian_noise_matches_reference(case):
    name = case[0]
    img = GOLD['in_' + name].copy()
    O.variable_gaussian_noise(img, O.base_deviate(case[3]), GOLD['var_' + name])
    assert np.array_equal(img, GOLD['out_' + name]), np.abs(img - GOLD['out_' + name]).max()


def test_variable_then_gaussian_stream():
    rng = O.base_deviate(4343)
    a = np.zeros((7, 9), np.float32)
    b = np.ones((5, 6), np.float32)
    O.variable_gaussian_noise(a, rng, MG.variance_image(a))
    O.gaussian_noise(b, rng, 2.)
    assert np.array_equal(a, GOLD['varstream_a'])
    assert np.array_equal(b, GOLD['varstream_b'])

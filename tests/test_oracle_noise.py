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


def _ogen(f, n):
    return [f() for _ in range(n)]


def test_deviate_sequences_match_reference():
    """The oracle's deviates (uniform_01, the boost 1.48 normal with its pair cache, the
    PoissonDeviate mean switching) reproduce the reference's deviate fixture script
    (make_golden.deviate_sequences) draw for draw."""
    r = O.base_deviate(1234)
    u = lambda: O.uniform01(r)
    assert np.array_equal(_ogen(u, 14), GOLD['dev_uniform'])

    r = O.base_deviate(2345)
    n = O.ONormal(1.5, 2.5)
    a = _ogen(lambda: n(r), 3)
    n.reset()                                    # generate clears the cache
    g = _ogen(lambda: n(r), 5)
    b = _ogen(lambda: n(r), 2)                   # the first from the cache
    unit = O.ONormal(0., 1.)                     # generate_from_variance: mean 0, sigma 1, fresh
    v = [unit(r) * np.sqrt(x) for x in (0.5, 2., 0., 9.)]
    n.reset()
    out = np.concatenate([a, g, b, v, [n(r)]])
    assert np.allclose(out, GOLD['dev_gaussian'], rtol=0, atol=0)

    r = O.base_deviate(3456)
    pd = O.OPoissonDeviate(r)
    pd.set_mean(7.3)
    a = _ogen(pd, 4) + _ogen(pd, 6)
    pd2 = O.OPoissonDeviate(r)
    pd2.set_mean(120.)
    b = _ogen(pd2, 3) + _ogen(pd2, 5)
    pz = O.OPoissonDeviate(r)
    pz.set_mean(0.)
    c = _ogen(pz, 3)
    ph = O.OPoissonDeviate(r)
    ph.set_mean(float(2 ** 31))
    d = _ogen(ph, 3)
    ph.gd.reset()                                # generate clears the normal branch's cache
    g3 = _ogen(ph, 3)
    d += _ogen(ph, 1) + g3                       # the script lists the call after it first
    e = []
    for m in (0., 3.2, 50., 0., float(2 ** 31), 7.):
        if m > 0.:
            pd.set_mean(m)
            e.append(pd())
        else:
            e.append(0.)
    pd.set_mean(7.3)
    out = np.concatenate([a, b, c, d, e, [pd()]])
    assert np.array_equal(out, GOLD['dev_poisson'])

    r = O.base_deviate(4567)
    sg = O.ONormal(0., 3.)
    s = [O.uniform01(r), sg(r), sg(r), sg(r), O.uniform01(r), O.uniform01(r)]
    assert np.array_equal(s, GOLD['dev_shared'])


def test_deviate_noise_matches_reference():
    for name, seed in (('uniform', 5678), ('gauss', 6789), ('poisson', 7890)):
        r = O.base_deviate(seed)
        if name == 'uniform':
            gen = lambda k: np.array([O.uniform01(r) for _ in range(k)])
        elif name == 'gauss':
            nrm = O.ONormal(-2., 0.5)

            def gen(k):
                nrm.reset()
                return np.array([nrm(r) for _ in range(k)])
        else:
            pdv = O.OPoissonDeviate(r)
            pdv.set_mean(4.5)
            gen = lambda k: np.array([pdv() for _ in range(k)])
        im = np.full((5, 7), 10., np.float32)
        im += gen(35).reshape(5, 7).astype(np.float32)
        imi = np.full((3, 6), 3, np.int32)
        imi += gen(18).reshape(3, 6).astype(np.int32)
        assert np.array_equal(im, GOLD['dev_devnoise_' + name])
        assert np.array_equal(imi, GOLD['dev_devnoise_i_' + name])


def test_host_deviates_match_reference():
    """Weibull, Gamma (k < 1, = 1, > 1) and Chi-square draws (boost 1.48 algorithms over the
    stream's uniforms) against the reference's sequences.  The fixture script generates an
    array first and then makes single calls, listing the first two calls before the array."""
    def order(f, ng):
        g = [f() for _ in range(ng)]
        c = [f() for _ in range(3)]
        return c[:2] + g + c[2:]
    r = O.base_deviate(2468)
    assert np.array_equal(order(lambda: O.weibull_draw(r, 1.7, 2.2), 6), GOLD['dev_weibull'])
    vals = []
    for k, th in ((0.6, 1.3), (1., 2.), (3.5, 0.7)):
        r = O.base_deviate(1357 + int(10 * k))
        vals += order(lambda: O.gamma_draw(r, k, th), 7)
    assert np.array_equal(vals, GOLD['dev_gamma'])
    r = O.base_deviate(9753)
    assert np.array_equal(order(lambda: 2. * O.gamma_draw(r, 2.5, 1.), 5), GOLD['dev_chi2'])


def test_binomial_matches_reference():
    """BinomialDeviate: boost 1.48's inversion and BTRD, restated over the oracle's stream
    (the product's algorithm, fed by the oracle's words, against the reference)."""
    import galsim_b200.random as R

    class Words(object):
        def __init__(self, seed):
            self.r = O.base_deviate(seed)

        def uniform01(self):
            return O.uniform01(self.r)

    vals = []
    for N, pr in ((20, 0.2), (15, 0.8)):
        bd = R.BinomialDeviate.__new__(R.BinomialDeviate)
        R.BinomialDeviate.__init__(bd, 1, N, pr)
        w = Words(4321 + N)
        g = [bd._sample(w) for _ in range(6)]
        c = [bd._sample(w) for _ in range(3)]
        vals += c[:2] + g + c[2:]
    for N, pr in ((200, 0.3), (500, 0.75)):
        bd = R.BinomialDeviate.__new__(R.BinomialDeviate)
        R.BinomialDeviate.__init__(bd, 1, N, pr)
        w = Words(4321 + N)
        vals += [bd._sample(w) for _ in range(9)]
    assert np.array_equal(vals, GOLD['dev_binomial'])


def test_dist_deviate_matches_reference():
    """DistDeviate from a tabulated density: the inverse CDF (trapezoid rule, linear inverse
    table) of the stream's uniforms against the reference's draws (host only)."""
    import galsim_b200 as galsim
    tab = galsim.LookupTable([0.5, 1., 1.7, 2.5, 4., 6.], [0.2, 1.5, 2.2, 1.1, 0.4, 0.05], interpolant='linear')
    dd = galsim.DistDeviate(1, function=tab)
    r = O.base_deviate(8642)
    u = [O.uniform01(r) for _ in range(10)]
    order = u[7:9] + u[:7] + u[9:]
    mine = [dd.val(p) for p in order] + [dd.val(0.37)]
    assert np.allclose(mine, GOLD['dev_dist'], rtol=1e-14, atol=0)
    with pytest.raises(galsim.GalSimNotImplementedError):
        galsim.DistDeviate(1, function=lambda x: x, x_min=0., x_max=1.)

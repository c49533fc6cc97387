"""StampBatch.host_async: the read-back on a copy stream returns the same pixels as host(),
for reads in flight while the next batch is drawn (the pipelined catalog loop)."""
import numpy as np
import pytest

import galsim_b200 as galsim

pytestmark = pytest.mark.gpu


def _obj(seed):
    rng = np.random.default_rng(seed)
    n = 16
    gal = galsim.Sersic(n=rng.uniform(0.8, 3.5, n), half_light_radius=rng.uniform(0.3, 1.0, n),
                        flux=1e3).shear(g1=rng.uniform(-0.2, 0.2, n), g2=0.05)
    return galsim.Convolve(gal, galsim.Kolmogorov(fwhm=0.7), galsim.Pixel(0.2))


def test_pipelined_reads_match_synchronous_reads():
    pending, expected, fluxes = [], [], []
    for seed in range(4):
        sb = galsim.draw_batch(_obj(seed), scale=0.2, dtype=np.float32)
        expected.append(sb.host(copy=True))
        fluxes.append(sb.added_flux)
        pending.append(sb.host_async())
        if len(pending) == 2:
            r = pending.pop(0)
            np.testing.assert_array_equal(r.result(), expected[seed - 1])
            np.testing.assert_array_equal(r.added_flux(), fluxes[seed - 1])
    r = pending.pop(0)
    np.testing.assert_array_equal(r.result(), expected[-1])
    np.testing.assert_array_equal(r.added_flux(), fluxes[-1])


@pytest.mark.parametrize('fixed', [False, True])
def test_draw_batches_matches_draw_batch(fixed):
    """draw_batches (next batch planned on a worker thread, reads on a copy stream) yields every
    batch's pixels and fluxes exactly as draw_batch draws them, in order."""
    size = dict(nx=40, ny=40) if fixed else {}
    expected = []
    for seed in range(5):
        sb = galsim.draw_batch(_obj(seed), scale=0.2, dtype=np.float32, **size)
        expected.append((sb.host(copy=True), np.array(sb.added_flux), list(sb.offsets)))
    got = [(sb, pix.copy(), flux.copy()) for sb, pix, flux in
           galsim.draw_batches((_obj(seed) for seed in range(5)), scale=0.2, dtype=np.float32, **size)]
    assert len(got) == len(expected)
    for (sb, pix, flux), (epix, eflux, eoff) in zip(got, expected):
        assert list(sb.offsets) == eoff
        np.testing.assert_array_equal(pix, epix)
        np.testing.assert_array_equal(flux, eflux)


def test_draw_batches_empty_sequence():
    assert list(galsim.draw_batches(iter(()), scale=0.2)) == []

"""CPU tests of the chromatic path's host-side arithmetic against numbers the reference
computed (tests/golden/reference_chromatic.npz): LookupTable interpolation and integration,
SED evaluation / redshift / flux through a bandpass, Bandpass throughput and effective
wavelength, differential chromatic refraction, and the integration rules' weights."""
import os
import sys

import numpy as np
import pytest

import galsim_b200 as galsim

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, 'golden'))
import chromatic_cases as CC  # noqa: E402

REF = np.load(os.path.join(HERE, 'golden', 'reference_chromatic.npz'))


def test_effective_wavelength_vs_reference():
    b1, b2 = CC.bandpasses(galsim)
    got = np.array([b1.effective_wavelength, b2.effective_wavelength])
    assert np.allclose(got, REF['effective_wavelength'], rtol=1e-14, atol=0)


def test_sed_flux_and_values_vs_reference():
    s1, s2 = CC.seds(galsim)
    b1, b2 = CC.bandpasses(galsim)
    got = np.array([s1.calculateFlux(b1), s2.calculateFlux(b2), s1.atRedshift(0.3).calculateFlux(b1),
                    s2.atRedshift(0.3).calculateFlux(b2), (s1 * 2.5).calculateFlux(b2)])
    assert np.allclose(got, REF['sed_flux'], rtol=1e-14, atol=0)
    waves = np.linspace(400., 600., 37)
    vals = np.array([s1(waves), s2(waves), s1.atRedshift(0.3)(waves)])
    assert np.allclose(vals, REF['sed_values'], rtol=1e-15, atol=0)
    bp = np.array([b1(waves), b2(np.linspace(540., 720., 37))])
    assert np.allclose(bp, REF['bp_values'], rtol=1e-15, atol=1e-300)


def test_refraction_vs_reference():
    w = np.array(CC.REFRACTION_WAVES)
    got = np.array([galsim.dcr.get_refraction(w, 30. * galsim.degrees),
                    galsim.dcr.get_refraction(w, 45. * galsim.degrees, temperature=280., pressure=75.)])
    assert np.allclose(got, REF['refraction'], rtol=1e-15, atol=0)


def test_lookup_table_integrals():
    x = np.array([0., 0.7, 1.1, 2.5, 3.0, 4.2])
    f = np.array([1., 2., 0.5, -1., 0.3, 2.])
    t = galsim.LookupTable(x, f, interpolant='linear')
    assert abs(t.integrate() - np.trapezoid(f, x)) <= 1e-15
    # a sub-range: the trapezoid rule on the table's points plus the interpolated ends
    xs = np.array([0.3, 0.7, 1.1, 2.5, 3.0, 3.6])
    assert abs(t.integrate(0.3, 3.6) - np.trapezoid(t(xs), xs)) <= 1e-14
    # the product with a linear function is exact for piecewise quadratics
    g = lambda w: 2. * w + 1.
    xx = np.linspace(0.3, 3.6, 200001)
    assert abs(t.integrate_product(g, 0.3, 3.6) - np.trapezoid(t(xx) * g(xx), xx)) <= 1e-8


@pytest.mark.parametrize('rule', ['midptRule', 'trapzRule', 'quadRule'])
def test_rule_weights_integrate_linear_throughput(rule):
    """With f = 1 the rules' weights sum to their estimate of the bandpass integral: exact
    for the quadratic and trapezoid rules on a linear table."""
    b1, _ = CC.bandpasses(galsim)
    xs = b1.wave_list
    gs = getattr(galsim.integ, rule).calculateWeights(xs, b1)
    exact = b1._tp.integrate()
    if rule == 'midptRule':
        assert abs(gs.sum() - exact) <= 0.05 * exact
    else:
        assert abs(gs.sum() - exact) <= 1e-12 * exact


def test_chromatic_types_and_errors():
    s1, s2 = CC.seds(galsim)
    gal = galsim.Exponential(half_light_radius=0.5) * s1
    assert isinstance(gal, galsim.SimpleChromaticTransformation) and gal.separable and gal.spectral
    psf = galsim.ChromaticAtmosphere(galsim.Kolmogorov(fwhm=0.7), 500., zenith_angle=30. * galsim.degrees)
    conv = galsim.Convolve(gal, psf)
    assert isinstance(conv, galsim.ChromaticConvolution) and not conv.separable
    assert isinstance(gal + galsim.Gaussian(sigma=1.) * s2, galsim.ChromaticSum)
    with pytest.raises(galsim.GalSimIncompatibleValuesError):
        galsim.Convolve(gal, galsim.Gaussian(sigma=1.) * s2)        # two spectral objects
    with pytest.raises(TypeError):
        galsim.Gaussian(sigma=1.) * (lambda w: w)                  # callable flux ratio must be an SED
    with pytest.raises(galsim.GalSimSEDError):
        galsim.ChromaticObject(galsim.Gaussian(sigma=1.)).drawImage(CC.bandpasses(galsim)[0])
    with pytest.raises(galsim.GalSimRangeError):
        s1(200.)                                                    # outside the SED's table


def test_real_space_records_follow_the_drawreal_walk():
    """The host flattening of drawReal (transform.py:571-583): composed Jacobian, offset with
    the outer Jacobian applied, flux scaling |det| x flux_ratio."""
    from galsim_b200.realspace import xleaf_records
    g = galsim.Gaussian(sigma=0.5, flux=2.).shear(g1=0.1, g2=0.2).shift(0.3, -0.1)
    prof = galsim.Transform(g, jac=[[0.5, 0.], [0., 0.5]], offset=(0.2, 0.1), flux_ratio=3.)
    rec = xleaf_records(prof, 1)[0, 0]
    m = galsim.Shear(g1=0.1, g2=0.2).getMatrix()
    assert np.allclose(rec['jac'].reshape(2, 2), 0.5 * m, rtol=1e-15, atol=0)
    assert np.allclose([rec['xoff'], rec['yoff']], [0.2 + 0.5 * 0.3, 0.1 - 0.5 * 0.1], rtol=1e-15)
    assert np.isclose(rec['flux_ratio'], 3. * 0.25, rtol=1e-15)
    assert rec['flags'] == galsim._lib.XLEAF_JAC and rec['flux'] == 2. and rec['p'][0] == 0.5

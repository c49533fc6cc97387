"""Wavelength integration rules and image integrators for chromatic drawing
(galsim/integ.py:118-330).

The rules turn the integration wavelengths and the bandpass throughput into per-wavelength
weights exactly as the reference's do.  The integrators differ from the reference's in how
the integrand images are made: instead of drawing one monochromatic image per wavelength in
turn and summing them on the host, the monochromatic profiles at all wavelengths form ONE
batched profile, drawn in one pass of the batched engine (each wavelength with its own FFT
size, as the reference sizes each drawImage call, or in real space where the reference draws
in real space), and the weighted sum of the stamps is taken on the device
(gsb_weighted_stamp_sum).
"""
import numpy as np

from .errors import GalSimValueError

__all__ = ['MidptRule', 'TrapzRule', 'QuadRule', 'midptRule', 'trapzRule', 'quadRule',
           'SampleIntegrator', 'ContinuousIntegrator']


class IntegrationRule(object):
    """integ.py:118-146: weights g_i such that sum_i g_i f(x_i) approximates int f w dx."""

    def calculateWeights(self, xs, w):
        raise NotImplementedError

    def __call__(self, f, xs, w=None):
        gs = self.calculateWeights(xs, w)
        return sum(g * f(x) for g, x in zip(gs, xs))


class MidptRule(IntegrationRule):
    """integ.py:148-170."""

    def calculateWeights(self, xs, w):
        if len(xs) < 2:
            raise GalSimValueError("Not enough points for midptRule integration", xs)
        xs = np.asarray(xs, dtype=float)
        gs = np.empty_like(xs)
        gs[0] = (xs[1] - xs[0])
        gs[1:-1] = 0.5 * (xs[2:] - xs[:-2])
        gs[-1] = (xs[-1] - xs[-2])
        if w is not None:
            gs *= w(xs)
        return gs


class TrapzRule(IntegrationRule):
    """integ.py:172-194."""

    def calculateWeights(self, xs, w):
        if len(xs) < 2:
            raise GalSimValueError("Not enough points for trapzRule integration", xs)
        xs = np.asarray(xs, dtype=float)
        gs = np.empty_like(xs)
        gs[0] = 0.5 * (xs[1] - xs[0])
        gs[1:-1] = 0.5 * (xs[2:] - xs[:-2])
        gs[-1] = 0.5 * (xs[-1] - xs[-2])
        if w is not None:
            gs *= w(xs)
        return gs


class QuadRule(IntegrationRule):
    """integ.py:196-225: f and w both linear between the points, so the product is quadratic."""

    def calculateWeights(self, xs, w):
        if len(xs) < 2:
            raise GalSimValueError("Not enough points for quadRule integration", xs)
        if w is None:
            return TrapzRule().calculateWeights(xs, w)
        xs = np.asarray(xs, dtype=float)
        ws = w(xs)
        gs = np.empty_like(xs)
        gs[0] = (xs[1] - xs[0]) * (2 * ws[0] + ws[1])
        gs[1:-1] = (xs[1:-1] - xs[:-2]) * (ws[:-2] + 2 * ws[1:-1])
        gs[1:-1] += (xs[2:] - xs[1:-1]) * (2 * ws[1:-1] + ws[2:])
        gs[-1] = (xs[-1] - xs[-2]) * (ws[-2] + 2 * ws[-1])
        gs /= 6.
        return gs


midptRule = MidptRule()
trapzRule = TrapzRule()
quadRule = QuadRule()


class ImageIntegrator(object):
    """integ.py:232-271, batched: see the module docstring."""

    def __call__(self, chromatic, bandpass, image, drawImageKwargs, doK=False):
        from .chromatic import _integrate_images, _integrate_kimages
        waves = np.asarray(self.calculateWaves(bandpass), dtype=float)
        self.last_n_eval = len(waves)
        drawImageKwargs.pop('add_to_image', None)
        gs = self.rule.calculateWeights(waves, bandpass)
        if doK:
            return _integrate_kimages(chromatic, waves, gs, image, drawImageKwargs)
        return _integrate_images(chromatic, waves, gs, image, drawImageKwargs)


class SampleIntegrator(ImageIntegrator):
    """Integrand at the bandpass's wave_list (integ.py:274-296)."""

    def __init__(self, rule):
        self.rule = rule

    def calculateWaves(self, bandpass):
        return bandpass.wave_list


class ContinuousIntegrator(ImageIntegrator):
    """Integrand at N equally spaced wavelengths (integ.py:299-330)."""

    def __init__(self, rule, N=250, use_endpoints=True):
        self.rule = rule
        self.N = N
        self.use_endpoints = use_endpoints

    def calculateWaves(self, bandpass):
        h = (bandpass.red_limit * 1.0 - bandpass.blue_limit) / self.N
        if self.use_endpoints:
            return [bandpass.blue_limit + h * i for i in range(self.N + 1)]
        return [bandpass.blue_limit + h * (i + 0.5) for i in range(self.N)]

"""GSParams: accuracy and size parameters (galsim/gsparams.py:31-260)."""
import copy

from .errors import GalSimIncompatibleValuesError


class GSParams(object):
    """Speed / accuracy trade-off parameters.  Same defaults, meaning and ``combine`` rule as
    the reference (galsim/gsparams.py:127-158, 217-240)."""

    def __init__(self, minimum_fft_size=128, maximum_fft_size=8192,
                 folding_threshold=5.e-3, stepk_minimum_hlr=5, maxk_threshold=1.e-3,
                 kvalue_accuracy=1.e-5, xvalue_accuracy=1.e-5, table_spacing=1,
                 realspace_relerr=1.e-4, realspace_abserr=1.e-6,
                 integration_relerr=1.e-6, integration_abserr=1.e-8,
                 shoot_accuracy=1.e-5):
        self._minimum_fft_size = int(minimum_fft_size)
        self._maximum_fft_size = int(maximum_fft_size)
        self._folding_threshold = float(folding_threshold)
        self._stepk_minimum_hlr = float(stepk_minimum_hlr)
        self._maxk_threshold = float(maxk_threshold)
        self._kvalue_accuracy = float(kvalue_accuracy)
        self._xvalue_accuracy = float(xvalue_accuracy)
        self._table_spacing = float(table_spacing)
        self._realspace_relerr = float(realspace_relerr)
        self._realspace_abserr = float(realspace_abserr)
        self._integration_relerr = float(integration_relerr)
        self._integration_abserr = float(integration_abserr)
        self._shoot_accuracy = float(shoot_accuracy)

    minimum_fft_size = property(lambda self: self._minimum_fft_size)
    maximum_fft_size = property(lambda self: self._maximum_fft_size)
    folding_threshold = property(lambda self: self._folding_threshold)
    stepk_minimum_hlr = property(lambda self: self._stepk_minimum_hlr)
    maxk_threshold = property(lambda self: self._maxk_threshold)
    kvalue_accuracy = property(lambda self: self._kvalue_accuracy)
    xvalue_accuracy = property(lambda self: self._xvalue_accuracy)
    table_spacing = property(lambda self: self._table_spacing)
    realspace_relerr = property(lambda self: self._realspace_relerr)
    realspace_abserr = property(lambda self: self._realspace_abserr)
    integration_relerr = property(lambda self: self._integration_relerr)
    integration_abserr = property(lambda self: self._integration_abserr)
    shoot_accuracy = property(lambda self: self._shoot_accuracy)

    @staticmethod
    def check(gsparams, default=None, **kwargs):
        if gsparams is None:
            gsparams = default if default is not None else GSParams.default
        elif not isinstance(gsparams, GSParams):
            raise TypeError("Invalid GSParams: %s" % gsparams)
        return gsparams.withParams(**kwargs)

    def withParams(self, **kwargs):
        if len(kwargs) == 0:
            return self
        ret = copy.copy(self)
        for k in kwargs:
            if not hasattr(ret, '_' + k):
                raise TypeError('parameter %s is invalid' % k)
            setattr(ret, '_' + k, kwargs[k])
        return ret

    @staticmethod
    def combine(gsp_list):
        """The most restrictive combination of a list of GSParams (gsparams.py:217-240)."""
        if len(gsp_list) == 1:
            return gsp_list[0]
        elif all(g == gsp_list[0] for g in gsp_list[1:]):
            return gsp_list[0]
        gl = [g for g in gsp_list if g is not None]
        return GSParams(
            max(g.minimum_fft_size for g in gl), max(g.maximum_fft_size for g in gl),
            min(g.folding_threshold for g in gl), max(g.stepk_minimum_hlr for g in gl),
            min(g.maxk_threshold for g in gl), min(g.kvalue_accuracy for g in gl),
            min(g.xvalue_accuracy for g in gl), min(g.table_spacing for g in gl),
            min(g.realspace_relerr for g in gl), min(g.realspace_abserr for g in gl),
            min(g.integration_relerr for g in gl), min(g.integration_abserr for g in gl),
            min(g.shoot_accuracy for g in gl))

    def _getinitargs(self):
        return (self.minimum_fft_size, self.maximum_fft_size,
                self.folding_threshold, self.stepk_minimum_hlr, self.maxk_threshold,
                self.kvalue_accuracy, self.xvalue_accuracy, self.table_spacing,
                self.realspace_relerr, self.realspace_abserr,
                self.integration_relerr, self.integration_abserr, self.shoot_accuracy)

    def __getstate__(self):
        return self._getinitargs()

    def __setstate__(self, state):
        self.__init__(*state)

    def __repr__(self):
        return 'galsim.GSParams(%d,%d,%r,%r,%r,%r,%r,%r,%r,%r,%r,%r,%r)' % self._getinitargs()

    def __eq__(self, other):
        return self is other or (isinstance(other, GSParams) and
                                 self._getinitargs() == other._getinitargs())

    def __ne__(self, other):
        return not self.__eq__(other)

    def __hash__(self):
        return hash(('galsim.GSParams', self._getinitargs()))


GSParams.default = GSParams()

__all__ = ['GSParams']

"""Exception and warning classes with the reference's names and meaning
(galsim/errors.py:142-448)."""
import warnings


class GalSimError(RuntimeError):
    """Base class for GalSim-specific run-time errors (galsim/errors.py:142)."""


class GalSimValueError(GalSimError, ValueError):
    def __init__(self, message, value, allowed_values=None):
        self.message = message
        self.value = value
        self.allowed_values = allowed_values
        s = message + " Value {0!s}".format(value)
        if allowed_values is not None:
            s += " not in {0!s}".format(allowed_values)
        super(GalSimValueError, self).__init__(s)


class GalSimKeyError(GalSimError, KeyError):
    pass


class GalSimIndexError(GalSimError, IndexError):
    pass


class GalSimRangeError(GalSimError, ValueError):
    def __init__(self, message, value, min, max=None):
        self.message = message
        self.value = value
        self.min = min
        self.max = max
        super(GalSimRangeError, self).__init__(
            "{0} Value {1!s} not in range [{2!s}, {3!s}]".format(message, value, min, max))


class GalSimBoundsError(GalSimError, ValueError):
    def __init__(self, message, pos, bounds):
        self.message = message
        self.pos = pos
        self.bounds = bounds
        super(GalSimBoundsError, self).__init__(
            "{0} {1!s} not in {2!s}".format(message, pos, bounds))


class GalSimUndefinedBoundsError(GalSimError):
    pass


class GalSimImmutableError(GalSimError):
    def __init__(self, message, image):
        self.image = image
        super(GalSimImmutableError, self).__init__(message)


class GalSimIncompatibleValuesError(GalSimError, ValueError, TypeError):
    def __init__(self, message, values={}, **kwargs):
        self.message = message
        self.values = dict(values, **kwargs)
        super(GalSimIncompatibleValuesError, self).__init__(
            message + " Values {0!s}".format(self.values))


class GalSimSEDError(GalSimError, TypeError):
    pass


class GalSimHSMError(GalSimError):
    pass


class GalSimFFTSizeError(GalSimError):
    """An FFT larger than maximum_fft_size was requested (galsim/errors.py:339-359)."""
    def __init__(self, message, size):
        self.message = message
        self.size = size
        self.mem = size * size * 24. / 1024. ** 3
        super(GalSimFFTSizeError, self).__init__(
            message + "\nThe required FFT size would be {0} x {0}, which requires "
            "{1:.2f} GB of memory.\nIf you can handle the large FFT, you may update "
            "gsparams.maximum_fft_size.".format(size, self.mem))


class GalSimConfigError(GalSimError, ValueError):
    pass


class GalSimConfigValueError(GalSimValueError, GalSimConfigError):
    pass


class GalSimNotImplementedError(GalSimError, NotImplementedError):
    pass


class GalSimWarning(UserWarning):
    pass


class GalSimFFTSizeWarning(GalSimWarning):
    pass


class GalSimDeprecationWarning(GalSimWarning):
    pass


#: When True, an oversized FFT raises GalSimFFTSizeError instead of warning
#: (galsim/errors.py:36).
raise_fft_size_error = False


def galsim_warn(message):
    warnings.warn(message, GalSimWarning)


def galsim_warn_fft(message, size):
    """Warn (or raise, if raise_fft_size_error) about a very large FFT (errors.py:437-441)."""
    if raise_fft_size_error:
        raise GalSimFFTSizeError(message, size)
    mem = size * size * 24. / 1024. ** 3
    warnings.warn(message + " The required FFT size would be {0} x {0}, which requires "
                  "{1:.2f} GB of memory.".format(size, mem), GalSimFFTSizeWarning)


class GSBLibraryError(GalSimError):
    """A call into libgsb failed; carries the library's status code."""
    def __init__(self, code, message):
        self.code = code
        super(GSBLibraryError, self).__init__("libgsb error %d: %s" % (code, message))


__all__ = [n for n in dir() if n.startswith('GalSim') or n in ('galsim_warn', 'galsim_warn_fft',
                                                                    'GSBLibraryError')]

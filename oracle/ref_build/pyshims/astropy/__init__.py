"""ORACLE-ONLY import shim for astropy (not installed here).

The reference GalSim package imports astropy.units / astropy.constants at module load
(galsim/sed.py, bandpass.py, airy.py, kolmogorov.py ...).  Nothing on the FFT drawing path
uses a Quantity; the shim only needs module-level unit arithmetic to evaluate and
``isinstance(x, units.Quantity)`` to be False for plain floats.
"""
from . import units, constants  # noqa: F401

"""ORACLE-ONLY shim: astropy.wcs is not used on the FFT drawing path."""
from ._inert import Inert


def __getattr__(name):
    return Inert()

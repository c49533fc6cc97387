"""ORACLE-ONLY shim: FITS I/O is not used on the FFT drawing path."""
from .._inert import Inert


def __getattr__(name):
    return Inert()

"""ORACLE-ONLY shim: see astropy/__init__.py."""
from ._inert import Inert


def __getattr__(name):
    return Inert()

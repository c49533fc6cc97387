"""ORACLE-ONLY shim: see astropy/__init__.py."""
from . import fits  # noqa: F401

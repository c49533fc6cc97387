"""ORACLE-ONLY: import the reference GalSim Python package from its checkout.

The reference package (``galsim/`` under the reference checkout) is loaded unmodified from
its own directory; its compiled extension ``_galsim`` comes from ``oracle/_ref`` (built by
``make -C oracle ref`` from the reference C++ sources), and the two absent third-party
dependencies (LSSTDESC.Coord, astropy) are served by the inert shims in
``oracle/ref_build/pyshims``.  Used only by ``tests/golden/make_golden.py`` and by tests
that validate the oracle restatement; nothing in the product imports it.
"""
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, '_ref')
SHIMS = os.path.join(HERE, 'ref_build', 'pyshims')


def reference_available(ref_root):
    return (os.path.isdir(os.path.join(ref_root, 'galsim')) and
            any(f.startswith('_galsim') and f.endswith('.so') for f in os.listdir(REF_OUT))
            if os.path.isdir(REF_OUT) else False)


def import_reference_galsim(ref_root):
    """Return the reference ``galsim`` module, importing it on first use."""
    if 'galsim' in sys.modules:
        return sys.modules['galsim']
    if SHIMS not in sys.path:
        sys.path.insert(0, SHIMS)
    pkg_dir = os.path.join(ref_root, 'galsim')
    spec = importlib.util.spec_from_file_location(
        'galsim', os.path.join(pkg_dir, '__init__.py'),
        submodule_search_locations=[pkg_dir, REF_OUT])
    mod = importlib.util.module_from_spec(spec)
    sys.modules['galsim'] = mod
    # galsim.hsm builds its C++ parameter object at import time, and the HSM C++ needs
    # Eigen, which is absent; shape measurement is not on the drawing path, so the
    # submodule is replaced by an empty placeholder.
    import types
    sys.modules['galsim.hsm'] = types.ModuleType('galsim.hsm')
    spec.loader.exec_module(mod)
    return mod

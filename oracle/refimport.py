"""
Import the reference ``macromax`` package: for fixture generation (tests/golden/make_golden.py), the tests that run
the reference's own API and test suite on this library, and the CPU baseline of bench.py.  Test infrastructure.

The reference package writes a log file next to itself on import (``macromax/__init__.py:61-67``) and needs
``coloredlogs`` and installed package metadata, neither of which exists here.  So this helper copies the package to
a temporary directory, puts a minimal ``coloredlogs`` stand-in on ``sys.path`` and answers the version lookup.
The package is looked up in ``$MACROMAX_REFERENCE`` (a directory holding ``macromax/``) and otherwise in the
repository's ``baseline/_ref`` (the reference package placed there for the reference arm; not part of the
repository's history).  Where neither exists, ``reference_available()`` is False and the tests that need it skip.
"""
from __future__ import annotations

import importlib
import importlib.metadata
import os
import shutil
import sys
import tempfile

_REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE_PYTHON = os.environ.get('MACROMAX_REFERENCE', os.path.join(_REPO, 'baseline', '_ref'))

_STUB = '''
import logging
DEFAULT_FIELD_STYLES = {'asctime': {}}
DEFAULT_LEVEL_STYLES = {}
def enable_ansi_support():
    pass
class ColoredFormatter(logging.Formatter):
    def __init__(self, fmt=None, datefmt=None, field_styles=None, level_styles=None):
        super().__init__(fmt)
'''


def reference_available() -> bool:
    return os.path.isdir(os.path.join(REFERENCE_PYTHON, 'macromax'))


def import_reference():
    """Return the reference ``macromax`` module, imported from a private copy."""
    if 'macromax' in sys.modules and getattr(sys.modules['macromax'], '_graft_reference_copy', False):
        return sys.modules['macromax']
    if not reference_available():
        raise ImportError(f'reference package not found under {REFERENCE_PYTHON}')
    tmp = tempfile.mkdtemp(prefix='macromax_ref_')
    shutil.copytree(os.path.join(REFERENCE_PYTHON, 'macromax'), os.path.join(tmp, 'macromax'))
    stubs = os.path.join(tmp, '_stubs')
    os.makedirs(stubs)
    with open(os.path.join(stubs, 'coloredlogs.py'), 'w') as f:
        f.write(_STUB)
    sys.path.insert(0, stubs)
    sys.path.insert(0, tmp)
    original_version = importlib.metadata.version

    def version(name):
        if name == 'macromax':
            return '0+reference'
        return original_version(name)

    importlib.metadata.version = version
    mm = importlib.import_module('macromax')
    mm._graft_reference_copy = True
    import logging
    mm.log.setLevel(logging.ERROR)
    for h in list(mm.log.handlers):
        if isinstance(h, logging.FileHandler):
            mm.log.removeHandler(h)
    return mm


def reference_tests_dir() -> str | None:
    """The reference's own test directory (``tests/`` beside the package), or None where it is absent."""
    d = os.path.join(REFERENCE_PYTHON, 'tests')
    return d if os.path.isfile(os.path.join(d, 'test_backend.py')) else None


def load_reference_test_module(name: str):
    """Import one of the reference's test modules (e.g. ``test_backend``) against the imported reference copy."""
    import importlib.util
    d = reference_tests_dir()
    if d is None:
        raise ImportError('the reference test directory is not present')
    import_reference()
    spec = importlib.util.spec_from_file_location(f'_reference_tests_{name}', os.path.join(d, f'{name}.py'))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod

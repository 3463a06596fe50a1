"""
Locate an installed copy of the reference package (difffea) for the drop-in tests.

The reference is a pure-Python package.  The repository's tooling installs it under ``baseline/_ref`` (a
directory kept out of version control); a difffea already importable in the environment also counts.  The
tests that need it skip, with this reason, where neither is present.
"""
import importlib
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INSTALL = os.path.join(ROOT, "baseline", "_ref")
MISSING = ("the reference package difffea is not installed (expected under baseline/_ref, installed by "
           "`pip install --no-deps --target baseline/_ref <reference checkout>`)")


def load():
    """The imported difffea package, or None."""
    if os.path.isdir(os.path.join(INSTALL, "difffea")) and INSTALL not in sys.path:
        sys.path.append(INSTALL)
    try:
        pkg = importlib.import_module("difffea")
        importlib.import_module("difffea.operators")
        importlib.import_module("difffea.newton_krylov")
        importlib.import_module("difffea.problem")
        return pkg
    except ImportError:
        return None

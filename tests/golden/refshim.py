"""Import the reference's Python modules on a CPU-only machine, unchanged.

Golden-vector harness: used by ``make_golden.py`` and by tests that compare
with the reference's own definitions (each skips itself when the reference is
absent).  Nothing on the GPU path imports it.

The stand-ins themselves live in ``baseline/refshim.py``: ``cupy`` becomes
numpy, and ``cupy.RawKernel`` compiles the reference's OWN kernel string
(physics.py:43-276, read from the imported module at run time, never copied)
as host C++ with g++ (``-ffp-contract=off``), run over the grid of blocks with
OpenMP; matplotlib becomes inert stubs.

Where the reference comes from: ``$AMHD_REFERENCE_DIR``, else the installed
copy in ``baseline/_ref`` (``python baseline/install_reference.py --source
<checkout>``).  ``REFERENCE_DIR`` is None when neither holds it.
"""
from __future__ import annotations

import importlib.util
import os
import sys

_PATH = os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))), "baseline",
                     "refshim.py")
_spec = importlib.util.spec_from_file_location("amhd_baseline_refshim", _PATH)
_shim = sys.modules.get("amhd_baseline_refshim")
if _shim is None:
    _shim = importlib.util.module_from_spec(_spec)
    sys.modules["amhd_baseline_refshim"] = _shim
    _spec.loader.exec_module(_shim)

try:
    REFERENCE_DIR = _shim.reference_dir()
except FileNotFoundError:
    REFERENCE_DIR = None


def load_reference():
    """Return the reference modules (config, physics, solver, main) over the numpy stand-in."""
    return _shim.load_reference("numpy")

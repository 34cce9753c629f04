"""`import zebsdsolve` for code written against the reference's Python package: put this
directory's parent (zebsdsolve_b200/compat) on PYTHONPATH and `zebsdsolve` resolves to
zebsdsolve_b200 — the same names (index, Solver, Result, Error, fit_pattern_center, fit_plane,
load_patterns, __version__) with the same meaning, on this package's CUDA kernels."""
import os as _os
import sys as _sys

_root = _os.path.dirname(_os.path.dirname(_os.path.dirname(_os.path.dirname(_os.path.abspath(__file__)))))
if _root not in _sys.path:
    _sys.path.insert(0, _root)

import zebsdsolve_b200 as _impl  # noqa: E402
from zebsdsolve_b200 import *  # noqa: E402,F401,F403
from zebsdsolve_b200 import Error, Result, Solver, __version__, api, fit_pattern_center, fit_plane, index  # noqa: E402,F401
from zebsdsolve_b200 import load_patterns  # noqa: E402,F401

_sys.modules.setdefault("zebsdsolve.api", api)

"""Import the reference pyFANTOM CPU path in this container, for golden-vector generation only.

The reference imports a few third-party modules that are absent here and play no part in
the numeric path.  They are stood in for before import:

* ``sksparse.cholmod`` (CHOLMOD): ``cholesky(K, beta)`` returns a factor of ``K + beta*I``
  built with ``scipy.sparse.linalg.splu``; ``factor(b)`` solves and
  ``factor.cholesky_inplace(K, beta)`` refactors;
* ``matplotlib``, ``vtk``, ``k3d`` (plotting only): ``MagicMock`` modules.

``NUMBA_CACHE_DIR`` is pointed at a writable directory because the reference tree is
read-only.  Nothing in the library or in the GPU tests uses this module.
"""
from __future__ import annotations

import os
import sys
import types
from unittest.mock import MagicMock



def reference_root() -> str:
    """The reference checkout to import (environment variable ``PYFANTOM_REFERENCE``)."""
    root = os.environ.get("PYFANTOM_REFERENCE")
    if not root:
        raise RuntimeError("set PYFANTOM_REFERENCE to the reference pyFANTOM checkout to generate goldens")
    return root


def install():
    if "pyFANTOM" in sys.modules:
        return
    import tempfile
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "pyfantom_ref_numba_cache"))
    import scipy.sparse as sp
    from scipy.sparse.linalg import splu

    class _Factor:
        def __init__(self, K, beta):
            self._lu = splu((sp.csc_matrix(K) + beta * sp.eye(K.shape[0], format="csc")).tocsc())

        def __call__(self, b):
            return self._lu.solve(b)

        def cholesky_inplace(self, K, beta=0.0):
            self.__init__(K, beta)

    sksparse = types.ModuleType("sksparse")
    cholmod = types.ModuleType("sksparse.cholmod")
    cholmod.cholesky = lambda K, beta=0.0, **kw: _Factor(K, beta)
    sksparse.cholmod = cholmod
    sys.modules["sksparse"] = sksparse
    sys.modules["sksparse.cholmod"] = cholmod
    for name in ["matplotlib", "matplotlib.pyplot", "matplotlib.markers", "matplotlib.path",
                 "matplotlib.collections", "matplotlib.colors", "vtk", "k3d"]:
        sys.modules.setdefault(name, MagicMock())
    root = reference_root()
    if root not in sys.path:
        sys.path.insert(0, root)

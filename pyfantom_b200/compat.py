"""The library under the reference's own import paths.

    import pyfantom_b200.compat
    pyfantom_b200.compat.install()
    from pyFANTOM.CUDA import StructuredMesh3D, FiniteElement, MinimumCompliance, OC
    from pyFANTOM.solvers.CUDA._solvers import MultiGrid

``install()`` registers module objects for the paths a pyFANTOM CUDA script imports
(``pyFANTOM.CUDA`` and its ``Kernels``/``Mesh``/``Filters``/``Solvers``/``Problems``/
``Optimizers``/``FiniteElement`` parts, ``pyFANTOM.stiffness.CUDA``,
``pyFANTOM.solvers.CUDA._solvers``, ``pyFANTOM.geom.CUDA``,
``pyFANTOM.FiniteElement.CUDA.FiniteElement``, ``pyFANTOM.Problem.CUDA.MinimumCompliance``,
``pyFANTOM.Optimizers.CUDA.OC`` / ``.PGD`` and ``pyFANTOM.physics.LinearElasticity``), each
holding this library's classes under the reference's names, so such a script runs
unchanged.  Only the structured-mesh path exists here: other reference names (general
meshes, MMA, CPU backends, visualisers) are absent and importing them fails.  Nothing is
registered until ``install()`` is called, and it refuses to shadow a real pyFANTOM that is
already imported.  ``uninstall()`` removes the aliases.
"""
from __future__ import annotations

import sys
import types

_MARK = "__pyfantom_b200_alias__"


def _table():
    from . import FiniteElement as fe_mod
    from . import Optimizers as opt_mod
    from . import Problem as prob_mod
    from . import geom, physics, solvers, stiffness
    geom_cuda = {"CuStructuredFilter2D": geom.CuStructuredFilter2D, "CuStructuredFilter3D": geom.CuStructuredFilter3D,
                 "StructuredMesh2D": geom.CuStructuredMesh2D, "StructuredMesh3D": geom.CuStructuredMesh3D,
                 "CuStructuredMesh2D": geom.CuStructuredMesh2D, "CuStructuredMesh3D": geom.CuStructuredMesh3D}
    kernels = {"StructuredStiffnessKernel": stiffness.StructuredStiffnessKernel}
    solv = {"CG": solvers.CG, "SPSOLVE": solvers.SPSOLVE, "MultiGrid": solvers.MultiGrid, "Solver": solvers.Solver}
    fem = {"FiniteElement": fe_mod.FiniteElement}
    prob = {"MinimumCompliance": prob_mod.MinimumCompliance}
    mesh = {"StructuredMesh2D": geom.CuStructuredMesh2D, "StructuredMesh3D": geom.CuStructuredMesh3D}
    filt = {"StructuredFilter2D": geom.CuStructuredFilter2D, "StructuredFilter3D": geom.CuStructuredFilter3D}
    opts = {"OC": opt_mod.OC, "PGD": opt_mod.PGD}
    facade = {**kernels, **mesh, **filt, **solv, **fem, **prob, **opts}
    return {
        "pyFANTOM": {},
        "pyFANTOM.CUDA": facade,
        "pyFANTOM.CUDA.Kernels": kernels,
        "pyFANTOM.CUDA.Mesh": mesh,
        "pyFANTOM.CUDA.Filters": filt,
        "pyFANTOM.CUDA.Solvers": solv,
        "pyFANTOM.CUDA.Problems": prob,
        "pyFANTOM.CUDA.Optimizers": opts,
        "pyFANTOM.CUDA.FiniteElement": fem,
        "pyFANTOM.stiffness": {},
        "pyFANTOM.stiffness.CUDA": kernels,
        "pyFANTOM.stiffness.CUDA._FEA": kernels,
        "pyFANTOM.solvers": {},
        "pyFANTOM.solvers.CUDA": solv,
        "pyFANTOM.solvers.CUDA._solvers": solv,
        "pyFANTOM.geom": {},
        "pyFANTOM.geom.CUDA": geom_cuda,
        "pyFANTOM.geom.CUDA._mesh": {"CuStructuredMesh2D": geom.CuStructuredMesh2D,
                                     "CuStructuredMesh3D": geom.CuStructuredMesh3D},
        "pyFANTOM.geom.CUDA._filters": {"CuStructuredFilter2D": geom.CuStructuredFilter2D,
                                        "CuStructuredFilter3D": geom.CuStructuredFilter3D},
        "pyFANTOM.FiniteElement": {},
        "pyFANTOM.FiniteElement.CUDA": fem,
        "pyFANTOM.FiniteElement.CUDA.FiniteElement": fem,
        "pyFANTOM.Problem": {},
        "pyFANTOM.Problem.CUDA": prob,
        "pyFANTOM.Problem.CUDA.MinimumCompliance": prob,
        "pyFANTOM.Optimizers": {},
        "pyFANTOM.Optimizers.CUDA": opts,
        "pyFANTOM.Optimizers.CUDA.OC": {"OC": opt_mod.OC},
        "pyFANTOM.Optimizers.CUDA.PGD": {"PGD": opt_mod.PGD},
        "pyFANTOM.physics": {},
        "pyFANTOM.physics.LinearElasticity": {"LinearElasticity": physics.LinearElasticity},
    }


def install() -> None:
    """Register the aliases (idempotent).  RuntimeError if a real pyFANTOM is imported."""
    top = sys.modules.get("pyFANTOM")
    if top is not None and not getattr(top, _MARK, False):
        raise RuntimeError("a pyFANTOM package is already imported; the aliases would shadow it")
    table = _table()
    mods = {}
    for name, attrs in table.items():
        m = sys.modules.get(name)
        if m is None or not getattr(m, _MARK, False):
            m = types.ModuleType(name, f"pyfantom_b200 under the reference path {name}")
            setattr(m, _MARK, True)
            m.__path__ = []  # a package, so that submodules resolve
            sys.modules[name] = m
        for k, v in attrs.items():
            setattr(m, k, v)
        mods[name] = m
    for name, m in mods.items():  # parent.child attributes; a class of the same name wins, as
        parent, _, child = name.rpartition(".")  # after the reference's `from .X import *`
        if parent in mods and child not in table[parent]:
            setattr(mods[parent], child, m)


def uninstall() -> None:
    """Remove every alias module registered by install()."""
    for name in [n for n, m in sys.modules.items() if n == "pyFANTOM" or n.startswith("pyFANTOM.")]:
        if getattr(sys.modules[name], _MARK, False):
            del sys.modules[name]

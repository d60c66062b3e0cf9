"""Facade with the documented names of the reference CUDA backend
(``from pyFANTOM.CUDA import ...``, docs/source/examples/2d_topology_optimization.rst:208-216).

    from pyfantom_b200.CUDA import (StructuredMesh3D, StructuredStiffnessKernel, MultiGrid,
                                    FiniteElement, StructuredFilter3D, MinimumCompliance, OC)
"""
from .geom import CuStructuredFilter2D as StructuredFilter2D  # noqa: F401
from .geom import CuStructuredFilter3D as StructuredFilter3D  # noqa: F401
from .geom import CuStructuredMesh2D as StructuredMesh2D  # noqa: F401
from .geom import CuStructuredMesh3D as StructuredMesh3D  # noqa: F401
from .stiffness import StructuredStiffnessKernel  # noqa: F401
from .solvers import CG, SPSOLVE, MultiGrid  # noqa: F401
from .FiniteElement import FiniteElement  # noqa: F401
from .Problem import MinimumCompliance  # noqa: F401
from .Optimizers import OC, PGD  # noqa: F401
from .physics import LinearElasticity  # noqa: F401

__all__ = ["StructuredMesh2D", "StructuredMesh3D", "StructuredFilter2D", "StructuredFilter3D",
           "StructuredStiffnessKernel", "CG", "SPSOLVE", "MultiGrid", "FiniteElement", "MinimumCompliance", "OC", "PGD",
           "LinearElasticity"]

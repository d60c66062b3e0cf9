"""CPU: the library under the reference's import paths (pyfantom_b200.compat)."""
import sys

import pytest


def test_reference_import_paths_resolve_to_the_library():
    from pyfantom_b200 import compat, geom, solvers, stiffness
    from pyfantom_b200.Optimizers import OC
    compat.install()
    try:
        from pyFANTOM.CUDA import FiniteElement, MinimumCompliance, MultiGrid, StructuredMesh3D  # noqa: F401
        from pyFANTOM.geom.CUDA import CuStructuredFilter3D, StructuredMesh2D
        from pyFANTOM.Optimizers.CUDA.OC import OC as OC2
        from pyFANTOM.solvers.CUDA._solvers import MultiGrid as MG2
        from pyFANTOM.stiffness.CUDA import StructuredStiffnessKernel
        import pyFANTOM.CUDA.Kernels as K
        assert StructuredStiffnessKernel is stiffness.StructuredStiffnessKernel is K.StructuredStiffnessKernel
        assert MultiGrid is MG2 is solvers.MultiGrid
        assert StructuredMesh3D is geom.CuStructuredMesh3D and StructuredMesh2D is geom.CuStructuredMesh2D
        assert CuStructuredFilter3D is geom.CuStructuredFilter3D
        assert OC2 is OC
        from pyfantom_b200.FiniteElement import FiniteElement as FE
        from pyfantom_b200.Problem import MinimumCompliance as MC
        from pyFANTOM.FiniteElement.CUDA.FiniteElement import FiniteElement as FE2
        assert FiniteElement is FE is FE2 and MinimumCompliance is MC
        compat.install()  # idempotent
        with pytest.raises(ImportError):
            from pyFANTOM.CUDA import GeneralStiffnessKernel  # noqa: F401  (not on the structured path)
    finally:
        compat.uninstall()
    assert "pyFANTOM" not in sys.modules


def test_install_refuses_to_shadow_a_real_package():
    import types
    from pyfantom_b200 import compat
    sys.modules["pyFANTOM"] = types.ModuleType("pyFANTOM")
    try:
        with pytest.raises(RuntimeError):
            compat.install()
    finally:
        del sys.modules["pyFANTOM"]

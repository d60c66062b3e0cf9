"""B200-native (sm_100a) structured SIMP / MGCG path with the object API of pyFANTOM's
CUDA backend.  Import the drop-in classes from ``pyfantom_b200.CUDA``.

Submodules: ``physics`` (host K0), ``geom`` (meshes, filters), ``stiffness``
(StructuredStiffnessKernel), ``solvers`` (CG, MultiGrid), ``FiniteElement``, ``Problem``
(MinimumCompliance), ``Optimizers`` (OC), ``workloads`` (synthetic benchmark problems).
The CUDA kernels live in ``libpyfantom_b200.so`` (C ABI: include/pyfantom_b200.h).
"""
__version__ = "0.1.0"

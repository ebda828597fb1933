"""B200-native explicit DG operator and SSP-RK3 time integrator for the 3D compressible Euler
equations on affine tetrahedra: a drop-in for the explicit convection path of FVE_DG
(ExplicitConvection, include/DG/DG_Schemes/ExplicitConvection.h:9-45).

The compute path is libfvedg_b200.so (hand-written sm_100a CUDA kernels behind the C ABI of
include/dg_gpu.h). This package is the host-side mirror of the reference interface."""
from .convection import Ensemble, ExplicitConvection, launch_count  # noqa: F401
from .mesh import Mesh, box_mesh  # noqa: F401
from . import problems  # noqa: F401
from ._lib import DGError, LIB_PATH  # noqa: F401

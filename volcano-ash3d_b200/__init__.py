"""volcano-ash3d_b200: Ash3d's per-time-step transport path on NVIDIA B200.

The CUDA library (``libash3d_b200.so``, sources in ``csrc/``, C-ABI in
``include/ash3d_b200.h``) keeps the concentration field resident on the GPU
and implements the reference routines AdvectHorz/advect_x/advect_y,
AdvectVert/advect_z, DiffuseHorz/DiffuseVert (explicit and Crank-Nicolson),
Set_BC, Adjust_DT and the TimeStepTotals mass sums.

Python modules:
  ``_lib``       ctypes binding of the C-ABI (fails loudly if not built)
  ``model``      ``Ash3dGPU``: the reference routine names over the C-ABI
  ``driver``     the Ash3d.F90 time loop for the transport path
  ``synthetic``  grids, geometry, met steps and source for the named workloads
  ``build``      the nvcc recipe (sm_100a)
"""
from . import adjoint, driver, ensemble, synthetic  # noqa: F401
from ._lib import A3GError  # noqa: F401


def Ash3dGPU(*args, **kwargs):
    """Constructs the GPU model (imports the ctypes layer lazily)."""
    from .model import Ash3dGPU as _M
    return _M(*args, **kwargs)

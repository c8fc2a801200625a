"""viVlasov1D's implicit variational time step on B200 (sm_100a).

The compute path is libvv.so (hand-written CUDA kernels behind a C ABI,
include/vv.h); this package is the host-side mirror of the reference's
solver-class interface.  Importing it does not touch the GPU.
"""
from .config import Config  # noqa: F401
from .solver import (Grid, PETScPoissonSolver, PETScVlasovSolver,  # noqa: F401
                     TensorProductPreconditioner, Toolbox)

__all__ = ["Config", "Grid", "PETScVlasovSolver", "PETScPoissonSolver",
           "TensorProductPreconditioner", "Toolbox"]

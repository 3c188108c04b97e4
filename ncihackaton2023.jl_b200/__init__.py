"""B200 matrix-free sum-factorized Laplacian apply (hex Q_p), with device CG.

Host-side mirror of JordiManyer/NCIHackaton2023.jl's operator API
(src/NCIHackaton2023.jl:25-35) over the CUDA library libsfb200.so, whose C
ABI is declared in include/sfb200.h.

The directory name contains a dot, so the package is loaded by path and
registered as ``ncihackaton2023_b200`` (see ``load()`` in __graft_entry__.py).
"""
from . import fem
from ._lib import LIB_PATH, SumFacError
from .fem import (CartesianDiscreteModel, FESpace, Measure, Table, TrialFESpace,
                  cell_quantities)
from . import adjoint, batch, distributed, multigrid
from .multigrid import Multigrid
from .operator import (LazyMatrix, SumFactorizationMap, assemble_rhs, cg, get_dimensional_parameters,
                       mul, mul_multi, quadrature_points, rhs)

__all__ = [
    "CartesianDiscreteModel", "FESpace", "TrialFESpace", "Measure", "Table", "cell_quantities",
    "SumFactorizationMap", "get_dimensional_parameters", "LazyMatrix", "mul", "mul_multi", "cg",
    "assemble_rhs", "rhs", "quadrature_points", "SumFacError", "LIB_PATH", "fem", "adjoint",
    "batch", "distributed", "multigrid", "Multigrid",
]

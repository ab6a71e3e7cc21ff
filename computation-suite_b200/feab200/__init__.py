"""feab200: the hex8 linear-elastic assembly + Jacobi-PCG path of fea_engine on B200 GPUs.

Drop-in names (same meaning as in fea_engine): FESystem, Mesh, box_mesh, Material, D_solid3d,
Hex8Solid3D, Hex8SolidBbar, preconditioned_cg, jacobi_preconditioner, torch_sparse_cg_solve,
fesystem_solve_static_torch, the SIMP functions in ``topopt`` and the
strain / stress / von Mises / reaction recovery in ``recovery`` (FESystem.stress etc.).
All compute runs in libfeab200.so (hand-written sm_100a CUDA); importing the package fails if
that library is missing.
"""
from . import _lib  # noqa: F401  (loads libfeab200.so; raises ImportError if it is missing)
from .device import DeviceMesh, ReducedOperator, SolveInfo, pcg_solve
from .elements import Hex8Solid3D, Hex8SolidBbar
from .fields import FEField
from .material import D_solid3d, Material
from .mesh import Mesh, box_mesh
from .solver import FESystem
from .iterative_solvers import jacobi_preconditioner, preconditioned_cg
from .batched import ProblemBatch, solve_static_batched
from .torch_sparse_solver import fesystem_solve_static_torch, torch_sparse_cg_solve
from . import batched, cantilever, facet_loads, recovery, topopt, torch_sparse_solver  # noqa: F401

__all__ = ["FESystem", "Mesh", "box_mesh", "Material", "D_solid3d", "Hex8Solid3D", "Hex8SolidBbar", "FEField",
           "DeviceMesh",
           "ReducedOperator", "SolveInfo", "pcg_solve", "preconditioned_cg", "jacobi_preconditioner",
           "ProblemBatch", "solve_static_batched", "torch_sparse_cg_solve", "fesystem_solve_static_torch",
           "batched", "torch_sparse_solver", "cantilever", "facet_loads", "recovery", "topopt"]

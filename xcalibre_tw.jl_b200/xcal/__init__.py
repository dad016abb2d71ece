"""xcal: B200 implementation of XCALibre's SIMPLE/PISO hot path, behind the
reference's API names.  See api.py for the function-by-function mapping."""
from . import _abi, meshgen  # noqa: F401
from .api import (  # noqa: F401
    BicgstabSolver, CgSolver, Configuration, ConstantScalar, DILU, Dirichlet, Euler, GmresSolver,
    ILU0, Jacobi, KOmega, KWallFunction, LDL, Laminar, Linear, Midpoint, Neumann, NormDiagonal,
    NutWallFunction, OmegaWallFunction, Orthogonal, RANS, ScalarField, Server, Solver, Steady, Upwind,
    VectorField, assign, build_mesh, initialise, isturbulent, make_case, piso, set_runtime,
    set_schemes, set_solver, simple, update_mesh_format, write_vtk, model2vtk)
from .mesh import Mesh2  # noqa: F401

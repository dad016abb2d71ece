"""xcal: B200 implementation of XCALibre's SIMPLE/PISO hot path, behind the
reference's API names.  See api.py for the function-by-function mapping."""
import os

# The serving loop (Server) gives every worker its own stream, and each stream
# needs a hardware work queue of its own: with the driver's default of 8
# queues, shared round-robin, a worker's uploads wait behind another worker's
# whole run.  The driver reads this when the process creates its CUDA
# context, so it is set on import, before any CUDA call of this package (a
# value the caller has set is kept).
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from . import _abi, meshgen  # noqa: F401
from .api import (  # noqa: F401
    BicgstabSolver, CgSolver, Configuration, ConstantScalar, DILU, Dirichlet, Euler, GmresSolver,
    ILU0, Jacobi, KOmega, KWallFunction, LDL, Laminar, Linear, Midpoint, Neumann, NormDiagonal,
    NutWallFunction, OmegaWallFunction, Orthogonal, RANS, ScalarField, Server, Solver, Steady, Upwind,
    VectorField, assign, build_mesh, initialise, isturbulent, make_case, piso, set_runtime,
    set_schemes, set_solver, simple, update_mesh_format, write_vtk, model2vtk)
from .mesh import Mesh2  # noqa: F401

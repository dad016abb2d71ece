"""The benchmark configurations as ready-made cases (mesh, model, config, pref).

    cavity2d   lid-driven cavity 0.1 m, n x n quads, Re=100 (lid 1 m/s, nu=1e-3)
    bfs        laminar backward-facing step h=10 mm, 27 cells/h (47,385 cells),
               graded 1.05, jittered +-10% (seed 20240101), inlet 0.5 m/s, nu=1e-4
    cavity3d   unit cube n^3 hexahedra, lid y=1 at (1,0,0), nu=1e-3

Schemes and solvers follow the configurations: divergence Upwind, Laplacian
Linear, gradient Orthogonal, steady; U relax 0.7, p relax 0.3; p CG+DILU and U
BiCGSTAB+DILU with itmax 100, atol sqrt(eps), rtol 1e-3.
"""
import os
import tempfile

import numpy as np

from . import api as X
from . import meshgen
from .mesh import Mesh2

_CACHE = os.environ.get("XCAL_MESH_CACHE", os.path.join(tempfile.gettempdir(), "xcal_meshes"))


def _unv(name, writer, **kw):
    os.makedirs(_CACHE, exist_ok=True)
    key = "_".join(f"{k}{v}" for k, v in sorted(kw.items()))
    path = os.path.join(_CACHE, f"{name}_{key}.unv")
    if not os.path.exists(path):
        tmp = path + f".{os.getpid()}.tmp"
        writer(tmp, **kw)
        os.replace(tmp, path)
    return path


def solvers_for(model, p_solver=X.CgSolver, u_solver=X.BicgstabSolver, precon=X.DILU,
                relax_u=0.7, relax_p=0.3, itmax=100):
    return dict(
        U=X.set_solver(model.U, solver=u_solver, preconditioner=precon(), convergence=1e-7,
                       relax=relax_u, itmax=itmax),
        p=X.set_solver(model.p, solver=p_solver, preconditioner=precon(), convergence=1e-7,
                       relax=relax_p, itmax=itmax))


def cavity2d(n=40, iterations=1000, divergence=X.Upwind, gradient=X.Orthogonal, nu=1e-3, mesh=None, **kw):
    if mesh is None:
        mesh = X.build_mesh(_unv("cavity", meshgen.cavity_unv, n=n, L=0.1))
    model = X.RANS(X.Laminar, mesh=mesh, viscosity=X.ConstantScalar(nu))
    X.assign(model, "U", X.Dirichlet("inlet", [0.0, 0.0, 0.0]), X.Dirichlet("outlet", [0.0, 0.0, 0.0]),
             X.Dirichlet("bottom", [0.0, 0.0, 0.0]), X.Dirichlet("top", [1.0, 0.0, 0.0]))
    X.assign(model, "p", *[X.Neumann(b, 0.0) for b in ("inlet", "outlet", "bottom", "top")])
    schemes = dict(U=X.set_schemes(divergence=divergence, gradient=gradient),
                   p=X.set_schemes(divergence=divergence, gradient=gradient))
    config = X.Configuration(solvers=solvers_for(model, **kw), schemes=schemes,
                             runtime=X.set_runtime(iterations=iterations, write_interval=-1, time_step=1))
    X.initialise(model.U, [0.0, 0.0, 0.0])
    X.initialise(model.p, 0.0)
    return mesh, model, config, 0.0


def bfs(cells_per_h=27, iterations=2000, divergence=X.Upwind, gradient=X.Orthogonal, nu=1e-4, mesh=None, **kw):
    if mesh is None:
        mesh = X.build_mesh(_unv("bfs", meshgen.bfs_unv, cells_per_h=cells_per_h))
    model = X.RANS(X.Laminar, mesh=mesh, viscosity=X.ConstantScalar(nu))
    X.assign(model, "U", X.Dirichlet("inlet", [0.5, 0.0, 0.0]), X.Neumann("outlet", 0.0),
             X.Dirichlet("wall", [0.0, 0.0, 0.0]), X.Dirichlet("top", [0.0, 0.0, 0.0]))
    X.assign(model, "p", X.Neumann("inlet", 0.0), X.Dirichlet("outlet", 0.0), X.Neumann("wall", 0.0),
             X.Neumann("top", 0.0))
    schemes = dict(U=X.set_schemes(divergence=divergence, gradient=gradient),
                   p=X.set_schemes(divergence=divergence, gradient=gradient))
    config = X.Configuration(solvers=solvers_for(model, **kw), schemes=schemes,
                             runtime=X.set_runtime(iterations=iterations, write_interval=-1, time_step=1))
    X.initialise(model.U, [0.0, 0.0, 0.0])
    X.initialise(model.p, 0.0)
    return mesh, model, config, None


def cavity3d(n=128, iterations=500, **kw):
    m = meshgen.hex_cavity(n)
    mesh = Mesh2.from_dict(m)
    model = X.RANS(X.Laminar, mesh=mesh, viscosity=X.ConstantScalar(1e-3))
    walls = ("xmin", "xmax", "ymin", "zmin", "zmax")
    X.assign(model, "U", *[X.Dirichlet(w, [0.0, 0.0, 0.0]) for w in walls],
             X.Dirichlet("lid", [1.0, 0.0, 0.0]))
    X.assign(model, "p", *[X.Neumann(w, 0.0) for w in walls + ("lid",)])
    schemes = dict(U=X.set_schemes(divergence=X.Upwind), p=X.set_schemes(divergence=X.Upwind))
    config = X.Configuration(solvers=solvers_for(model, **kw), schemes=schemes,
                             runtime=X.set_runtime(iterations=iterations, write_interval=-1, time_step=1))
    X.initialise(model.U, [0.0, 0.0, 0.0])
    X.initialise(model.p, 0.0)
    return mesh, model, config, 0.0


def fields(model):
    n = model.mesh.ncells
    U = np.stack([model.U.x.values, model.U.y.values, model.U.z.values])
    return U.reshape(3, n).copy(), model.p.values.copy()


def flatplate(nx=600, ny=250, iterations=3000, wall_functions=False, mesh=None, **kw):
    """k-omega flat plate 1 m x 0.2 m, U = 10 m/s, nu = 1.5e-5, inlet k from 1 %
    intensity (0.015) and omega from a viscosity ratio of 10 (100); BCs as the
    reference's low-Re flat-plate case (omega wall function on the plate).  With
    wall_functions, k and nut also use their wall functions on the plate."""
    if mesh is None:
        mesh = X.build_mesh(_unv("flatplate", meshgen.flatplate_unv, nx=nx, ny=ny))
    model = X.RANS(X.KOmega, mesh=mesh, viscosity=X.ConstantScalar(1.5e-5))
    Uin, kin = 10.0, 1.5 * (0.01 * 10.0) ** 2
    win = kin / (10 * 1.5e-5)
    X.assign(model, "U", X.Dirichlet("inlet", [Uin, 0.0, 0.0]), X.Neumann("outlet", 0.0),
             X.Dirichlet("wall", [0.0, 0.0, 0.0]), X.Neumann("top", 0.0))
    X.assign(model, "p", X.Neumann("inlet", 0.0), X.Dirichlet("outlet", 0.0), X.Neumann("wall", 0.0),
             X.Neumann("top", 0.0))
    X.assign(model, "turbulence.k", X.Dirichlet("inlet", kin), X.Neumann("outlet", 0.0),
             X.KWallFunction("wall") if wall_functions else X.Dirichlet("wall", 0.0), X.Neumann("top", 0.0))
    X.assign(model, "turbulence.omega", X.Dirichlet("inlet", win), X.Neumann("outlet", 0.0),
             X.OmegaWallFunction("wall"), X.Neumann("top", 0.0))
    X.assign(model, "turbulence.nut", X.Dirichlet("inlet", kin / win), X.Neumann("outlet", 0.0),
             X.NutWallFunction("wall") if wall_functions else X.Dirichlet("wall", 0.0), X.Neumann("top", 0.0))
    up = dict(divergence=X.Upwind)
    schemes = dict(U=X.set_schemes(**up), p=X.set_schemes(**up), k=X.set_schemes(**up),
                   omega=X.set_schemes(**up))
    s = solvers_for(model, relax_u=0.8, relax_p=0.2, **kw)
    s["k"] = X.set_solver(model.turbulence.k, solver=X.BicgstabSolver, preconditioner=X.DILU(),
                          convergence=1e-7, relax=0.8)
    s["omega"] = X.set_solver(model.turbulence.omega, solver=X.BicgstabSolver, preconditioner=X.DILU(),
                              convergence=1e-7, relax=0.8)
    config = X.Configuration(solvers=s, schemes=schemes,
                             runtime=X.set_runtime(iterations=iterations, write_interval=-1, time_step=1))
    X.initialise(model.U, [Uin, 0.0, 0.0])
    X.initialise(model.p, 0.0)
    X.initialise(model.turbulence.k, kin)
    X.initialise(model.turbulence.omega, win)
    X.initialise(model.turbulence.nut, kin / win)
    return mesh, model, config, None


def serving_stream(n_cases=512, rate=20.0, seed=12345, nmin=40, nmax=400, p_bfs=0.5, re_max=1000.0):
    """The serving workload: n_cases arrivals of a Poisson process (rate per
    second), each a cavity or (probability p_bfs) a BFS case of about N x N
    quads, N = round(exp(U(ln nmin, ln nmax))), Reynolds number U(50, re_max)
    applied through the viscosity (lid 1 m/s over 0.1 m; inlet 0.5 m/s over
    h = 10 mm).  The BFS gets N^2 cells split between its blocks by area
    (5h x h inlet and 30h x 2h outlet: 65 c^2 cells for c cells per h).
    Meshes are built once per (kind, size).  Returns a list of dicts with
    arrival time t, kind, N, Re, mesh, model, config, pref."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, n_cases)
    t = np.cumsum(gaps) - gaps[0]
    meshes = {}
    out = []
    for k in range(n_cases):
        is_bfs = rng.random() < p_bfs
        N = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        Re = float(rng.uniform(50.0, re_max))
        if is_bfs:
            c = max(2, int(round(N / np.sqrt(65.0))))
            key = ("bfs", c)
            if key not in meshes:
                meshes[key] = X.build_mesh(_unv("bfs", meshgen.bfs_unv, cells_per_h=c))
            mesh, model, config, pref = bfs(c, iterations=1, nu=0.5 * 0.01 / Re, mesh=meshes[key])
        else:
            key = ("cavity", N)
            if key not in meshes:
                meshes[key] = X.build_mesh(_unv("cavity", meshgen.cavity_unv, n=N, L=0.1))
            mesh, model, config, pref = cavity2d(N, iterations=1, nu=1.0 * 0.1 / Re, mesh=meshes[key])
        out.append(dict(t=float(t[k]), kind=key[0], N=N, Re=Re, mesh=mesh, model=model, config=config, pref=pref))
    return out

"""Seeded synthetic inputs with the shapes of the benchmark configurations, written as
Exasim datain/ folders (app, master, mesh, sol .bin) by exasim_b200.inputs.

* poisson2d_tri : 2D Poisson, p=3 triangles on an n x n grid split into 2n^2 triangles,
                  interior vertices moved by U(-0.05h, 0.05h); block Jacobi; GMRES(50) to 1e-10
                  (examples/Poisson/poisson2d/pdemodel.txt)
* poisson2d_quad: 2D Poisson on an n x n grid of quadrilaterals (element i + n j)
* convdiff3d_hex: 3D convection-diffusion, p=4 hexahedra on an n^3 grid of the unit cube,
                  c = (1, 0.5, 0.25), kappa = 0.01, Gaussian source at the centre (sigma 0.1),
                  u = 0 on the boundary, DIRK(3,3) with dt = 0.01; block Jacobi; GMRES(50) to 1e-8
* ns2d_tgv_quad : 2D compressible Navier-Stokes, Taylor-Green vortex on the periodic [0, 2 pi]^2,
                  p=3 quadrilaterals, Mach 0.1, Re 1600, gamma 1.4, Pr 0.72, DIRK(3,3) dt 0.05,
                  Newton to 1e-8, GMRES(100) with block ILU(0) on 4 x 4-element sub-domains
                  (periodic=False: the same square with boundary code 1 on every side)
* euler3d_vortex_hex: 3D Euler (no q), isentropic vortex of strength 5 on the periodic
                  [-5, 5]^3, p=3 hexahedra (320 x 320 element blocks), Mach 0.5, DIRK(2,2)
* cdsin2d_quad  : one request of the served stream: 2D convection-diffusion on the unit square,
                  kappa, velocity (cos theta, sin theta), source sin(a pi x) sin(b pi y), u = 0,
                  one Newton step, block Jacobi GMRES
"""
from __future__ import annotations

import os

import numpy as np

from . import inputs as I


def _on(axis, value):
    return lambda x: abs(x[axis] - value) < 1e-8


def write_case(datain: str, grid: I.Grid, master: I.Master, app: I.PDEApp, exprs, bcs, cartgridpart=()):
    os.makedirs(datain, exist_ok=True)
    bf = I.assign_bf(grid, exprs, bcs)
    I.write_app_bin(os.path.join(datain, "app.bin"), app)
    I.write_master_bin(os.path.join(datain, "master.bin"), master)
    I.write_mesh_bin(os.path.join(datain, "mesh.bin"), grid, master, bf, bcs, cartgridpart=cartgridpart)
    I.write_sol_bin(os.path.join(datain, "sol.bin"), I.dgnodes(grid, master), nc=app.nc, ncu=app.ncu)
    return datain


def poisson2d_tri(datain: str, n: int = 16, porder: int = 3, seed: int = 0, preconditioner: int = 0,
                  gmres_tol: float = 1e-10, restart: int = 50, ortho: int = 0):
    grid = I.square_tri_grid(n, perturb=0.05, seed=seed)
    master = I.make_master(2, 0, porder, 2 * porder)
    app = I.PDEApp(nd=2, ncu=1, model="ModelD", preconditioner=preconditioner, NewtonIter=1,
                   NewtonTol=1e-6, GMRESiter=1000, GMRESrestart=restart, GMREStol=gmres_tol, GMRESortho=ortho,
                   RBdim=0, ppdegree=1, tau=[1.0], physicsparam=[1.0], externalparam=[0.0, 0.0])
    exprs = [_on(1, 0.0), _on(0, 1.0), _on(1, 1.0), _on(0, 0.0)]
    return write_case(datain, grid, master, app, exprs, [1, 1, 1, 1])


def poisson2d_quad(datain: str, n: int = 16, porder: int = 3, preconditioner: int = 0, gmres_tol: float = 1e-10,
                   restart: int = 50, ortho: int = 0, cartgridpart=()):
    grid = I.square_quad_grid(n)
    master = I.make_master(2, 1, porder, 2 * porder)
    app = I.PDEApp(nd=2, ncu=1, model="ModelD", preconditioner=preconditioner, NewtonIter=1,
                   NewtonTol=1e-6, GMRESiter=1000, GMRESrestart=restart, GMREStol=gmres_tol, GMRESortho=ortho,
                   RBdim=0, ppdegree=1, tau=[1.0], physicsparam=[1.0], externalparam=[0.0, 0.0])
    exprs = [_on(1, 0.0), _on(0, 1.0), _on(1, 1.0), _on(0, 0.0)]
    return write_case(datain, grid, master, app, exprs, [1, 1, 1, 1], cartgridpart)


def convdiff3d_hex(datain: str, n: int = 16, porder: int = 4, nsteps: int = 20, dt: float = 0.01,
                   preconditioner: int = 0, gmres_tol: float = 1e-8, restart: int = 50, ortho: int = 0,
                   nstage: int = 3, torder: int = 3, cartgridpart=(), rbdim: int = 0):
    grid = I.cube_hex_grid(n)
    master = I.make_master(3, 1, porder, 2 * porder)
    app = I.PDEApp(nd=3, ncu=1, model="ModelD", preconditioner=preconditioner, NewtonIter=20,
                   NewtonTol=1e-6, GMRESiter=1000, GMRESrestart=restart, GMREStol=gmres_tol, GMRESortho=ortho,
                   RBdim=rbdim, ppdegree=1, tau=[1.0], torder=torder, nstage=nstage, dt=[dt] * nsteps,
                   physicsparam=[0.01, 1.0, 0.5, 0.25, 0.5, 0.5, 0.5, 0.1], externalparam=[0.0, 0.0])
    exprs = [_on(2, 0.0), _on(2, 1.0), _on(1, 0.0), _on(0, 1.0), _on(1, 1.0), _on(0, 0.0)]
    return write_case(datain, grid, master, app, exprs, [1, 1, 1, 1, 1, 1], cartgridpart)


def ns2d_tgv_quad(datain: str, n: int = 64, porder: int = 3, nsteps: int = 10, dt: float = 0.05,
                  preconditioner: int = 2, block: int = 4, restart: int = 100, gmres_tol: float = 1e-8,
                  newton_tol: float = 1e-8, mach: float = 0.1, tau: float = 2.0, periodic: bool = True):
    grid = I.periodic_square_quad_grid(n, 0.0, 2 * np.pi) if periodic else I.square_quad_grid(n, 2 * np.pi)
    master = I.make_master(2, 1, porder, 2 * porder)
    app = I.PDEApp(nd=2, ncu=4, model="ModelD", preconditioner=preconditioner, NewtonIter=20,
                   NewtonTol=newton_tol, GMRESiter=1000, GMRESrestart=restart, GMREStol=gmres_tol,
                   RBdim=0, ppdegree=1, tau=[tau], torder=3, nstage=3, dt=[dt] * nsteps,
                   physicsparam=[1.4, 1600.0, 0.72, mach], externalparam=[0.0, 0.0])
    cgp = (2, n, n, block, block, 0) if preconditioner == 2 else ()
    # periodic: no face carries a boundary code, but the list of boundary conditions still has
    # one entry, as the preprocessor writes it for a periodic domain (the reader builds
    # connectivity only when that list is non-empty, backend/Discretization/readbinaryfiles.cpp:
    # 390-393).  Otherwise every side gets boundary code 1, FbouHdg = f(u, q).n + tau (u - uhat).
    return write_case(datain, grid, master, app, [lambda x: True], [1], cgp)


def euler3d_vortex_hex(datain: str, n: int = 32, porder: int = 3, nsteps: int = 5, dt: float = 0.05,
                       preconditioner: int = 0, restart: int = 50, gmres_tol: float = 1e-8,
                       newton_tol: float = 1e-8, mach: float = 0.5, periodic: bool = True, hybrid: int = 1,
                       precMatrixType: int = 0):
    """hybrid = 0 selects the LDG discretisation with its pseudo-transient solver; periodic =
    False closes the cube with boundary code 1 on every side (the model's Ubou / Fbou)."""
    if periodic:
        grid = I.periodic_cube_hex_grid(n, -5.0, 10.0)
    else:
        grid = I.cube_hex_grid(n, 10.0)
        grid.p = grid.p - 5.0
    master = I.make_master(3, 1, porder, 2 * porder)
    app = I.PDEApp(nd=3, ncu=5, model="ModelC", preconditioner=preconditioner, NewtonIter=20,
                   NewtonTol=newton_tol, GMRESiter=1000, GMRESrestart=restart, GMREStol=gmres_tol,
                   RBdim=0, ppdegree=1, tau=[1.0 + 1.0 / mach], torder=2, nstage=2, dt=[dt] * nsteps,
                   physicsparam=[1.4, mach], externalparam=[0.0, 0.0], hybrid=hybrid,
                   precMatrixType=precMatrixType)
    return write_case(datain, grid, master, app, [lambda x: True], [1])


def cdsin2d_quad(datain: str, n: int = 16, porder: int = 3, kappa: float = 0.01, theta: float = 0.0,
                 a: int = 1, b: int = 1, gmres_tol: float = 1e-8, restart: int = 50, preconditioner: int = 0):
    grid = I.square_quad_grid(n)
    master = I.make_master(2, 1, porder, 2 * porder)
    # up to 100 restart cycles: strongly convective requests (kappa near 1e-3) need more than
    # 1000 block-Jacobi GMRES iterations to reach the tolerance
    app = I.PDEApp(nd=2, ncu=1, model="ModelD", preconditioner=preconditioner, NewtonIter=1,
                   NewtonTol=1e-8, GMRESiter=5000, GMRESrestart=restart, GMREStol=gmres_tol,
                   RBdim=0, ppdegree=1, tau=[1.0],
                   physicsparam=[kappa, float(np.cos(theta)), float(np.sin(theta)), float(a), float(b)],
                   externalparam=[0.0, 0.0])
    exprs = [_on(1, 0.0), _on(0, 1.0), _on(1, 1.0), _on(0, 0.0)]
    return write_case(datain, grid, master, app, exprs, [1, 1, 1, 1])

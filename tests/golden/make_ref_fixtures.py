"""Golden fixtures from the reference's own solver: inputs, intermediate arrays and solutions.

For each case below this script writes the case's datain/ folder (exasim_b200.cases, seeded),
runs the reference's cput2cEXASIM on it (oracle/refsolver.py; built from the reference tree
by oracle/build_ref_full.py) twice, and packs the result into tests/golden/ref_<case>.npz:

* datain: the four input files, byte for byte, so tests feed the CUDA path the very same input.
* The arrays the reference writes in debug mode at its first Newton step
  (backend/Discretization/uequation.cpp:764-774, matvec.cpp:114-116,185-187,203-205,
  solution.cpp:140-184): the condensed block H (its DinvH), the condensed residual Rh,
  D^-1 F (DinvF), D^-1 Ru, the right-hand side b, the preconditioner blocks, and the Newton
  step's GMRES solution x.  Arrays up to 200,000 entries are stored whole.  Larger element
  blocks are stored as their product with a seeded random vector per element (the seed is in
  the file), which a test recomputes from its own blocks.
* From a normal run of the same input: the solved trace field (outuhat) and, for DIRK cases,
  the last solution snapshot (outudg), the reference's Newton residual norms and GMRES counts,
  and per Newton solve (a steady solve or a DIRK stage) its Newton steps and GMRES iterations.

Every case's initial state is written into sol.bin (u only, the model's initial condition
from oracle/models.py), so both solvers start from the same numbers.  Usage:
    python tests/golden/make_ref_fixtures.py [case ...]
"""
from __future__ import annotations

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from exasim_b200 import cases, inputs as I  # noqa: E402
from oracle import refsolver as R  # noqa: E402

SEED = 20261203
FULL_LIMIT = 200_000


def _explicit_initial_state(datain, model):
    """Write u0 (the model's initial condition at the element nodes) into sol.bin."""
    from oracle.models import MODELS
    sol = I.read_sol_bin(os.path.join(datain, "sol.bin"))
    nd_s = sol["ndims"].astype(int)
    ne, npe, nd = nd_s[0], nd_s[3], nd_s[11]
    xdg = sol["xdg"].reshape(npe, nd, ne, order="F")
    app = I.read_app_bin(os.path.join(datain, "app.bin"))
    param = app["physicsparam"]
    ncu = int(app["ndims"][6])
    m = MODELS[model]()
    x = xdg.transpose(0, 2, 1).reshape(npe * ne, nd)
    u = np.asarray(m.initu(x, param)).reshape(npe * ne, ncu) if hasattr(m, "initu") else np.zeros((npe * ne, ncu))
    u = u.reshape(npe, ne, ncu).transpose(0, 2, 1)
    I.write_sol_bin(os.path.join(datain, "sol.bin"), xdg, udg=u, nc=int(app["ndims"][5]), ncu=ncu)


def _with_problem(datain, index, value):
    """Entry `index` of app.bin's problem part (27: ppdegree) set to value."""
    R.set_app_flag(datain, index, value, part=3)
    return datain


# name -> (model, writer(datain))
CASES = {
    # the first benchmark configuration at its full size: 512 perturbed p=3 triangles,
    # block Jacobi, GMRES(50) to 1e-10, one Newton step
    "poisson2d_tri16_p3": ("poisson2d", lambda d: cases.poisson2d_tri(d, n=16)),
    # elemental additive Schwarz on quadrilaterals
    "poisson2d_quad6_p3_eas": ("poisson2d", lambda d: cases.poisson2d_quad(d, n=6, preconditioner=1)),
    # the second configuration's physics on 3^3 p=4 hexahedra: DIRK(3,3), dt 0.01, two steps
    "convdiff3d_hex3_p4": ("convdiff3d", lambda d: cases.convdiff3d_hex(d, n=3, nsteps=2)),
    # the third configuration's physics: Taylor-Green vortex, 8 x 8 periodic p=3 quadrilaterals,
    # GMRES(100), Newton to 1e-8, one DIRK(3,3) step, block Jacobi (the reference's block ILU(0)
    # set-up overruns a buffer on fully periodic meshes: backend/Common/cpuimpl.h:1277 takes the
    # largest second element of f2e from the first-element row, and on a periodic mesh the last
    # element is never a face's first element)
    "ns2d_tgv_quad8_p3": ("ns2d", lambda d: cases.ns2d_tgv_quad(d, n=8, nsteps=1, preconditioner=0)),
    # block ILU(0) on Cartesian sub-domains (cartgridpart), on meshes with a boundary: 2D
    # quadrilaterals in 4 x 4-element blocks and 3D hexahedra in 2 x 2 x 2-element blocks
    "poisson2d_quad8_p3_bilu0": ("poisson2d", lambda d: cases.poisson2d_quad(
        d, n=8, preconditioner=2, cartgridpart=(2, 8, 8, 4, 4, 0))),
    "convdiff3d_hex4_p2_bilu0": ("convdiff3d", lambda d: cases.convdiff3d_hex(
        d, n=4, porder=2, nsteps=1, preconditioner=2, cartgridpart=(3, 4, 4, 4, 2, 2, 2, 0))),
    # the fifth configuration's physics: isentropic vortex, 3^3 periodic hexahedra (ModelC), one
    # DIRK(2,2) step, at p=2 (135 x 135 element blocks) and p=3 (320 x 320, the configuration's
    # own block size)
    "euler3d_hex3_p2": ("euler3d", lambda d: cases.euler3d_vortex_hex(d, n=3, porder=2, nsteps=1)),
    "euler3d_hex3_p3": ("euler3d", lambda d: cases.euler3d_vortex_hex(d, n=3, porder=3, nsteps=1)),
    # the first configuration with the polynomial preconditioner of degree 3 (ppdegree, GMRES
    # applies it after block Jacobi)
    "poisson2d_tri16_p3_poly3": ("poisson2d", lambda d: _with_problem(cases.poisson2d_tri(d, n=16), 27, 3)),
    # one request of the served stream: 8 x 8 quadrilaterals, p=3, kappa 0.05, theta 0.7
    "cdsin2d_quad8_p3": ("cdsin2d", lambda d: cases.cdsin2d_quad(d, n=8, kappa=0.05, theta=0.7, a=2, b=1)),
    # the LDG discretisation with the pseudo-transient solver (hybrid = 0): the isentropic
    # vortex on 3^3 p=2 hexahedra, one DIRK(2,2) step, periodic and closed by the model's
    # Ubou / Fbou on every side
    "euler3d_hex3_p2_ldg": ("euler3d", lambda d: cases.euler3d_vortex_hex(d, n=3, porder=2, nsteps=1, hybrid=0)),
    "euler3d_hex3_p2_ldg_bnd": ("euler3d", lambda d: cases.euler3d_vortex_hex(d, n=3, porder=2, nsteps=1, hybrid=0,
                                                                             periodic=False)),
    # the same with the reduced-basis initial guess of 5 vectors over two DIRK steps
    "euler3d_hex3_p2_ldg_rb": ("euler3d", lambda d: _with_problem(
        cases.euler3d_vortex_hex(d, n=3, porder=2, nsteps=2, hybrid=0), 16, 5)),
    # the periodic case with the polynomial preconditioner of degree 3
    "euler3d_hex3_p2_ldg_poly3": ("euler3d", lambda d: _with_problem(
        cases.euler3d_vortex_hex(d, n=3, porder=2, nsteps=1, hybrid=0), 27, 3)),
    # the closed cube with the element mass inverse as the preconditioner (precMatrixType 1)
    "euler3d_hex3_p2_ldg_minv": ("euler3d", lambda d: cases.euler3d_vortex_hex(
        d, n=3, porder=2, nsteps=1, hybrid=0, periodic=False, precMatrixType=1)),
}

# reference dump name -> fixture key, and the block shape used to project it (None: vector)
DUMPS = {
    "uEquationElemSchur_DinvH": ("H", "mm"),
    "uEquationElemSchur_DinvF": ("F", "nm"),
    "uEquationElemSchur_Rh": ("Rh", None),
    "uEquationElemSchur_Ru": ("Ru", None),
    "hdgAssembleRHS": ("b", None),
    "hdgBlockJacobi": ("P_bj", "bj"),
    "hdgElementalAdditiveSchwarz": ("P_eas", "mm"),
    "qEquationElem_Minv": ("Minv", "pp"),
    "1newton_x": ("x", None),
}


def projection_vector(rows_cols, nblocks, seed=SEED):
    """The seeded vector a blocked array [r, c, nblocks] is multiplied with, per block."""
    return np.random.default_rng(seed).standard_normal((rows_cols[1], nblocks))


def make(name, out_dir=HERE):
    model, writer = CASES[name]
    with tempfile.TemporaryDirectory() as tmp:
        d = os.path.join(tmp, "datain")
        writer(d)
        _explicit_initial_state(d, model)
        pack = {k: np.fromfile(os.path.join(d, k + ".bin"), dtype=np.uint8) for k in ("app", "master", "mesh", "sol")}
        pack["model"] = np.array(model)
        pack["seed"] = np.array(SEED)
        # normal run
        full = R.run(d, model, os.path.join(tmp, "full"))
        assert full.returncode == 0, full.stdout[-2000:]
        # an LDG run writes no trace field
        if os.path.exists(os.path.join(full.dataout, "outuhat_np0.bin")):
            pack["outuhat"] = full.uhat()
        pack["outudg"] = full.udg()
        pack["newton_norms"] = np.array([[a, b] for _, _, a, b in full.newton]).reshape(-1, 2)
        pack["gmres_iters"] = np.array(full.gmres_iters)
        # per Newton solve (steady solve or DIRK stage): Newton steps and GMRES iterations
        pack["solves"] = np.array([[a, b] for a, b, _, _ in full.solves], dtype=np.int64).reshape(-1, 2)
        if int(I.read_app_bin(os.path.join(d, "app.bin"))["problem"][0]) == 0:
            return _finish_ldg(name, model, d, tmp, full, pack, out_dir)
        # debug run: arrays of the first Newton step
        dbg_in = os.path.join(tmp, "dbg_in")
        shutil.copytree(d, dbg_in)
        R.set_app_flag(dbg_in, 3, 1)
        dbg = R.run(dbg_in, model, os.path.join(tmp, "dbg"))
        sizes = {}
        s = I.read_sol_bin(os.path.join(d, "sol.bin"))["ndims"].astype(int)
        m_ = I.read_master_bin(os.path.join(d, "master.bin"))
        for dump, (key, shape) in DUMPS.items():
            if dump not in dbg.dumps():
                continue
            a = dbg.dump(dump)
            if dump == "hdgElementalAdditiveSchwarz":
                # its debug write covers nf blocks of the ne-block array (matvec.cpp:185-187);
                # only the first ne are the element blocks
                r, c, _ = _block_shape(a.size, shape, d)
                a = a[:r * c * int(I.read_blob(os.path.join(d, "mesh.bin"))[1][1])]
            if a.size <= FULL_LIMIT or shape is None:
                pack[key] = a
            else:
                # [r, c, nblocks] column-major blocks: store A_k @ v_k per block
                sizes[key] = a.size
                pack["shape_" + key] = np.array(_block_shape(a.size, shape, d))
                r, c, nb = pack["shape_" + key]
                v = projection_vector((r, c), nb)
                pack["proj_" + key] = np.einsum("ijk,jk->ik", a.reshape(r, c, nb, order="F"), v)
        pack["dumped"] = np.array(sorted(k for k in pack if k in {v[0] for v in DUMPS.values()}
                                         or k.startswith("proj_")))
        fn = os.path.join(out_dir, f"ref_{name}.npz")
        np.savez_compressed(fn, **pack)
        print(f"{name}: {os.path.getsize(fn) / 1e6:.2f} MB, Newton {pack['newton_norms'].tolist()}, "
              f"GMRES {pack['gmres_iters'].tolist()}", flush=True)
        return fn


def _finish_ldg(name, model, d, tmp, full, pack, out_dir):
    """An LDG case: the PTC residual norms of each stage, and from a debug run without PTC
    steps (NewtonIter = 0) the residual of its last evaluation: the second DIRK stage's at
    the initial state (residual.cpp:613-617 writes it at every evaluation)."""
    pack["ptc_norms"] = np.array([v for s in full.ptc for v in s])
    pack["ptc_lengths"] = np.array([len(s) for s in full.ptc])
    dbg_in = os.path.join(tmp, "dbg_in")
    shutil.copytree(d, dbg_in)
    R.set_app_flag(dbg_in, 3, 1)
    R.set_app_flag(dbg_in, 13, 0, part=3)
    dbg = R.run(dbg_in, model, os.path.join(tmp, "dbg"))
    assert dbg.returncode == 0, dbg.stdout[-2000:]
    pack["Ru_stage2_initial"] = dbg.dump("_Ru")
    pack["dumped"] = np.array(["Ru_stage2_initial"])
    fn = os.path.join(out_dir, f"ref_{name}.npz")
    np.savez_compressed(fn, **pack)
    print(f"{name}: {os.path.getsize(fn) / 1e6:.2f} MB, PTC {full.ptc}, GMRES {pack['gmres_iters'].tolist()}",
          flush=True)
    return fn


def _block_shape(size, kind, datain):
    """Block shape [rows, cols, count] of a dump from the case's sizes."""
    app = I.read_app_bin(os.path.join(datain, "app.bin"))
    ncu = int(app["ndims"][6])
    mst = I.read_master_bin(os.path.join(datain, "master.bin"))
    npe, npf = int(mst["ndims"][5]), int(mst["ndims"][6])
    mesh = I.read_blob(os.path.join(datain, "mesh.bin"))
    ne, nfe = int(mesh[1][1]), int(mesh[1][4])
    n, m = npe * ncu, npf * nfe * ncu
    if kind == "mm":
        return [m, m, size // (m * m)]
    if kind == "nm":
        return [n, m, size // (n * m)]
    if kind == "pp":
        return [npe, npe, size // (npe * npe)]
    if kind == "bj":
        b = ncu * npf
        return [b, b, size // (b * b)]
    raise ValueError(kind)


if __name__ == "__main__":
    for c in (sys.argv[1:] or list(CASES)):
        make(c)

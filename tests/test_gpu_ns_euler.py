"""GPU parity on systems: 2D compressible Navier-Stokes (four conserved variables with
q, periodic, block ILU(0)) and 3D compressible Euler (ModelC: no q, periodic, element
blocks up to 320 x 320 through the blocked inverse).  Calls go through the C ABI; the
oracle's model Jacobians come from complex steps, independently of the symbolic
derivatives in the generated model sources.

Periodic meshes need at least 3 elements per periodic direction: with 2, the vertex
identification gives two different faces the same vertex set.

Tolerances:
  * initial state from the model's cpuInitu, geometry and assembled blocks H, Rh, b and
    preconditioner blocks: max |gpu - oracle| <= 1e-12 max |oracle|
  * D^-1 F and D^-1 Ru: 1e-11 (Gauss-Jordan against LAPACK; 1e-10 for the 320 x 320 blocked
    inverse, whose Schur complement adds its own rounding)
  * DIRK solutions after Newton to 1e-8: relative 2-norm distance <= 1e-6, Newton counts equal
"""
import numpy as np
import pytest

from exasim_b200 import HDGSolver, build as B, cases
from oracle.hdg import HDGOracle
from oracle.models import MODELS

pytestmark = pytest.mark.gpu
ASM_TOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build(["ns2d", "euler3d"])


def rel(a, b):
    a, b = np.asarray(a).ravel(order="F"), np.asarray(b).ravel(order="F")
    assert a.shape == b.shape
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def stage_state(s, o, seed, scale):
    """A DIRK-stage state near the initial one: perturbed udg/uh, a source sdg, time and
    d_jj / dt as the stage sets them."""
    rng = np.random.default_rng(seed)
    udg = o.udg * (1 + scale * rng.standard_normal(o.udg.shape))
    uh = o.uh * (1 + scale * rng.standard_normal(o.uh.shape))
    sdg = o.udg[:, :o.ncu] * 20.0
    for name, v in (("udg", udg), ("uh", uh), ("sdg", sdg)):
        s.set(name, v)
    o.udg, o.uh, o.sdg = udg.copy(), uh.copy(), sdg.copy()
    o.sdgg = np.einsum("gj,jce->gec", o.shapegt[:, :, 0], o.sdg)
    o.time, o.dtfactor = 0.0123, 20.0
    s.set_time(o.time, o.dtfactor)


def check_blocks(s, o, inv_tol):
    if o.ncq > 0:
        s.hdgGetQ()
        o.get_q(o.udg, o.uh)
        assert rel(s.get("udg"), o.udg) < ASM_TOL
    s.hdgAssembleLinearSystem()
    o.assemble()
    errs = {"H": rel(s.get("H"), o.H), "Rh": rel(s.get("Rh"), o.Rh), "b": rel(s.get("b"), o.assemble_rhs(o.Rh)),
            "F": rel(s.get("F"), o.DinvF), "Ru": rel(s.get("Ru"), o.Ru)}
    o.build_precond()
    if o.preconditioner == 2:
        ncf = o.ncu * o.npf
        got = s.get("P").reshape(ncf, ncf, o.bilu.nse, len(o.bilu.col_ind), order="F")
        errs["P"] = rel(got, np.transpose(o.P, (2, 3, 0, 1)))
    else:
        errs["P"] = rel(s.get("P"), o.P)
    print({k: float(f"{v:.2e}") for k, v in errs.items()})
    for k, v in errs.items():
        assert v < (inv_tol if k in ("F", "Ru") else ASM_TOL), (k, v, errs)


def test_ns2d_tgv_blocks_bilu0(tmp_path):
    d = cases.ns2d_tgv_quad(str(tmp_path / "ns"), n=4, porder=3, nsteps=1, block=2)
    s = HDGSolver(d, "ns2d")
    o = HDGOracle(d, MODELS["ns2d"]())
    assert rel(s.get("udg"), o.udg) < ASM_TOL   # cpuInitu at the element nodes
    stage_state(s, o, 1, 1e-3)
    check_blocks(s, o, 1e-11)
    s.close()


def test_ns2d_tgv_dirk_bilu0(tmp_path):
    d = cases.ns2d_tgv_quad(str(tmp_path / "ns"), n=4, porder=3, nsteps=1, block=2)
    s = HDGSolver(d, "ns2d")
    o = HDGOracle(d, MODELS["ns2d"]())
    its = s.DIRK(1)
    oits = o.dirk_solve(nsteps=1)
    assert list(its[:len(oits)]) == oits
    u, ref = s.get("udg"), o.udg.ravel(order="F")
    assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-6
    s.close()


def test_ns2d_mixed_dirk_matches_fp64(tmp_path):
    d = cases.ns2d_tgv_quad(str(tmp_path / "ns"), n=4, porder=3, nsteps=1, block=2)
    s64 = HDGSolver(d, "ns2d")
    s64.DIRK(1)
    s32 = HDGSolver(d, "ns2d")
    s32.set_precision(1, inner_tol=1e-4, rtol=1e-10)
    s32.DIRK(1)
    u, ref = s32.get("udg"), s64.get("udg")
    assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-6
    s64.close()
    s32.close()


@pytest.mark.parametrize("porder,inv_tol", [(2, 1e-11), (3, 1e-10)])
def test_euler3d_vortex_blocks(tmp_path, porder, inv_tol):
    d = cases.euler3d_vortex_hex(str(tmp_path / "eu"), n=3, porder=porder, nsteps=1)
    s = HDGSolver(d, "euler3d")
    o = HDGOracle(d, MODELS["euler3d"]())
    assert rel(s.get("udg"), o.udg) < ASM_TOL
    stage_state(s, o, 2, 1e-3)
    check_blocks(s, o, inv_tol)
    s.close()


@pytest.mark.parametrize("porder", [2, 3])
def test_euler3d_mixed_dirk_matches_fp64(tmp_path, porder):
    """The mixed form on 135 x 135 and 320 x 320 blocks (blocked FP32 inverse, products of
    more than 256 columns in chunks)."""
    d = cases.euler3d_vortex_hex(str(tmp_path / "eu"), n=3, porder=porder, nsteps=1)
    s64 = HDGSolver(d, "euler3d")
    s64.DIRK(1)
    s32 = HDGSolver(d, "euler3d")
    s32.set_precision(1, inner_tol=1e-4, rtol=1e-10)
    s32.DIRK(1)
    u, ref = s32.get("udg"), s64.get("udg")
    assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-6
    s64.close()
    s32.close()


@pytest.mark.parametrize("porder", [2, 3])
def test_euler3d_vortex_dirk(tmp_path, porder):
    d = cases.euler3d_vortex_hex(str(tmp_path / "eu"), n=3, porder=porder, nsteps=1)
    s = HDGSolver(d, "euler3d")
    o = HDGOracle(d, MODELS["euler3d"]())
    its = s.DIRK(1)
    oits = o.dirk_solve(nsteps=1)
    assert list(its[:len(oits)]) == oits
    u, ref = s.get("udg"), o.udg.ravel(order="F")
    assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-6
    s.close()

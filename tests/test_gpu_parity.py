"""GPU parity of the CUDA HDG path against the oracle (and, for Poisson3D, against the
reference's own golden solution).  Every call goes through the C ABI.

Tolerances (FP64 plain form):
  * assembled blocks H, Rh, RHS b, preconditioner blocks, matvec: max |gpu - oracle| <=
    1e-12 * max |oracle| (relative to the array's scale)
  * arrays that pass through the explicit element inverse alone (D^-1 F, D^-1 Ru) and the
    q matrices (Minv C, Minv E): 1e-11, since Gauss-Jordan and LAPACK getrf+getri round
    differently by about cond(D) * eps (cond(D) ~ 1e3 on these meshes)
  * solutions: |uh - uh_oracle| / |uh_oracle| <= the case's solver tolerance (the GMRES
    tolerance of a one-step linear solve, the Newton tolerance of a DIRK run)
"""
import os

import numpy as np
import pytest

from exasim_b200 import HDGSolver, build as B, cases
from oracle.hdg import HDGOracle
from oracle.models import MODELS
from tests.cases import poisson3d_datain

pytestmark = pytest.mark.gpu
ASM_TOL = 1e-12
INV_TOL = 1e-11


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build()


def rel(a, b):
    a = np.asarray(a).ravel(order="F")
    b = np.asarray(b).ravel(order="F")
    assert a.shape == b.shape
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def check_assembly(s: HDGSolver, o: HDGOracle, tol=ASM_TOL):
    s.hdgAssembleLinearSystem()
    o.assemble()
    errs = {
        "H": rel(s.get("H"), o.H),
        "Rh": rel(s.get("Rh"), o.Rh),
        "F": rel(s.get("F"), o.DinvF),
        "Ru": rel(s.get("Ru"), o.Ru),
        "b": rel(s.get("b"), o.assemble_rhs(o.Rh)),
    }
    o.build_precond()
    errs["P"] = rel(s.get("P"), o.P)
    for k, v in errs.items():
        assert v < (INV_TOL if k in ("F", "Ru") else tol), (k, v, errs)
    print("assembly parity (max rel err):", {k: float(f"{v:.2e}") for k, v in errs.items()})
    return errs


@pytest.fixture(scope="module")
def poisson2d_case(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("p2d") / "datain")
    cases.poisson2d_tri(d, n=4)
    return d


@pytest.fixture(scope="module")
def convdiff3d_case(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("cd3") / "datain")
    cases.convdiff3d_hex(d, n=2, nsteps=2)
    return d


def test_geometry_and_q_matrices(poisson2d_case):
    s = HDGSolver(poisson2d_case, "poisson2d")
    o = HDGOracle(poisson2d_case, MODELS["poisson2d"]())
    f2e, ec = s.connectivity()
    assert np.array_equal(f2e, o.f2e) and np.array_equal(ec, o.elemcon)
    ne, nge, nd = o.ne, o.nge, o.nd
    eg = s.get("elemg").reshape(-1, ne, order="F")
    xg = eg[:nge * nd].reshape(nge, nd, ne, order="F")
    Xx = eg[nge * nd:nge * (nd + nd * nd)].reshape(nge, nd * nd, ne, order="F")
    jac = eg[nge * (nd + nd * nd):].reshape(nge, ne, order="F")
    assert rel(xg, o.xg) < ASM_TOL and rel(Xx, o.Xx) < ASM_TOL and rel(jac, o.jac) < ASM_TOL
    # stored per element as [npe, nd, npe] and [npe, nd, ndf] (rows (l, d) stacked)
    MC = s.get("MinvC").reshape(o.npe, nd, o.npe, ne, order="F")
    ME = s.get("MinvE").reshape(o.npe, nd, o.npf * o.nfe, ne, order="F")
    assert rel(MC, np.transpose(o.MinvC, (0, 3, 1, 2))) < INV_TOL
    assert rel(ME, np.transpose(o.MinvE, (0, 3, 1, 2))) < INV_TOL
    s.close()


@pytest.mark.parametrize("precond", [0, 1])
def test_poisson2d_assembly_matvec_newton(tmp_path, precond):
    d = str(tmp_path / "datain")
    cases.poisson2d_tri(d, n=4, preconditioner=precond)
    s = HDGSolver(d, "poisson2d")
    o = HDGOracle(d, MODELS["poisson2d"]())
    s.hdgGetQ()
    o.get_q(o.udg, o.uh)
    assert rel(s.get("udg"), o.udg) < ASM_TOL
    check_assembly(s, o)
    # matvec and preconditioner on a random trace vector, through device pointers
    import torch
    N = s.sizes["ndofuhat"]
    rng = np.random.default_rng(3)
    v = rng.standard_normal(N)
    vt = torch.tensor(v, dtype=torch.float64, device="cuda")
    wt = torch.empty_like(vt)
    s.evalMatVec(vt.data_ptr(), wt.data_ptr())
    shape = (o.ncu, o.npf, o.nf)
    assert rel(wt.cpu().numpy(), o.matvec(v.reshape(shape, order="F"))) < ASM_TOL
    s.ApplyPreconditioner(vt.data_ptr(), wt.data_ptr())
    assert rel(wt.cpu().numpy(), o.apply_precond(v.reshape(shape, order="F"))) < ASM_TOL
    # residual norm (hdgAssembleResidual) and the Newton solve
    o2 = HDGOracle(d, MODELS["poisson2d"]())
    s2 = HDGSolver(d, "poisson2d")
    its, nrm = s2.NewtonSolver()
    oits, onrm = o2.newton()
    assert its == oits
    uh, uho = s2.get("uh"), o2.uh.ravel(order="F")
    assert np.linalg.norm(uh - uho) / np.linalg.norm(uho) < o2.gmres_tol
    assert abs(s2.stats()["gmres_total"] - o2.gmres_log[0].iters) <= 2
    s.close()
    s2.close()


def test_convdiff3d_time_dependent_assembly(convdiff3d_case):
    """DIRK-stage assembly (sdg, dtfactor) on p=4 hexahedra with q elimination."""
    s = HDGSolver(convdiff3d_case, "convdiff3d")
    o = HDGOracle(convdiff3d_case, MODELS["convdiff3d"]())
    rng = np.random.default_rng(7)
    udg = rng.standard_normal(o.udg.shape) * 0.1
    uh = rng.standard_normal(o.uh.shape) * 0.1
    sdg = rng.standard_normal((o.npe, o.ncu, o.ne))
    s.set("udg", udg)
    s.set("uh", uh)
    s.set("sdg", sdg)
    o.udg, o.uh = udg.copy(), uh.copy()
    o.sdg = sdg.copy()
    o.sdgg = np.einsum("gj,jce->gec", o.shapegt[:, :, 0], o.sdg)
    o.time, o.dtfactor = 0.0043, 229.4280360323567
    s.set_time(o.time, o.dtfactor)
    s.hdgGetQ()
    o.get_q(o.udg, o.uh)
    check_assembly(s, o)
    nrm = s.hdgAssembleResidual()
    onrm, _ = o.residual_norm()
    assert abs(nrm - onrm) / onrm < ASM_TOL
    s.close()


def test_convdiff3d_dirk_steps(convdiff3d_case):
    s = HDGSolver(convdiff3d_case, "convdiff3d")
    o = HDGOracle(convdiff3d_case, MODELS["convdiff3d"]())
    its = s.DIRK(2)
    oits = o.dirk_solve(nsteps=2)
    assert list(its[:len(oits)]) == oits
    u, uo = s.get("udg"), o.udg.ravel(order="F")
    # within the solver tolerance of the case (its Newton tolerance)
    assert np.linalg.norm(u - uo) / np.linalg.norm(uo) < o.newton_tol
    s.close()


def test_poisson3d_matches_reference_golden(tmp_path):
    """The reference's own golden output (24,576 p=2 tets, EAS, GMRES(50) to 1e-8)."""
    d, gold = poisson3d_datain(tmp_path)
    s = HDGSolver(d, "poisson3d")
    assert (s.sizes["ncu"], s.sizes["npf"], s.sizes["nf"]) == tuple(int(v) for v in gold[:3])
    its, nrm = s.NewtonSolver()
    assert its == 1 and nrm < 1e-6
    uh, ref = s.get("uh"), gold[3:]
    assert np.linalg.norm(uh - ref) / np.linalg.norm(ref) < 1e-10
    s.close()


def test_poisson3d_assembly_matches_oracle(tmp_path):
    d, _ = poisson3d_datain(tmp_path)
    s = HDGSolver(d, "poisson3d")
    o = HDGOracle(d, MODELS["poisson3d"]())
    s.hdgGetQ()
    o.get_q(o.udg, o.uh)
    check_assembly(s, o)
    s.close()

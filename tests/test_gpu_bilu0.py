"""GPU parity of the block ILU(0) preconditioner on Cartesian sub-domains (preconditioner 2)
against the oracle (oracle/bilu0.py, whose ordering is checked against the reference's own
routines in tests/test_bilu0_ordering.py).  Calls go through the C ABI.

Tolerances: factorized blocks and the preconditioner apply, max |gpu - oracle| <= 1e-11
max |oracle| (block inverses by Gauss-Jordan against LAPACK, through up to nfse factorization
steps); Newton solution to 1e3 x the GMRES tolerance; GMRES iteration counts within 2."""
import numpy as np
import pytest

from exasim_b200 import HDGSolver, build as B, cases
from oracle.hdg import HDGOracle
from oracle.models import MODELS

pytestmark = pytest.mark.gpu
TOL = 1e-11


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build()


def rel(a, b):
    a, b = np.asarray(a).ravel(order="F"), np.asarray(b).ravel(order="F")
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def make(tmp_path, nd):
    d = str(tmp_path / f"bilu{nd}")
    if nd == 2:
        cases.poisson2d_quad(d, n=8, porder=2, preconditioner=2, cartgridpart=(2, 8, 8, 4, 2, 0))
        return d, "poisson2d"
    cases.convdiff3d_hex(d, n=4, porder=2, nsteps=2, preconditioner=2, cartgridpart=(3, 4, 4, 4, 2, 2, 2, 0))
    return d, "convdiff3d"


@pytest.mark.parametrize("nd", [2, 3])
def test_bilu0_blocks_and_apply(tmp_path, nd):
    d, model = make(tmp_path, nd)
    s = HDGSolver(d, model)
    o = HDGOracle(d, MODELS[model]())
    if nd == 3:
        # a DIRK-stage state: source sdg, time and d_jj / dt as the stage sets them
        rng = np.random.default_rng(7)
        udg = rng.standard_normal(o.udg.shape) * 0.1
        uh = rng.standard_normal(o.uh.shape) * 0.1
        sdg = rng.standard_normal((o.npe, o.ncu, o.ne))
        s.set("udg", udg)
        s.set("uh", uh)
        s.set("sdg", sdg)
        o.udg, o.uh, o.sdg = udg.copy(), uh.copy(), sdg.copy()
        o.sdgg = np.einsum("gj,jce->gec", o.shapegt[:, :, 0], o.sdg)
        o.time, o.dtfactor = 0.0043, 229.4280360323567
        s.set_time(o.time, o.dtfactor)
    s.hdgGetQ()
    o.get_q(o.udg, o.uh)
    s.hdgAssembleLinearSystem()
    o.assemble()
    o.build_precond()
    ncf = o.ncu * o.npf
    b = o.bilu
    got = s.get("P").reshape(ncf, ncf, b.nse, len(b.col_ind), order="F")
    assert rel(got, np.transpose(o.P, (2, 3, 0, 1))) < TOL
    # the device factors reproduce the assembled sub-domain matrix on its block pattern
    from tests.test_bilu0_ordering import ilu_pattern_error
    orig = b.assemble(o.H.reshape(o.ncu * o.npf * o.nfe, o.ncu * o.npf * o.nfe, o.ne, order="F"))
    fac = np.transpose(got, (2, 3, 0, 1))
    assert max(ilu_pattern_error(fac[r], orig[r], b.row_ptr, b.col_ind) for r in range(b.nse)) < 1e-10
    import torch
    N = s.sizes["ndofuhat"]
    v = np.random.default_rng(5).standard_normal(N)
    vt = torch.tensor(v, dtype=torch.float64, device="cuda")
    wt = torch.empty_like(vt)
    s.ApplyPreconditioner(vt.data_ptr(), wt.data_ptr())
    ref = o.apply_precond(v.reshape(o.ncu, o.npf, o.nf, order="F"))
    assert rel(wt.cpu().numpy(), ref) < TOL
    s.close()


def test_bilu0_newton_2d(tmp_path):
    d, model = make(tmp_path, 2)
    s = HDGSolver(d, model)
    o = HDGOracle(d, MODELS[model]())
    its, nrm = s.NewtonSolver()
    oits, onrm = o.newton()
    assert its == oits
    assert abs(s.stats()["gmres_total"] - o.gmres_log[0].iters) <= 2
    uh, ref = s.get("uh"), o.uh.ravel(order="F")
    assert np.linalg.norm(uh - ref) / np.linalg.norm(ref) < 1e3 * o.gmres_tol
    s.close()


def test_bilu0_dirk_3d(tmp_path):
    d, model = make(tmp_path, 3)
    s = HDGSolver(d, model)
    o = HDGOracle(d, MODELS[model]())
    its = s.DIRK(1)
    oits = o.dirk_solve(nsteps=1)
    assert list(its[:len(oits)]) == oits
    u, ref = s.get("udg"), o.udg.ravel(order="F")
    assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-6
    s.close()


def test_bilu0_mixed_precision(tmp_path):
    d, model = make(tmp_path, 2)
    s64 = HDGSolver(d, model)
    s64.NewtonSolver()
    s32 = HDGSolver(d, model)
    s32.set_precision(1, inner_tol=1e-4, rtol=1e-10)
    s32.NewtonSolver()
    a0, a1 = s32.last_residual()
    assert a1 <= 1e-10 * a0
    u, ref = s32.get("uh"), s64.get("uh")
    assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-6
    s64.close()
    s32.close()

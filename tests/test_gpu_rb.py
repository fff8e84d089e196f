"""The reduced-basis initial guess of GMRES (RBdim > 0, the reference's default of 5;
ptcsolver.cpp:217-236, 374-379, preconditioner.cpp:133-181) against the oracle's
restatement: DIRK steps on the 3D convection-diffusion case, where every stage starts its
GMRES from the projection onto the last Newton updates.  Newton counts must be equal,
GMRES counts within 2, the solution within 1e-6 (2-norm, relative); with the guess GMRES
takes fewer iterations than without it."""
import numpy as np
import pytest

from exasim_b200 import HDGSolver, build as B, cases
from oracle.hdg import HDGOracle
from oracle.models import MODELS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build(["convdiff3d"])


@pytest.mark.parametrize("precision", [0, 1])
def test_rb_guess_dirk_matches_oracle(tmp_path, precision):
    d = cases.convdiff3d_hex(str(tmp_path / "rb"), n=3, porder=2, nsteps=3, rbdim=5)
    s = HDGSolver(d, "convdiff3d")
    if precision:
        s.set_precision(1, inner_tol=1e-4, rtol=1e-10)
    iters = []
    for istep in range(3):
        for j in range(3):
            its, _ = s.DIRKStage(istep, j)
            iters.append(s.stats()["gmres_total"])
    o = HDGOracle(d, MODELS["convdiff3d"]())
    ologs = []
    o.dirk_solve(nsteps=3, on_stage=lambda i, j, oo: ologs.append(sum(g.iters for g in oo.gmres_log)))
    assert o.rb_cur == 5
    u, ref = s.get("udg"), o.udg.ravel(order="F")
    assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-6
    if precision == 0:
        assert all(abs(a - b) <= 2 for a, b in zip(iters, ologs)), (iters, ologs)
        d0 = cases.convdiff3d_hex(str(tmp_path / "rb0"), n=3, porder=2, nsteps=3, rbdim=0)
        s0 = HDGSolver(d0, "convdiff3d")
        it0 = []
        for istep in range(3):
            for j in range(3):
                s0.DIRKStage(istep, j)
                it0.append(s0.stats()["gmres_total"])
        assert sum(iters) < sum(it0), (iters, it0)
        s0.close()
    s.close()

"""Mixed-precision form (3xTF32 tensor-core element elimination, FP32 condensed blocks, FP64
residual refinement) through the C ABI.

Tolerances:
  * condensed block H (FP32, from 3xTF32 products and an FP32 inverse): max |H32 - H_oracle|
    <= 1e-4 max |H_oracle| (FP32 rounding amplified by cond(D) ~ 1e3 through D^-1)
  * solution of a mixed solve: relative 2-norm distance to the FP64 solve <= 1e-6, and the
    FP64 residual norm reaches the requested ratio
"""
import numpy as np
import pytest

from exasim_b200 import HDGSolver, build as B, cases
from oracle.hdg import HDGOracle
from oracle.models import MODELS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build()


@pytest.fixture(scope="module")
def cd3(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("cd3m") / "datain")
    cases.convdiff3d_hex(d, n=3, nsteps=2)
    return d


def rel2(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def test_mixed_condensed_blocks_close_to_fp64(cd3):
    s = HDGSolver(cd3, "convdiff3d")
    o = HDGOracle(cd3, MODELS["convdiff3d"]())
    s.set_precision(1)
    rng = np.random.default_rng(11)
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
    H = s.get("H32")
    err = np.abs(H - o.H.ravel(order="F")).max() / np.abs(o.H).max()
    assert err < 1e-4, err
    s.close()


@pytest.mark.parametrize("case", ["poisson2d", "convdiff3d"])
def test_mixed_newton_matches_fp64(tmp_path, cd3, case):
    if case == "poisson2d":
        d = str(tmp_path / "datain")
        cases.poisson2d_tri(d, n=6)
    else:
        d = cd3
    s64 = HDGSolver(d, case)
    its64, _ = s64.NewtonSolver()
    u64 = s64.get("uh")
    r0, r1 = s64.last_residual()
    s32 = HDGSolver(d, case)
    s32.set_precision(1, inner_tol=1e-4, rtol=1e-10)
    its, nrm = s32.NewtonSolver()
    a0, a1 = s32.last_residual()
    assert a1 <= 1e-10 * a0, (a0, a1, its)
    assert rel2(s32.get("uh"), u64) < 1e-6
    assert rel2(s32.get("udg"), s64.get("udg")) < 1e-6
    print(f"{case}: fp64 {its64} Newton steps, ratio {r1 / r0:.2e}; mixed {its} steps, ratio {a1 / a0:.2e}, "
          f"GMRES {s32.stats()['gmres_total']}")
    s64.close()
    s32.close()


def test_mixed_dirk_steps_match_fp64(cd3):
    s64 = HDGSolver(cd3, "convdiff3d")
    s64.DIRK(2)
    s32 = HDGSolver(cd3, "convdiff3d")
    s32.set_precision(1, inner_tol=1e-4, rtol=1e-10)
    s32.DIRK(2)
    assert rel2(s32.get("udg"), s64.get("udg")) < 1e-6
    s64.close()
    s32.close()


def test_switching_forms_on_one_context(cd3):
    """A context that solves in FP64 (capturing its GMRES steps as CUDA graphs), switches to the
    mixed form (which frees the FP64 blocks it does not read) and back solves each stage as a
    context that never switched: FP64 stages bit for bit, the mixed stage within 1e-6."""
    ref = HDGSolver(cd3, "convdiff3d")
    s = HDGSolver(cd3, "convdiff3d")
    for j in range(2):  # FP64 stages on both: the second replays captured GMRES steps
        ref.DIRKStage(0, j)
        s.DIRKStage(0, j)
    assert np.array_equal(s.get("udg"), ref.get("udg"))
    s.set_precision(1, inner_tol=1e-4, rtol=1e-10)
    ref.DIRKStage(0, 2)
    s.DIRKStage(0, 2)
    assert rel2(s.get("udg"), ref.get("udg")) < 1e-6
    with pytest.raises(Exception):
        s.get("F")  # D^-1 F in FP64 is not held in the mixed form
    s.set_precision(0)
    s.set("udg", ref.get("udg"))
    s.set("uh", ref.get("uh"))
    for j in range(3):
        ref.DIRKStage(1, j)
        s.DIRKStage(1, j)
    assert np.array_equal(s.get("udg"), ref.get("udg"))
    assert np.array_equal(s.get("F"), ref.get("F"))
    s.close()
    ref.close()

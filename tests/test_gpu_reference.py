"""The CUDA path against the reference's own solver, through the C ABI.

Each fixture in tests/golden/ref_*.npz (tests/golden/make_ref_fixtures.py) holds a case's
datain/ folder, the arrays the reference's cput2cEXASIM wrote at its first Newton step, and the
outputs of its normal run.  The CUDA path reads the same datain/ and must reproduce:

  * H, Rh, b and the block-Jacobi / additive-Schwarz preconditioner blocks of the first
    Newton step: max |gpu - reference| <= 1e-12 max |reference|;
  * D^-1 F and D^-1 Ru (through the explicit element inverse; Gauss-Jordan here, LAPACK getrf +
    getri in the reference; last-bit differences of D grow by cond(D), about 1e3): 5e-12;
  * the residual vectors of a DIRK stage, relative to the larger of max |reference| and the
    size of the same vector without the stage source (the mass term and the stage source
    cancel at a stage's first Newton step, so both solvers round at the mass term's scale);
  * the final solution: |gpu - reference| / |reference| <= the case's solver tolerance
    (GMREStol for the one-step linear cases, NewtonTol for the others), with the same Newton
    step count per solve and GMRES counts within 2 of the reference's (counted as Arnoldi steps:
    the reference prints one fewer per call that converges inside a restart cycle).

The reference was built with its own flags (-O3 -ffast-math); its spread against an IEEE-strict
build of itself is 4.8e-13 on H and 2.1e-13 on D^-1 F on the 512-triangle case.

Each case runs twice: with the model library built from this package's model sources
(exasim_b200/models/<model>), and with one built from the very files the reference's own
text2code generated for the case's pdemodel.txt (oracle/_ref/models/<model>/gen, made by
oracle/build_ref_full.py), compiled unchanged: the model plugin boundary dropped in as is.
"""
import os

import numpy as np
import pytest

from exasim_b200 import HDGSolver, build as B
from exasim_b200 import inputs as I
from tests import ref_fixtures as RF

pytestmark = pytest.mark.gpu
ASM_TOL = 1e-12
INV_TOL = 5e-12
GEN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "models")
SOURCES = ("package", "text2code")


def model_library(model: str, source: str) -> str:
    """Name of the solver library for `model` built from `source` (building it if needed)."""
    if source == "package":
        B.build([model])
        return model
    gen = os.path.join(GEN, model, "gen")
    if not os.path.isdir(gen):
        pytest.skip("text2code output of the reference build is absent (oracle/build_ref_full.py)")
    B.build(sources={"t2c_" + model: gen})
    return "t2c_" + model


def _first_step(s, stage, zero_source=False, ncq=0):
    if stage is not None:
        t, dtf, sdg = stage
        s.set_time(t, dtf)
        s.set("sdg", np.zeros_like(sdg).ravel(order="F") if zero_source else sdg.ravel(order="F"))
    if ncq > 0:
        s.hdgGetQ()
    s.hdgAssembleLinearSystem()


@pytest.mark.parametrize("source", SOURCES)
@pytest.mark.parametrize("name", RF.names())
def test_first_newton_step_matches_reference(name, source, tmp_path):
    fx = RF.load(name)
    d = RF.write_datain(fx, str(tmp_path / "datain"))
    model = model_library(str(fx["model"]), source)
    app = I.read_app_bin(d + "/app.bin")
    ncq = int(app["ndims"][7])
    precond = int(app["flag"][6])
    stage = RF.first_stage_state(d)
    s = HDGSolver(d, model)
    scale = {}
    if stage is not None:
        _first_step(s, stage, zero_source=True, ncq=ncq)
        scale = {k: np.abs(s.get(k)).max() for k in ("Ru", "Rh", "b")}
        s.close()
        s = HDGSolver(d, model)
    _first_step(s, stage, ncq=ncq)
    errs = {}
    for key, field in (("H", "H"), ("Rh", "Rh"), ("F", "F"), ("Ru", "Ru"), ("b", "b")):
        a, r = RF.reference_view(fx, key, s.get(field))
        den = max(np.abs(r).max(), scale.get(key, 0.0), 1e-300)
        errs[key] = float(np.abs(np.ravel(a) - np.ravel(r)).max() / den)
    pkey = {0: "P_bj", 1: "P_eas"}.get(precond)
    if pkey and RF.has(fx, pkey):
        errs["P"] = RF.rel_err(fx, pkey, s.get("P"))
    s.close()
    print(name, {k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < (INV_TOL if k in ("F", "Ru") else ASM_TOL), (name, k, v, errs)


@pytest.mark.parametrize("source", SOURCES)
@pytest.mark.parametrize("name", RF.names())
def test_solution_matches_reference(name, source, tmp_path):
    fx = RF.load(name)
    d = RF.write_datain(fx, str(tmp_path / "datain"))
    model = model_library(str(fx["model"]), source)
    app = I.read_app_bin(d + "/app.bin")
    dt = app["dt"]
    newton_tol, gmres_tol = app["solversparam"][0], app["solversparam"][1]
    s = HDGSolver(d, model)
    if int(app["problem"][27]) > 1:
        # the polynomial preconditioner's Arnoldi process starts from the reference's own vector
        from oracle.hdg import HDGOracle
        from oracle.models import MODELS
        s.set("randvect", RF.reference_randvect(HDGOracle(d, MODELS[str(fx["model"])]())))
    uh_ref = fx["outuhat"]
    ncu, npf, nf = (int(v) for v in uh_ref[:3])
    N = ncu * npf * nf
    if dt.size and dt[0] > 0:
        nsteps = dt.size
        counts = s.DIRK(nsteps)[:nsteps * int(app["problem"][4])]
        udg_ref = fx["outudg"]
        nud = int(np.prod(udg_ref[:3]))
        u_ref = udg_ref[3:].reshape(-1, nud)[-1]
        tol = newton_tol
        u = s.get("udg")
        rel_u = np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref)
        assert rel_u < tol, (name, "udg", rel_u)
    else:
        its, _ = s.NewtonSolver()
        counts = [its]
        tol = gmres_tol if int(app["problem"][13]) == 1 else newton_tol
        rel_u = None
    uh = s.get("uh")
    ref = uh_ref[3:].reshape(-1, N)[-1]
    rel = np.linalg.norm(uh - ref) / np.linalg.norm(ref)
    gmres_last = s.stats()["gmres_total"]
    s.close()
    ref_newton = [int(v) for v in fx["solves"][:, 0]]
    # the reference reports one iteration fewer per GMRES call than the Arnoldi steps it takes
    # when it converges inside a restart cycle (gmres.cpp:535-545 returns j before the loop's
    # j++), so each of the last solve's calls (one per Newton step) adds one to its count
    ref_gmres_last = int(fx["solves"][-1, 1]) + int(fx["solves"][-1, 0])
    print(name, f"uhat rel {rel:.2e}", f"udg rel {rel_u:.2e}" if rel_u is not None else "",
          "Newton", list(counts), ref_newton, "GMRES (last solve)", gmres_last, ref_gmres_last)
    assert rel < tol, (name, rel, tol)
    assert [int(c) for c in counts] == ref_newton, (list(counts), ref_newton)
    assert abs(gmres_last - ref_gmres_last) <= 2, (gmres_last, ref_gmres_last)


def test_reference_builtin_poisson3d_sources_reproduce_golden(tmp_path):
    """The generated model sources the reference ships (backend/Main/BuiltIn/Poisson3D, with its
    numbered HdgFlux1/HdgFlux2 siblings that libpdemodel.cpp does not include), compiled
    unchanged, reproduce the reference's own golden trace solution
    (examples/Poisson/poisson3d/dataout/outuhat_np0.bin) to 1e-10."""
    from tests.cases import poisson3d_datain
    gen = os.path.join(GEN, "poisson3d_builtin", "gen")
    if not os.path.isdir(gen):
        pytest.skip("the reference's built-in model sources were not copied (oracle/build_ref_full.py)")
    B.build(sources={"t2c_poisson3d_builtin": gen})
    d, gold = poisson3d_datain(tmp_path)
    s = HDGSolver(d, "t2c_poisson3d_builtin")
    its, nrm = s.NewtonSolver()
    uh, ref = s.get("uh"), gold[3:]
    s.close()
    assert its == 1
    assert np.linalg.norm(uh - ref) / np.linalg.norm(ref) < 1e-10

"""The CUDA LDG path (problem[0] = 0: element residuals, finite-difference Jacobian products,
pseudo-transient solves) through the C ABI, against the reference's own LDG runs
(tests/golden/ref_*_ldg*.npz, cput2cEXASIM) and the LDG oracle (oracle/ldg.py):

  * the residual of one evaluation (the second DIRK stage's at the initial state, the
    reference's debug dump): |gpu - reference| / |reference| <= 1e-12;
  * the residual at a perturbed, non-smooth state against the oracle: the same bound;
  * the DIRK(2,2) steps of PTC solves (one; two with the reduced-basis guess; the mass-inverse
    and polynomial preconditioners): the solution within the PTC tolerance of the reference's
    and the same PTC step count per stage;
  * the configurations the path does not cover are refused with EXA_ERR_UNSUPPORTED.

Each case runs with the model library built from this package's model sources and with one
built from the reference's text2code output for the model (its KokkosUbou / KokkosFbou
included), compiled unchanged.
"""
import os
import shutil

import numpy as np
import pytest

from exasim_b200 import ExaError, HDGSolver, cases
from oracle.hdg import dirk_coeff
from oracle.ldg import LDGOracle
from oracle.models import MODELS
from oracle.refsolver import set_app_flag
from tests import ref_fixtures as RF
from tests.test_gpu_reference import SOURCES, model_library

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _stage2_source(o, u):
    c, dd, tt = dirk_coeff(o.nstage, o.torder)
    S, dt = o.nstage, o.dt[0]
    sdg = u * (dd[0] / dt)
    sdg = u * (-dd[1] / dt) + sdg * ((dd[1] + dd[S + 1]) / dd[0])
    return o.factor[0] + dt * tt[1], dd[S + 1] / dt, sdg


@pytest.mark.parametrize("source", SOURCES)
@pytest.mark.parametrize("name", RF.ldg_names())
def test_ldg_residual_reference(name, source, tmp_path):
    fx = RF.load(name)
    d = RF.write_datain(fx, str(tmp_path / "datain"))
    set_app_flag(d, 13, 0, part=3)  # no PTC steps: each stage evaluates its initial residual only
    s = HDGSolver(d, model_library(str(fx["model"]), source))
    s.DIRK(len(fx["ptc_lengths"]) // 2)  # the dump is the last stage's (DIRK(2,2))
    R = s.get("Ru")
    ref = fx["Ru_stage2_initial"]
    s.close()
    rel = np.linalg.norm(R - ref) / np.linalg.norm(ref)
    print(name, source, f"residual rel {rel:.2e}")
    assert rel < TOL, rel


@pytest.mark.parametrize("name", RF.ldg_names())
def test_ldg_residual_perturbed_oracle(name, tmp_path):
    fx = RF.load(name)
    d = RF.write_datain(fx, str(tmp_path / "datain"))
    o = LDGOracle(d, MODELS[str(fx["model"])]())
    u0 = o.udg[:, :o.ncu].copy()
    t, dtf, sdg = _stage2_source(o, u0)
    u = u0 * (1.0 + 1e-2 * np.random.default_rng(7).standard_normal(u0.shape))
    o.time, o.dtfactor, o.sdg = t, dtf, sdg
    o.sdgg = np.einsum("gj,jce->gec", o.shapegt[:, :, 0], sdg)
    R_o = o.residual_ldg(u)
    s = HDGSolver(d, model_library(str(fx["model"]), "package"))
    s.set_time(t, dtf)
    s.set("sdg", sdg.ravel(order="F"))
    s.set("udg", u.ravel(order="F"))
    nrm = s.evalResidual()
    R = s.get("Ru")
    s.close()
    rel = np.linalg.norm(R - R_o.ravel(order="F")) / np.linalg.norm(R_o)
    print(name, f"perturbed residual rel {rel:.2e}")
    assert rel < TOL, rel
    assert abs(nrm - np.linalg.norm(R_o)) <= 1e-12 * np.linalg.norm(R_o)


@pytest.mark.parametrize("source", SOURCES)
@pytest.mark.parametrize("name", RF.ldg_names())
def test_ldg_dirk_step_reference(name, source, tmp_path):
    fx = RF.load(name)
    d = RF.write_datain(fx, str(tmp_path / "datain"))
    s = HDGSolver(d, model_library(str(fx["model"]), source))
    o = LDGOracle(d, MODELS[str(fx["model"])]())
    if o.ppdegree > 1:
        # the polynomial's Arnoldi process starts from the reference's own vector
        s.set("randvect", RF.reference_randvect(o, faces=False))
    nsolves = len(fx["ptc_lengths"])
    its = s.DIRK(nsolves // 2)[:nsolves]  # DIRK(2,2): two stage solves per step
    u = s.get("udg")
    s.close()
    udg_ref = fx["outudg"]
    nud = int(np.prod(udg_ref[:3]))
    u_ref = udg_ref[3:].reshape(-1, nud)[-1]
    rel = np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref)
    ref_its = [int(v) for v in fx["solves"][:, 0]]
    print(name, source, f"udg rel {rel:.2e}", "PTC", list(its), ref_its)
    assert rel < 1e-8, rel
    assert list(its) == ref_its


def test_ldg_refusals(tmp_path):
    # q (ncq > 0): the reference's GetQ gives no parity target
    d = str(tmp_path / "cd")
    cases.convdiff3d_hex(d, n=2, porder=2, nsteps=1)
    set_app_flag(d, 0, 0, part=3)
    with pytest.raises(ExaError) as e:
        HDGSolver(d, model_library("convdiff3d", "package"))
    assert e.value.code == 2 and "LDG" in str(e.value)
    # the mixed-precision form condenses the HDG system only
    d2 = str(tmp_path / "eu")
    cases.euler3d_vortex_hex(d2, n=2, porder=2, nsteps=1, hybrid=0)
    s = HDGSolver(d2, model_library("euler3d", "package"))
    with pytest.raises(ExaError) as e:
        s.set_precision(1)
    assert e.value.code == 2
    s.close()

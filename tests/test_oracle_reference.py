"""The oracle against the reference's own solver (CPU).

Each fixture in tests/golden/ref_*.npz holds a case's datain/ folder and the arrays that the
reference's cput2cEXASIM wrote at its first Newton step (tests/golden/make_ref_fixtures.py).
The oracle reads the same datain/, assembles the same first Newton step and must reproduce:

  * the condensed block H, the condensed residual Rh, the right-hand side b and the
    preconditioner blocks: max |oracle - reference| <= 1e-12 max |reference|;
  * D^-1 F and D^-1 Ru, which pass through the explicit element inverse (LAPACK getrf + getri
    in both): the last-bit differences of two assemblies of D grow by cond(D) (about 1e3 here)
    in the inverse, so 5e-12 of max |reference| (the worst case, 512 perturbed p=3 triangles,
    gives 2.1e-12);
  * residual vectors of a DIRK stage (Ru, Rh, b): at the first Newton step of a stage the mass
    term dtfactor M u and the stage source M sdg cancel down to the spatial residual, so both
    solvers round at the scale of the mass term; the tolerance 1e-12 is taken relative to the
    larger of max |reference| and max |same vector with the stage source set to zero|.

The reference was built with its own flags (-O3 -ffast-math).  The spread between that build
and an IEEE-strict build of the same sources is 4.8e-13 on H and 2.1e-13 on D^-1 F
(poisson2d_tri16_p3), so 1e-12 is twice the reference's own flag spread.
"""
import numpy as np
import pytest

from oracle.hdg import HDGOracle
from oracle.models import MODELS
from tests import ref_fixtures as RF

ASM_TOL = 1e-12
INV_TOL = 5e-12


def _oracle_first_step(datain, model, stage, zero_source=False):
    o = HDGOracle(datain, MODELS[model]())
    if stage is not None:
        o.time, o.dtfactor, sdg = stage
        o.sdg = np.zeros_like(sdg) if zero_source else sdg
        o.sdgg = np.einsum("gj,jce->gec", o.shapegt[:, :, 0], o.sdg)
    if o.ncq > 0:
        o.get_q(o.udg, o.uh)
    o.assemble()
    return o


@pytest.mark.parametrize("name", RF.names())
def test_oracle_matches_reference_first_newton_step(name, tmp_path):
    fx = RF.load(name)
    d = RF.write_datain(fx, str(tmp_path / "datain"))
    model = str(fx["model"])
    stage = RF.first_stage_state(d)
    o = _oracle_first_step(d, model, stage)
    b = o.assemble_rhs(o.Rh)
    scale = {}
    if stage is not None:
        o0 = _oracle_first_step(d, model, stage, zero_source=True)
        scale = {"Ru": np.abs(o0.Ru).max(), "Rh": np.abs(o0.Rh).max(), "b": np.abs(o0.assemble_rhs(o0.Rh)).max()}
    errs = {}
    for key, mine in (("H", o.H), ("Rh", o.Rh), ("F", o.DinvF), ("Ru", o.Ru), ("b", b)):
        a, r = RF.reference_view(fx, key, mine)
        den = max(np.abs(r).max(), scale.get(key, 0.0), 1e-300)
        errs[key] = float(np.abs(np.ravel(a) - np.ravel(r)).max() / den)
    o.build_precond()
    pkey = {0: "P_bj", 1: "P_eas"}.get(o.preconditioner)
    if pkey and RF.has(fx, pkey):
        errs["P"] = RF.rel_err(fx, pkey, o.P)
    print(name, {k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < (INV_TOL if k in ("F", "Ru") else ASM_TOL), (name, k, v)


@pytest.mark.parametrize("name", [n for n in RF.names() if "poly" in n])
def test_oracle_polynomial_preconditioner_matches_reference(name, tmp_path):
    """GMRES with the polynomial preconditioner (ppdegree > 1), started from the reference's own
    Arnoldi vector: the same iteration count as the reference (plus one: it reports one fewer per
    call that converges inside a restart cycle) and the same solution within the GMRES tolerance."""
    fx = RF.load(name)
    d = RF.write_datain(fx, str(tmp_path / "datain"))
    o = HDGOracle(d, MODELS[str(fx["model"])]())
    assert o.ppdegree > 1
    o.randvect = RF.reference_randvect(o)
    its, _ = o.newton()
    assert [its] == [int(v) for v in fx["solves"][:, 0]]
    assert [g.iters for g in o.gmres_log] == [int(fx["solves"][0, 1]) + 1]
    ref = fx["outuhat"][3:]
    assert np.linalg.norm(o.uh.ravel(order="F") - ref) / np.linalg.norm(ref) < o.gmres_tol

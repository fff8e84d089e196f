"""The LDG oracle (oracle/ldg.py) against the reference's own LDG runs (tests/golden/
ref_*_ldg*.npz from cput2cEXASIM with problem[0] = 0): the residual of one evaluation at 1e-12,
the DIRK steps of pseudo-transient solves to the PTC tolerance (with and without the
reduced-basis guess), the residual norms the reference
prints, and its GMRES counts."""
from __future__ import annotations

import numpy as np
import pytest

import ref_fixtures as RF
from oracle.hdg import dirk_coeff
from oracle.ldg import LDGOracle
from oracle.models import MODELS


def _oracle(fx, tmp_path):
    d = RF.write_datain(fx, str(tmp_path / "datain"))
    o = LDGOracle(d, MODELS[str(fx["model"])]())
    if o.ppdegree > 1:
        # the polynomial's Arnoldi process starts from the reference's own vector
        o.randvect = RF.reference_randvect(o, faces=False)
    return o


def _stage_setup(o, j, u):
    """The source and time of DIRK stage j of the first step with the state u unchanged
    since the step began (UpdateSource, updatesource.cpp:45-80)."""
    c, dd, tt = dirk_coeff(o.nstage, o.torder)
    S, dt = o.nstage, o.dt[0]
    sdg = u * (dd[0] / dt)
    for k in range(1, j + 1):
        if k == 1:
            sdg = u * (-dd[1] / dt) + sdg * ((dd[1] + dd[S + 1]) / dd[0])
        else:
            raise NotImplementedError
    o.time = o.factor[0] + dt * tt[j]
    o.dtfactor = dd[j * S + j] / dt
    o.sdg = sdg
    o.sdgg = np.einsum("gj,jce->gec", o.shapegt[:, :, 0], sdg)


@pytest.mark.parametrize("name", RF.ldg_names())
def test_ldg_residual_matches_reference(name, tmp_path):
    fx = RF.load(name)
    o = _oracle(fx, tmp_path)
    u = o.udg[:, :o.ncu].copy()
    _stage_setup(o, 1, u)
    R = o.residual_ldg(u).ravel(order="F")
    ref = fx["Ru_stage2_initial"]
    rel = np.linalg.norm(R - ref) / np.linalg.norm(ref)
    assert rel < 1e-12, rel


@pytest.mark.parametrize("name", RF.ldg_names())
def test_ldg_dirk_step_matches_reference(name, tmp_path):
    fx = RF.load(name)
    o = _oracle(fx, tmp_path)
    out = o.dirk_solve_ldg()
    udg_ref = fx["outudg"]
    nud = int(np.prod(udg_ref[:3]))
    u_ref = udg_ref[3:].reshape(-1, nud)[-1]
    u = o.udg.ravel(order="F")
    rel = np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref)
    assert rel < o.newton_tol, rel
    # per stage: PTC steps and the printed norms (6 significant digits) down to 1e-6
    lens = fx["ptc_lengths"].astype(int)
    norms = np.split(fx["ptc_norms"], np.cumsum(lens)[:-1])
    assert len(out) == len(norms)
    for (it, mine, gm), ref in zip(out, norms):
        assert len(mine) == len(ref), (mine, ref)
        for a, b in zip(mine, ref):
            if b > 1e-6:
                assert abs(a - b) <= 1e-5 * b, (a, b)
    # GMRES: the reference reports one step fewer per call that converges inside a cycle
    # (gmres.cpp:269-272 returns j before the loop's j++); finite-difference products move
    # the counts by a step or two more
    mine_g = [g for _, _, gm in out for g in gm]
    ref_g = [int(v) for v in fx["gmres_iters"]]
    assert len(mine_g) == len(ref_g)
    for a, b in zip(mine_g, ref_g):
        assert abs(a - (b + 1)) <= 3, (mine_g, ref_g)

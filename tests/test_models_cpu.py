"""CPU checks of the system models and periodic meshes used by the Navier-Stokes and
Euler parity cases: the oracle's complex-step Jacobians against central differences of its
own fluxes, and the face counts of the periodic grids (every face interior)."""
import numpy as np
import pytest

from exasim_b200 import inputs as I
from oracle.models import MODELS


def states(model, ng, rng):
    uq = rng.standard_normal((ng, model.nc)) * 0.1
    uq[:, 0] = 1.0 + 0.1 * rng.random(ng)
    uq[:, 1:model.ncu - 1] += 0.5
    uq[:, model.ncu - 1] = 5.0 + rng.random(ng)
    return uq


@pytest.mark.parametrize("name,param", [("ns2d", [1.4, 1600.0, 0.72, 0.3]), ("euler3d", [1.4, 0.5])])
def test_flux_jacobian_against_differences(name, param):
    m = MODELS[name]()
    rng = np.random.default_rng(0)
    ng = 7
    uq = states(m, ng, rng)
    x = rng.random((ng, m.nd))
    f, J = m.flux(x, uq, param, 0.0)
    assert f.shape == (ng, m.ncu, m.nd) and J.shape == (ng, m.ncu, m.nd, m.nc)
    h = 1e-6
    for k in range(m.nc):
        up, um = uq.copy(), uq.copy()
        up[:, k] += h
        um[:, k] -= h
        fd = (m.flux(x, up, param, 0.0)[0] - m.flux(x, um, param, 0.0)[0]) / (2 * h)
        assert np.abs(fd - J[..., k]).max() <= 1e-6 * max(1.0, np.abs(J).max())
    n = rng.standard_normal((ng, m.nd))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    uh = states(m, ng, rng)[:, :m.ncu]
    fb, fq, fh = m.fbou(1, x, uq, uh, n, [2.0], param, 0.0)
    for k in range(m.ncu):
        up, um = uh.copy(), uh.copy()
        up[:, k] += h
        um[:, k] -= h
        fd = (m.fbou(1, x, uq, up, n, [2.0], param, 0.0)[0] - m.fbou(1, x, uq, um, n, [2.0], param, 0.0)[0]) / (2 * h)
        assert np.abs(fd - fh[..., k]).max() <= 1e-6


@pytest.mark.parametrize("nd,n", [(2, 3), (2, 5), (3, 3)])
def test_periodic_grids_have_no_boundary(nd, n):
    g = I.periodic_square_quad_grid(n, 0.0, 2 * np.pi) if nd == 2 else I.periodic_cube_hex_grid(n, -5.0, 10.0)
    assert not I.boundary_faces(g).any()
    lf = I.elem_faces(nd, 1)
    keys = {tuple(sorted(g.tp[lf[:, l], e])) for e in range(g.ne) for l in range(lf.shape[1])}
    assert len(keys) == nd * n ** nd
    # element nodes keep the unidentified coordinates
    assert np.ptp(g.p[:, g.t].reshape(nd, -1), axis=1).max() > 0.9 * (2 * np.pi if nd == 2 else 10.0)

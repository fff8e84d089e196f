"""Oracle (test infrastructure only): numpy statements of the pointwise PDE models
used by the parity cases, written from the same ``pdemodel.txt`` math as the
generated-format model sources under ``exasim_b200/models/``.

Each model returns what Exasim's generated functions return, with Exasim's
argument roles (backend/Model/libpdemodel.hpp:3-41):

* ``flux(x, uq, param, t)``      -> f [ng, ncu, nd], df/duq [ng, ncu, nd, nc]   (HdgFlux)
* ``source(x, uq, param, t)``    -> s [ng, ncu], ds/duq [ng, ncu, nc]           (HdgSource)
* ``fbou(ib, x, uq, uh, n, tau, param, t)``
                                 -> fb [ng, ncu], dfb/duq [ng, ncu, nc],
                                    dfb/duh [ng, ncu, ncu]                       (HdgFbou)
* ``tdfunc`` / ``initu``         -> ones / initial u                           (KokkosTdfunc, cpuInitu)

The Jacobian layout is Exasim's: entry (out, in) at ``J[:, out, in]`` where the flux's
``out`` index runs over (component, dimension) with the component fastest.
"""
from __future__ import annotations

import numpy as np

PI = np.pi


class Poisson:
    """-div(kappa grad u) = s with q = -grad u, flux kappa*q (examples/Poisson/poisson{2,3}d/pdemodel.txt).

    Source 2 pi^2 sin(pi x) sin(pi y) in 2D, 3 pi^2 sin sin sin in 3D; boundary code 1 is
    FbouHdg = tau*(0 - uhat).
    """

    def __init__(self, nd):
        self.nd = nd
        self.ncu = 1
        self.nc = nd + 1

    def flux(self, x, uq, param, t):
        ng, nd = x.shape[0], self.nd
        kappa = param[0]
        f = np.zeros((ng, 1, nd))
        J = np.zeros((ng, 1, nd, self.nc))
        for d in range(nd):
            f[:, 0, d] = uq[:, 1 + d] * kappa
            J[:, 0, d, 1 + d] = kappa
        return f, J

    def source(self, x, uq, param, t):
        ng = x.shape[0]
        s = np.zeros((ng, 1))
        # same literals and operation order as exasim_b200/models/poisson{2,3}d/HdgSource.cpp
        if self.nd == 2:
            s[:, 0] = np.sin(x[:, 0] * 3.141592653589793) * np.sin(x[:, 1] * 3.141592653589793) * 1.973920880217872E+1
        else:
            s[:, 0] = (np.sin(x[:, 0] * 3.141592653589793) * np.sin(x[:, 1] * 3.141592653589793)
                       * np.sin(x[:, 2] * 3.141592653589793) * 2.960881320326807E+1)
        return s, np.zeros((ng, 1, self.nc))

    def fbou(self, ib, x, uq, uh, n, tau, param, t):
        ng = x.shape[0]
        if ib != 1:
            raise ValueError(f"boundary code {ib} not defined for this model")
        fb = np.zeros((ng, 1))
        fb[:, 0] = -tau[0] * uh[:, 0]
        Jh = np.zeros((ng, 1, 1))
        Jh[:, 0, 0] = -tau[0]
        return fb, np.zeros((ng, 1, self.nc)), Jh

    def tdfunc(self, x, uq, param, t):
        return np.ones((x.shape[0], 1))

    def initu(self, x, param):
        return np.zeros((x.shape[0], 1))


class ConvectionDiffusion:
    """div(c u + kappa q) = s, q = -grad u (pattern of
    examples/ConvectionDiffusion/BoundaryLayer/pdemodel.py).

    param = [kappa, c_1, ..., c_nd, x0_1..x0_nd, sigma]; source exp(-|x-x0|^2/(2 sigma^2));
    boundary code 1 is FbouHdg = tau*(0 - uhat).
    """

    def __init__(self, nd):
        self.nd = nd
        self.ncu = 1
        self.nc = nd + 1

    def flux(self, x, uq, param, t):
        ng, nd = x.shape[0], self.nd
        kappa = param[0]
        f = np.zeros((ng, 1, nd))
        J = np.zeros((ng, 1, nd, self.nc))
        for d in range(nd):
            c = param[1 + d]
            f[:, 0, d] = uq[:, 0] * c + uq[:, 1 + d] * kappa
            J[:, 0, d, 0] = c
            J[:, 0, d, 1 + d] = kappa
        return f, J

    def source(self, x, uq, param, t):
        nd = self.nd
        sig = param[1 + 2 * nd]
        r2 = np.zeros(x.shape[0])
        for d in range(nd):
            r2 = r2 + (x[:, d] - param[1 + nd + d]) ** 2
        s = np.exp(-r2 / (2 * sig * sig)).reshape(-1, 1)
        return s, np.zeros((x.shape[0], 1, self.nc))

    fbou = Poisson.fbou
    tdfunc = Poisson.tdfunc
    initu = Poisson.initu


MODELS = {"poisson2d": lambda: Poisson(2), "poisson3d": lambda: Poisson(3),
          "convdiff2d": lambda: ConvectionDiffusion(2), "convdiff3d": lambda: ConvectionDiffusion(3)}

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


def _cstep(fun, z, k0, k1, ng):
    """Columns k0..k1-1 of the Jacobian of fun at z [ng, nz] by complex steps (exact to
    rounding for analytic fun): J[..., k - k0] = Im fun(z + i h e_k) / h."""
    h = 1e-30
    cols = []
    for k in range(k0, k1):
        zc = z.astype(np.complex128)
        zc[:, k] += 1j * h
        cols.append(np.imag(fun(zc)) / h)
    return np.stack(cols, axis=-1)


class _PointModel:
    """A model given by a pointwise flux f(uq) [ng, ncu, nd] and boundary flux; its
    Jacobians are taken by complex steps, independently of the symbolic derivatives that
    the generated sources carry.  Source zero unless overridden; one boundary code (1):
    FbouHdg = f(u, q) . n + tau (u - uhat)."""

    def flux(self, x, uq, param, t):
        f = self._flux(uq, param).real
        return f, _cstep(lambda z: self._flux(z, param), uq, 0, self.nc, uq.shape[0])

    def source(self, x, uq, param, t):
        ng = x.shape[0]
        return np.zeros((ng, self.ncu)), np.zeros((ng, self.ncu, self.nc))

    def fbou(self, ib, x, uq, uh, n, tau, param, t):
        ncu, nc = self.ncu, self.nc

        def fb(z):
            f = self._flux(z[:, :nc], param)
            return np.einsum("pkd,pd->pk", f, n) + tau[0] * (z[:, :ncu] - z[:, nc:])

        z = np.concatenate([uq, uh], axis=1)
        J = _cstep(fb, z, 0, nc + ncu, z.shape[0])
        return fb(z).real, J[:, :, :nc], J[:, :, nc:]

    def tdfunc(self, x, uq, param, t):
        return np.ones((x.shape[0], self.ncu))


class NavierStokes2D(_PointModel):
    """Compressible Navier-Stokes in 2D, q = -grad u (examples/NavierStokes/TaylorGreenVortex/
    pdemodel.m with the z terms dropped); param = [gamma, Re, Pr, Minf].  Initial state: the
    2D Taylor-Green vortex rho = 1, u = sin x cos y, v = -cos x sin y,
    p = 1/(gamma Minf^2) + (cos 2x + cos 2y)/4."""

    def __init__(self):
        self.nd, self.ncu, self.nc = 2, 4, 12

    @staticmethod
    def _flux(uq, param):
        gam, Re, Pr, Minf = param[0], param[1], param[2], param[3]
        gam1 = gam - 1.0
        M2 = Minf * Minf
        fc = 1.0 / (gam1 * M2 * Re * Pr)
        r, ru, rv, rE = uq[:, 0], uq[:, 1], uq[:, 2], uq[:, 3]
        rx, rux, rvx, rEx = uq[:, 4], uq[:, 5], uq[:, 6], uq[:, 7]
        ry, ruy, rvy, rEy = uq[:, 8], uq[:, 9], uq[:, 10], uq[:, 11]
        uv, vv = ru / r, rv / r
        ke = 0.5 * (uv * uv + vv * vv)
        p = gam1 * (rE - r * ke)
        h = rE / r + p / r
        ux, vx = (rux - rx * uv) / r, (rvx - rx * vv) / r
        uy, vy = (ruy - ry * uv) / r, (rvy - ry * vv) / r
        px = gam1 * (rEx - rx * ke - r * (uv * ux + vv * vx))
        py = gam1 * (rEy - ry * ke - r * (uv * uy + vv * vy))
        Tx = gam * M2 * (px * r - p * rx) / (r * r)
        Ty = gam * M2 * (py * r - p * ry) / (r * r)
        txx = (2.0 / 3.0) * (2 * ux - vy) / Re
        txy = (uy + vx) / Re
        tyy = (2.0 / 3.0) * (2 * vy - ux) / Re
        f = np.stack([np.stack([ru, ru * uv + p + txx, rv * uv + txy, ru * h + uv * txx + vv * txy + fc * Tx], 1),
                      np.stack([rv, ru * vv + txy, rv * vv + p + tyy, rv * h + uv * txy + vv * tyy + fc * Ty], 1)],
                     axis=2)
        return f

    def initu(self, x, param):
        gam, Minf = param[0], param[3]
        u = np.sin(x[:, 0]) * np.cos(x[:, 1])
        v = -np.cos(x[:, 0]) * np.sin(x[:, 1])
        p = 1.0 / (gam * Minf * Minf) + (np.cos(2 * x[:, 0]) + np.cos(2 * x[:, 1])) / 4
        return np.stack([np.ones_like(u), u, v, p / (gam - 1) + 0.5 * (u * u + v * v)], axis=1)


class Euler3D(_PointModel):
    """Compressible Euler in 3D, no q (ModelC; examples/Euler/EulerVortex/pdemodel.py extended
    to 3D); param = [gamma, Minf].  Initial state: the isentropic vortex of strength 5 about
    the z axis at t = 0, no z velocity."""

    def __init__(self):
        self.nd, self.ncu, self.nc = 3, 5, 5

    @staticmethod
    def _flux(uq, param):
        gam1 = param[0] - 1.0
        r, ru, rv, rw, rE = (uq[:, k] for k in range(5))
        uv, vv, wv = ru / r, rv / r, rw / r
        p = gam1 * (rE - 0.5 * r * (uv * uv + vv * vv + wv * wv))
        h = rE / r + p / r
        return np.stack([np.stack([ru, ru * uv + p, rv * uv, rw * uv, ru * h], 1),
                         np.stack([rv, ru * vv, rv * vv + p, rw * vv, rv * h], 1),
                         np.stack([rw, ru * wv, rv * wv, rw * wv + p, rw * h], 1)], axis=2)

    def ubou(self, ib, x, uq, n, tau, param, t):
        """KokkosUbou of the model: uhat = u on every boundary."""
        return uq[:, :self.ncu].copy()

    def fbou_ldg(self, ib, x, uq, uh, n, tau, param, t):
        """KokkosFbou of the model: f(u) . n + tau (u - uhat)."""
        f = self._flux(uq[:, :self.nc], param)
        return np.einsum("pkd,pd->pk", f, n) + tau[0] * (uq[:, :self.ncu] - uh)

    def initu(self, x, param):
        gam, M = param[0], param[1]
        phi = 5.0
        r2 = x[:, 0] ** 2 + x[:, 1] ** 2
        rho = (1 - ((gam - 1) / (16 * PI ** 2)) * phi ** 2 * np.exp(2 * (1 - r2))) ** (1 / (gam - 1))
        ru = rho * (1 - phi * np.exp(1 - r2) * x[:, 1] / (2 * PI * M))
        rv = rho * phi * np.exp(1 - r2) * x[:, 0] / (2 * PI * M)
        p = rho ** gam / (gam * M * M)
        return np.stack([rho, ru, rv, np.zeros_like(rho), p / (gam - 1) + 0.5 * (ru * ru + rv * rv) / rho], axis=1)


class ConvectionDiffusionSin2D(ConvectionDiffusion):
    """The served stream's model: flux kappa q + c u, source sin(a pi x) sin(b pi y);
    param = [kappa, c_x, c_y, a, b]; boundary code 1 is FbouHdg = tau*(0 - uhat)."""

    def __init__(self):
        super().__init__(2)

    def source(self, x, uq, param, t):
        s = (np.sin(param[3] * PI * x[:, 0]) * np.sin(param[4] * PI * x[:, 1])).reshape(-1, 1)
        return s, np.zeros((x.shape[0], 1, self.nc))


MODELS = {"poisson2d": lambda: Poisson(2), "poisson3d": lambda: Poisson(3),
          "convdiff2d": lambda: ConvectionDiffusion(2), "convdiff3d": lambda: ConvectionDiffusion(3),
          "ns2d": NavierStokes2D, "euler3d": Euler3D, "cdsin2d": ConvectionDiffusionSin2D}

"""CPU restatement of the reference's LDG discretisation and its pseudo-transient (PTC) solver.

Test infrastructure only (the checker of the CUDA LDG path): tests/, smoke() and bench.py's CPU
leg use it; nothing in exasim_b200/ imports it.

The path, for models without q (ncq = 0, the reference's ModelC):

* Residual (backend/Discretization/residual.cpp:252-293, 589-617): uhat on the faces
  (GetUhat, getuhat.cpp:64-150: the average of the two sides at the face nodes inside, the
  model's Ubou at the face nodes on the boundary), the element integrals RuElem
  (uresidual.cpp:45-130, the HDG volume residual's quadrature), the face integrals RuFace
  (uresidual.cpp:259-334 with FhatDriver / FbouDriver, backend/Model/KokkosDrivers.cpp:349-438:
  the averaged flux dotted with the normal plus tau times the jump inside, the model's Fbou on
  the boundary), their sum into the elements (PutFaceNodes, kokkosimpl.h:1575-1603: side 1
  minus, side 2 plus), then Ru <- -Ru and, time-dependent, Ru <- Ru / dtfactor.
* The Jacobian-vector product by a finite difference of residuals (MatVec, matvec.cpp:41-100).
* The preconditioner: identity (precMatrixType 0) or the element mass inverse per component
  (ApplyMatrix, applymatrix.cpp:66-98; preconditioner.cpp:130-137; the element's own inverse
  mass matrix, which for an affine element equals the reference's master inverse over the
  element's jacobian up to rounding).
* GMRES on J x = -R (gmres.cpp:140-318), the PTC loop (ptcsolver.cpp:53-120, 255-330) with
  its reduced-basis guess (preconditioner.cpp:78-128), the polynomial preconditioner of
  degree ppdegree (getpoly.cpp:176-200, gmres.cpp:90-176), and the DIRK stages around it
  (solution.cpp:451-527).

Models with q are not restated: the reference's GetQ (residual.cpp:74-127) calls RuFace for
the q face term where qresidual.cpp's RqFace and the GetQ timing label name RqFace, so the
reference's own output is no parity target there.
"""
from __future__ import annotations

import numpy as np

from oracle.hdg import HDGOracle, GmresInfo, _givens, _backsolve, _F, _read_blob, dirk_coeff
import os


class LDGOracle(HDGOracle):
    def __init__(self, datain: str, model, verbose: bool = False):
        super().__init__(datain, model, verbose)
        if self.ncq != 0:
            raise NotImplementedError("LDG with q (ncq > 0)")
        m = _read_blob(os.path.join(datain, "master.bin"))
        npf, nd = self.npf, self.nd
        self.shapfnt = _F(m[8], (npf, npf, nd))
        self.matvec_order = int(self.flag[4])
        self.prec_matrix = int(self.flag[7])
        self.matvec_tol = float(self.solversparam[2])
        self.ntau = self.tau.size
        if self.prec_matrix != 0:
            sgds = np.einsum("jgd,gi->jigd", self.shapegw, self.shapegt[:, :, 0])
            mass = np.einsum("jig,ge->jie", sgds[:, :, :, 0], self.jac)
            from oracle.hdg import _inverse
            self.Minv = _inverse(mass)
        self._boundary_geometry()

    # ------------------------------------------------------------------ geometry
    def _boundary_geometry(self):
        """Face-node coordinates and normals of the boundary faces (UhatBlock,
        getuhat.cpp:121-136: shapfnt in place of the face Gauss basis)."""
        npf, nd, ncx = self.npf, self.nd, self.ncx
        e1, l1, e2 = self.f2e[0], self.f2e[1], self.f2e[2]
        self.bfaces = np.nonzero(e2 < 0)[0]
        xb = []
        nb = []
        for f in self.bfaces:
            x = self.xdg[self.perm[:, l1[f]], :, e1[f]]                     # [npf, ncx]
            xn = self.shapfnt[:, :, 0] @ x
            J = np.einsum("gjr,jc->gcr", self.shapfnt[:, :, 1:], x)        # [npf, x, r]
            jac, nl = self._facegeom(J[:, None, :, :, None])
            xb.append(xn)
            nb.append(nl[:, 0, :, 0])
        self.xbn = xb
        self.nbn = nb

    # ------------------------------------------------------------------ residual
    def residual_ldg(self, u):
        """Ru [npe, ncu, ne] of the state u [npe, ncu, ne] (Residual, residual.cpp:589-617)."""
        npe, ncu, ne, npf, ngf, nd = self.npe, self.ncu, self.ne, self.npf, self.ngf, self.nd
        udg = u.copy()
        Rv, _, _ = self._volume(udg, jacobian=False)                      # [npe, ne, ncu]
        Ru = np.transpose(Rv, (0, 2, 1)).copy()                            # [npe, ncu, ne]
        Rh = self.face_residual(udg)                                       # [npf, ncu, nf]
        fc = self.facecon                                                  # [2, npf, nf]
        R2 = np.transpose(Ru, (2, 0, 1)).reshape(ne * npe, ncu)            # row e*npe + node
        Rf = np.transpose(Rh, (2, 0, 1)).reshape(-1, ncu)                   # row f*npf + a
        k1 = fc[0].T.ravel()
        k2 = fc[1].T.ravel()
        inner = np.repeat(self.f2e[2] >= 0, npf)
        np.subtract.at(R2, k1, Rf)
        np.add.at(R2, k2[inner], Rf[inner])
        Ru = np.transpose(R2.reshape(ne, npe, ncu), (1, 2, 0)).copy()
        Ru = -1.0 * Ru
        if self.tdep:
            Ru = (1.0 / self.dtfactor) * Ru
        return Ru

    def face_residual(self, udg):
        """Rh [npf, ncu, nf] = shapfgw . (jac fhat) per face (RuFaceBlock)."""
        npe, ncu, nc, npf, ngf, nd, nf = self.npe, self.ncu, self.nc, self.npf, self.ngf, self.nd, self.nf
        fc = self.facecon
        e1, l1, e2 = self.f2e[0], self.f2e[1], self.f2e[2]
        ub = udg.transpose(2, 0, 1).reshape(self.ne * npe, nc)             # row e*npe + node
        u1 = ub[fc[0]]                                                     # [npf, nf, nc]
        u2 = ub[fc[1]]
        S = self.shapfgt[:, :, 0]
        ug1 = np.einsum("ga,afc->gfc", S, u1)
        ug2 = np.einsum("ga,afc->gfc", S, u2)
        xg = np.transpose(self.xgf[:, l1, :, e1], (1, 0, 2))                  # [ngf, nf, ncx]
        nl = np.transpose(self.nlf[:, l1, :, e1], (1, 0, 2))                  # [ngf, nf, nd]
        jac = self.jacf[:, l1, e1]                                         # [ngf, nf]
        X = xg.reshape(-1, self.ncx)
        f1, _ = self.model.flux(X, ug1.reshape(-1, nc), self.param, self.time)
        f2, _ = self.model.flux(X, ug2.reshape(-1, nc), self.param, self.time)
        f1 = f1.reshape(ngf, nf, ncu, nd)
        f2 = f2.reshape(ngf, nf, ncu, nd)
        avg = 0.5 * (f1 + f2)                                              # AverageFlux
        fh = avg[..., 0] * nl[:, :, None, 0]                               # AverageFluxDotNormal
        for d in range(1, nd):
            fh = fh + avg[..., d] * nl[:, :, None, d]
        du = ug1[..., :ncu] - ug2[..., :ncu]
        tau = self.tau
        if self.ntau <= 1:
            fh = fh + tau[0] * du
        elif self.ntau == ncu:
            fh = fh + tau[None, None, :] * du
        else:
            T = tau.reshape(ncu, ncu, order="F")                           # tau[k*ncu + j]
            fh = fh + np.einsum("kj,gfk->gfj", T, du)
        # boundary faces: Ubou at the face nodes, Fbou at the Gauss points
        for t, f in enumerate(self.bfaces):
            ib = int(self.bf[l1[f], e1[f]])
            uhn = self.model.ubou(ib, self.xbn[t], u1[:, f], self.nbn[t], tau, self.param, self.time)
            uhg = S @ uhn
            fh[:, f] = self.model.fbou_ldg(ib, xg[:, f], ug1[:, f], uhg, nl[:, f], tau, self.param, self.time)
        sg = fh * jac[:, :, None]                                          # ApplyJacFhat
        return np.einsum("ag,gfk->akf", self.shapfgw[:, :, 0], sg)          # [npf, ncu, nf]

    # ------------------------------------------------------------ linear solver
    def matvec_fd(self, u, Ru, v):
        """J(u) v by residual differences (MatVec, matvec.cpp:41-100)."""
        eps = self.matvec_tol
        if self.matvec_order == 1:
            w = 1.0 * u + eps * v
            return (1.0 / eps) * self.residual_ldg(w) + (-1.0 / eps) * Ru
        w = 1.0 * u + (-eps) * v
        Rm = self.residual_ldg(w)
        w = 1.0 * u + eps * v
        return (0.5 / eps) * self.residual_ldg(w) + (-0.5 / eps) * Rm

    def precond_ldg(self, x):
        if self.prec_matrix == 0:
            return x.copy()
        return np.einsum("ije,jke->ike", self.Minv, x)

    def gmres_ldg(self, u, b, x0=None):
        """GMRES for J x = -b (gmres.cpp:140-318) from x0 (zero if None); returns (x, iterations)."""
        shape = b.shape
        N = b.size
        bv = b.ravel(order="F")
        mv = lambda v: self.matvec_fd(u, b, v.reshape(shape, order="F")).ravel(order="F")
        pc0 = lambda v: self.precond_ldg(v.reshape(shape, order="F")).ravel(order="F")
        pc = pc0
        if self.ppdegree > 1:
            pc = self._poly_precond(mv, pc0, N)
        nrest, maxit = self.restart, self.gmres_maxit
        n1 = nrest + 1
        nrmb = np.sqrt(np.dot(bv, bv))
        x = np.zeros(N) if x0 is None else x0.ravel(order="F").copy()
        if np.sqrt(np.dot(x, x)) > 1e-12:
            r = -1.0 * bv + (-1.0) * mv(x)
            nrmr = np.sqrt(np.dot(r, r))
        else:
            r = -1.0 * bv + 0.0 * bv
            nrmr = nrmb
        tol = min(0.1, self.gmres_tol * (nrmb / nrmr))
        r = pc(r)
        nrmb = np.sqrt(np.dot(r, r))
        nrmr = nrmb
        V = np.zeros((N, n1))
        Hh = np.zeros((n1, nrest))
        j = 0
        relerr = 1.0
        while j < maxit:
            V[:, 0] = r * (1.0 / nrmr)
            s = np.zeros(n1)
            s[0] = nrmr
            cs = np.zeros(n1)
            sn = np.zeros(n1)
            i = 0
            while i < nrest and j < maxit:
                w = pc(mv(V[:, i]))
                h = Hh[:, i]
                if self.ortho == 0:
                    for k in range(i + 1):
                        h[k] = np.dot(w, V[:, k])
                        w = w - h[k] * V[:, k]
                else:
                    h[:i + 1] = V[:, :i + 1].T @ w
                    w = w - V[:, :i + 1] @ h[:i + 1]
                h[i + 1] = np.sqrt(np.dot(w, w))
                V[:, i + 1] = w * (1.0 / h[i + 1])
                _givens(h, s, cs, sn, i)
                relerr = abs(s[i + 1]) / nrmb
                if relerr < tol:
                    x = x + V[:, :i + 1] @ _backsolve(Hh, s, i)
                    return x.reshape(shape, order="F"), j + 1
                i += 1
                j += 1
            x = x + V[:, :nrest] @ _backsolve(Hh, s, nrest - 1)
            r = pc(-1.0 * bv + (-1.0) * mv(x))
            nrmr = np.sqrt(np.dot(r, r))
            relerr = nrmr / nrmb
            if relerr < tol:
                return x.reshape(shape, order="F"), j
        return x.reshape(shape, order="F"), j

    def _rb_guess_ldg(self, u, b):
        """ComputeInitialGuessAndPreconditioner, LDG form (preconditioner.cpp:78-128): U_i = J W_i
        for the newest basis vector, coef = (U^T U)^-1 U^T b, x = -W coef."""
        cur = self.rb_cur
        i = self.rb_removed - 1 if self.rb_removed > 0 else cur - 1
        shape = b.shape
        self.rb_U[:, i] = self.matvec_fd(u, b, self.rb_W[:, i].reshape(shape, order="F")).ravel(order="F")
        U, W = self.rb_U[:, :cur], self.rb_W[:, :cur]
        coef = np.linalg.inv(U.T @ U) @ (U.T @ b.ravel(order="F"))
        return (-(W @ coef)).reshape(shape, order="F")

    def _poly_precond(self, mv, pc0, N):
        """getPoly (getpoly.cpp:176-200: m Arnoldi steps of P J from randvect, the harmonic Ritz
        values in Leja order, with GMRES's post-processing, gmres.cpp:163-176) and ApplyPoly
        (gmres.cpp:90-130) after the preconditioner, as the HDG oracle's GMRES applies them."""
        from oracle.poly import poly_ritz
        m = self.ppdegree
        Vp = np.zeros((N, m + 1))
        Hp = np.zeros((m + 1, m))
        rv = self.randvect.ravel(order="F")
        Vp[:, 0] = rv / np.sqrt(np.dot(rv, rv))
        for jj in range(m):
            w = pc0(mv(Vp[:, jj]))
            for k in range(jj + 1):
                Hp[k, jj] = np.dot(w, Vp[:, k])
                w = w - Hp[k, jj] * Vp[:, k]
            Hp[jj + 1, jj] = np.sqrt(np.dot(w, w))
            Vp[:, jj + 1] = w / Hp[jj + 1, jj]
        sr, si = poly_ritz(Hp)

        def pc(v):
            w = pc0(v)
            q = w.copy()
            w = np.zeros_like(q)
            i = 0
            while i < m - 1:
                if si[i] == 0:
                    w = w + q / sr[i]
                    q = q - pc0(mv(q)) / sr[i]
                    i += 1
                else:
                    a2b2 = sr[i] ** 2 + si[i] ** 2
                    p = 2 * sr[i] * q - pc0(mv(q))
                    w = w + p / a2b2
                    if i < m - 2:
                        q = q - pc0(mv(p)) / a2b2
                    i += 2
            if si[m - 1] == 0:
                w = w + q / sr[m - 1]
            return w
        return pc

    def ptc(self, maxit=None, tol=None):
        """PTCsolver (ptcsolver.cpp:255-330) with LinearSolver (:53-120): the reduced-basis guess
        when RBdim > 0 (kept if R(u + x) <= 1.05 |R(u)|, the step itself below the tolerance),
        GMRES from it, UpdateRB after GMRES steps; returns (iterations, norms, gmres)."""
        maxit = self.newton_maxit if maxit is None else maxit
        tol = self.newton_tol if tol is None else tol
        ncu = self.ncu
        u = self.udg[:, :ncu].copy()
        r = self.residual_ldg(u)
        norms = [np.linalg.norm(r)]
        gm = []
        it = 0
        for it in range(maxit):
            status = 0
            x0 = None
            if self.RBdim > 0 and self.rb_cur > 0:
                oldnrm = norms[-1]
                x0 = self._rb_guess_ldg(u, r)
                nv = np.linalg.norm(self.residual_ldg(1.0 * u + 1.0 * x0))
                if nv > 1.05 * oldnrm:
                    x0 = 0.0 * x0
                    self.rb_removed = 0
                    self.rb_cur = 0
                if nv < tol:
                    status = 1
            if status == 0:
                x, nit = self.gmres_ldg(u, r, x0)
                gm.append(nit)
            else:
                x = x0
            u = u + 1.0 * x
            r = self.residual_ldg(u)
            nrmr = np.linalg.norm(r)
            norms.append(nrmr)
            if not nrmr <= 1.0e6:
                raise FloatingPointError("PTC residual above 1e6 or NaN")
            if status == 0 and self.RBdim > 0:
                self._rb_update(x)
            if nrmr < tol:
                break
        self.udg[:, :ncu] = u
        return it, norms, gm

    def dirk_solve_ldg(self, nsteps=None):
        """DIRK time stepping around PTC (solution.cpp:451-527); per-stage (iterations, norms, gmres)."""
        ncu = self.ncu
        c, dvec, tt = dirk_coeff(self.nstage, self.torder)
        S = self.nstage
        dd = dvec
        nsteps = len(self.dt) if nsteps is None else nsteps
        time = self.factor[0]
        out = []
        for istep in range(nsteps):
            dt = self.dt[istep]
            udgprev = self.udg[:, :ncu].copy()
            utmp = (1.0 - c.sum()) * udgprev
            for j in range(S):
                self.time = time + dt * tt[j]
                self.dtfactor = dd[j * S + j] / dt
                u = self.udg[:, :ncu].copy()
                if j == 0:
                    self.sdg = u * (dd[0] / dt)
                elif j == 1:
                    sc = (dd[1] + dd[S + 1]) / dd[0]
                    self.sdg = u * (-dd[1] / dt) + self.sdg * sc
                elif j == 2:
                    sc = dd[2] / dd[1]
                    pc = dd[2] + dd[S + 2] + dd[2 * S + 2] - sc * (dd[1] + dd[S + 1])
                    self.sdg = u * (-dd[S + 2] / dt) + self.sdg * sc + udgprev * (pc / dt)
                else:
                    raise NotImplementedError("DIRK stage > 3")
                self.sdgg = np.einsum("gj,jce->gec", self.shapegt[:, :, 0], self.sdg)
                out.append(self.ptc())
                utmp = utmp + c[j] * self.udg[:, :ncu]
            self.udg[:, :ncu] = utmp
            time = time + dt
        return out

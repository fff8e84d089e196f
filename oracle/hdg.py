"""Oracle (test infrastructure only): a numpy restatement of Exasim's HDG implicit
hot path, used by tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg to check the CUDA solver in ``exasim_b200``.  Nothing in the product imports it.

It follows the reference's algorithm and data layouts step by step (column-major
arrays, first index fastest; numpy arrays here carry the same axis order):

* inputs        backend/Discretization/readbinaryfiles.cpp:65-618 (app/master/mesh/sol)
* connectivity  backend/Discretization/connectivity.cpp:1212-1385 (oracle/conn.cpp)
* geometry      backend/Discretization/geometry.cpp:44-222, kokkosimpl.h:2321-2415
* q-equation    backend/Discretization/qequation.cpp:66-370 (Minv*C, Minv*E), :372-484 (hdgGetQ)
* assembly      backend/Discretization/uequation.cpp:45-203 (volume), :206-557 (faces + BCs),
                :559-775 (Schur condensation), :790-1088 (residual only)
* linear system backend/Discretization/matvec.cpp:103-117 (RHS), :190-217 (block Jacobi),
                :168-188 (elemental additive Schwarz), :219-238 (dudg), :240-389 (matvec)
* GMRES         backend/Solver/gmres.cpp:361-597, getpoly.cpp:33-65 (MGS), gmres.cpp:81-89 (CGS),
                backend/Common/cpuimpl.h:167-208 (Givens, back solve)
* Newton        backend/Solution/solution.cpp:125-243
* DIRK          backend/Solution/updatesource.cpp:32-80, updatesolution.cpp:118-160,
                previoussolutions.cpp:23-45, timestepcoeff.cpp:35-104

The dense element inverses use LAPACK getrf+getri as the reference's CPU path does
(backend/Common/pblas.h:234-246).  Parity is pinned by the reference's own golden
solution examples/Poisson/poisson3d/dataout/outuhat_np0.bin (tests/test_oracle_golden.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np
from scipy.linalg import lapack

HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(HERE, "_build")
_CONN = None


def build():
    """Compile the connectivity restatement (oracle/conn.cpp) into oracle/_build/."""
    os.makedirs(_BUILD, exist_ok=True)
    so = os.path.join(_BUILD, "libexa_oracle_conn.so")
    src = os.path.join(HERE, "conn.cpp")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", src, "-o", so])
    return so


def _conn_lib():
    global _CONN
    if _CONN is None:
        _CONN = ctypes.CDLL(build())
        _CONN.oracle_build_conn.restype = ctypes.c_int
    return _CONN


def _F(a, shape):
    return np.asarray(a).reshape(shape, order="F")


def _read_blob(fn):
    a = np.fromfile(fn, dtype=np.float64)
    ls = int(a[0])
    nsize = a[1:1 + ls].astype(np.int64)
    out, o = [nsize], 1 + ls
    for n in nsize:
        out.append(a[o:o + n])
        o += n
    return out


def _inverse(A):
    """Explicit inverse via LAPACK getrf + getri (pblas.h:234-246), batched over the last axis."""
    n = A.shape[0]
    out = np.empty_like(A)
    for k in range(A.shape[2]):
        lu, piv, info = lapack.dgetrf(A[:, :, k])
        if info != 0:
            raise np.linalg.LinAlgError(f"singular block {k}")
        inv, info = lapack.dgetri(lu, piv)
        out[:, :, k] = inv
    return out


def dirk_coeff(nstage, torder):
    """DIRK tables (timestepcoeff.cpp:35-104): returns (c, d [nstage, nstage] col-major, t)."""
    tabs = {
        (1, 1): ([1.0], [1.0], [1.0]),
        (1, 2): ([2.0], [2.0], [0.5]),
        (2, 2): ([0.0, 1.0], [3.414213562373096, -8.242640687119289, 0.0, 3.414213562373096],
                 [0.292893218813452, 1.0]),
        (2, 3): ([1.098076211353316, 0.633974596215561],
                 [1.267949192431123, 0.928203230275509, 0.0, 1.267949192431123],
                 [0.788675134594813, 0.211324865405187]),
        (3, 3): ([0.0, 0.0, 1.0],
                 [2.294280360323567, -1.484721005721436, -8.556127801733982, 0.0,
                  2.294280360323568, 3.391748836909791, 0.0, 0.0, 2.294280360323567],
                 [0.435866521500000, 0.717933260750000, 1.000000000000000]),
    }
    c, d, t = tabs[(nstage, torder)]
    return np.array(c), np.array(d), np.array(t)


@dataclass
class GmresInfo:
    iters: int
    relerr: float
    tol: float


class HDGOracle:
    """The reference's single-rank HDG discretisation and solver on CPU."""

    def __init__(self, datain: str, model, verbose: bool = False):
        self.model = model
        self.verbose = verbose
        self._read(datain)
        self._connect()
        self._geometry()
        self._init_solution()
        if self.ncq > 0:
            self._qequation()
        self.time = self.factor[0] if self.tdep else 0.0
        self.dtfactor = 0.0
        self.sdg = None

    # ------------------------------------------------------------------ inputs
    def _read(self, d):
        app = _read_blob(os.path.join(d, "app.bin"))
        self.ndims_app = app[1].astype(int)
        self.flag = app[2].astype(int)
        self.problem = app[3].astype(int)
        self.uinf = app[4]
        self.dt = app[5]
        self.factor = app[6]
        self.param = app[7]
        self.solversparam = app[8]
        self.tau = app[9]
        nd_a = self.ndims_app
        self.nc, self.ncu, self.ncq = nd_a[5], nd_a[6], nd_a[7]
        self.nco, self.ncx, self.ncw = nd_a[9], nd_a[11], nd_a[13]
        if self.nco != 0 or self.ncw != 0:
            raise NotImplementedError("odg/wdg fields are outside the HDG hot path")
        self.tdep, self.wave = self.flag[0], self.flag[1]
        self.preconditioner = self.flag[6]
        self.ortho = self.flag[5]
        self.tdfunc = self.flag[10]
        self.newton_maxit = self.problem[13]
        self.gmres_maxit = self.problem[14]
        self.restart = self.problem[15]
        # reduced-basis initial guess of GMRES (ptcsolver.cpp:217-236, 374-379;
        # preconditioner.cpp:133-181): the last RBdim Newton updates
        self.RBdim = int(self.problem[16]) if self.problem.size > 16 else 0
        self.ppdegree = int(self.problem[27]) if self.problem.size > 27 else 0
        self.randvect = None  # start vector of the polynomial's Arnoldi process (ppdegree > 1)
        self.poly_sr = self.poly_si = None
        self.rb_W = self.rb_U = None
        self.rb_cur = self.rb_removed = 0
        self.torder, self.nstage = self.problem[3], self.problem[4]
        self.newton_tol = self.solversparam[0]
        self.gmres_tol = self.solversparam[1]

        m = _read_blob(os.path.join(d, "master.bin"))
        mnd = m[1].astype(int)
        self.nd, self.elemtype, self.porder = mnd[0], mnd[1], mnd[3]
        self.npe, self.npf, self.nge, self.ngf = mnd[5], mnd[6], mnd[7], mnd[8]
        nd, npe, npf, nge, ngf = self.nd, self.npe, self.npf, self.nge, self.ngf
        self.shapegt = _F(m[2], (nge, npe, nd + 1))
        self.shapegw = _F(m[3], (npe, nge, nd + 1))
        self.shapfgt = _F(m[4], (ngf, npf, nd))
        self.shapfgw = _F(m[5], (npf, ngf, nd))
        self.xpf = _F(m[13], (npf, max(nd - 1, 1)))

        me = _read_blob(os.path.join(d, "mesh.bin"))
        ns = me[0]
        self.ne = int(me[1][1])
        self.nfe = int(me[1][4])
        if ns[1] != 0:
            raise NotImplementedError("pre-connected mesh.bin; this oracle reads the raw-t form")
        self.perm = _F(me[24], (npf, self.nfe)).astype(np.int64)
        self.bf = _F(me[25], (self.nfe, self.ne)).astype(np.int64)
        nve = ns[26] // self.ne
        self.t = _F(me[27], (nve, self.ne)).astype(np.int64)
        # Cartesian sub-domains for block ILU(0) (readbinaryfiles.cpp:356)
        self.cartgridpart = me[26].astype(np.int64) if ns[25] > 0 else np.zeros(0, dtype=np.int64)

        s = _read_blob(os.path.join(d, "sol.bin"))
        self.xdg = _F(s[2], (npe, self.ncx, self.ne))
        self.udg0 = s[3] if len(s) > 3 else np.zeros(0)
        self.uh0 = s[6] if len(s) > 6 else np.zeros(0)

    # ------------------------------------------------------------ connectivity
    def _connect(self):
        lib = _conn_lib()
        ne, nfe, npf, npe = self.ne, self.nfe, self.npf, self.npe
        t = np.ascontiguousarray(self.t.ravel(order="F"), dtype=np.int32)
        bf = np.ascontiguousarray(self.bf.ravel(order="F"), dtype=np.int32)
        perm = np.ascontiguousarray(self.perm.ravel(order="F"), dtype=np.int32)
        xpf = np.ascontiguousarray(self.xpf.ravel(order="F"), dtype=np.float64)
        f2e = np.zeros(4 * nfe * ne, dtype=np.int32)
        elemcon = np.zeros(npf * nfe * ne, dtype=np.int32)
        facecon = np.zeros(2 * npf * nfe * ne, dtype=np.int32)
        nf0 = ctypes.c_int(0)
        P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        nf = lib.oracle_build_conn(P(t), P(bf), P(perm), P(xpf), int(self.nd), int(self.elemtype),
                                   int(ne), int(npe), int(npf), P(f2e), P(elemcon), P(facecon),
                                   ctypes.byref(nf0))
        if nf < 0:
            raise RuntimeError("mesh connectivity is wrong")
        self.nf = nf
        self.nf0 = nf0.value
        self.f2e = _F(f2e[:4 * nf], (4, nf)).astype(np.int64)
        self.elemcon = _F(elemcon, (npf * nfe, ne)).astype(np.int64)
        self.facecon = _F(facecon[:2 * npf * nf], (2, npf, nf)).astype(np.int64)

    # ---------------------------------------------------------------- geometry
    def _geometry(self):
        nd, npe, npf, nge, ngf, ne, nfe = self.nd, self.npe, self.npf, self.nge, self.ngf, self.ne, self.nfe
        x = self.xdg                                                    # [npe, nd, ne]
        self.xg = np.einsum("gj,jce->gce", self.shapegt[:, :, 0], x)     # [nge, ncx, ne]
        Jg = np.einsum("gjr,jce->gcre", self.shapegt[:, :, 1:], x)       # [nge, x, r, ne]
        self.jac, self.Xx = self._elemgeom(Jg)
        # element faces: xdg at face nodes through perm (kokkosimpl.h:984-997)
        xf = x[self.perm.ravel(order="F")].reshape(npf, nfe, nd, ne, order="F")
        self.xgf = np.einsum("gj,jlce->glce", self.shapfgt[:, :, 0], xf)  # [ngf, nfe, ncx, ne]
        Jf = np.einsum("gjr,jlce->glcre", self.shapfgt[:, :, 1:], xf)     # [ngf, nfe, x, r, ne]
        self.jacf, self.nlf = self._facegeom(Jf)                          # [ngf,nfe,ne], [ngf,nfe,nd,ne]

    def _elemgeom(self, J):
        """ElemGeom2D/3D (kokkosimpl.h:2329-2360): jac and Xx[g, j + nd*m] = jac * dxi_m/dx_j."""
        nd = self.nd
        nge, ne = J.shape[0], J.shape[3]
        Xx = np.zeros((nge, nd * nd, ne))
        if nd == 1:
            jac = J[:, 0, 0]
            Xx[:, 0] = 1.0
        elif nd == 2:
            J11, J12, J21, J22 = J[:, 0, 0], J[:, 1, 0], J[:, 0, 1], J[:, 1, 1]
            jac = J11 * J22 - J12 * J21
            Xx[:, 0] = J22        # Xx11
            Xx[:, 1] = -J21       # Xx21 = jac * dxi/dy
            Xx[:, 2] = -J12       # Xx12 = jac * deta/dx
            Xx[:, 3] = J11        # Xx22
        else:
            J11, J12, J13 = J[:, 0, 0], J[:, 1, 0], J[:, 2, 0]
            J21, J22, J23 = J[:, 0, 1], J[:, 1, 1], J[:, 2, 1]
            J31, J32, J33 = J[:, 0, 2], J[:, 1, 2], J[:, 2, 2]
            jac = (J11 * J22 * J33 - J11 * J32 * J23 + J21 * J32 * J13 - J21 * J12 * J33
                   + J31 * J12 * J23 - J31 * J22 * J13)
            Xx[:, 0] = J22 * J33 - J23 * J32
            Xx[:, 1] = J23 * J31 - J21 * J33
            Xx[:, 2] = J21 * J32 - J22 * J31
            Xx[:, 3] = J13 * J32 - J12 * J33
            Xx[:, 4] = J11 * J33 - J13 * J31
            Xx[:, 5] = J12 * J31 - J11 * J32
            Xx[:, 6] = J12 * J23 - J13 * J22
            Xx[:, 7] = J13 * J21 - J11 * J23
            Xx[:, 8] = J11 * J22 - J12 * J21
        return jac, Xx

    def _facegeom(self, J):
        """FaceGeom1D/2D/3D (kokkosimpl.h:2362-2415)."""
        nd = self.nd
        ngf, nfe, _, _, ne = J.shape
        nl = np.zeros((ngf, nfe, nd, ne))
        if nd == 1:
            jac = np.ones((ngf, nfe, ne))
            nl[:, :, 0] = 1.0
            nl[:, 0::2, 0] = -1.0      # FixNormal1D: even local faces point left
        elif nd == 2:
            Jx, Jy = J[:, :, 0, 0], J[:, :, 1, 0]
            jac = np.sqrt(Jx * Jx + Jy * Jy)
            nl[:, :, 0] = Jy / jac
            nl[:, :, 1] = -Jx / jac
        else:
            a1, a2, a3 = J[:, :, 0, 0], J[:, :, 1, 0], J[:, :, 2, 0]
            b1, b2, b3 = J[:, :, 0, 1], J[:, :, 1, 1], J[:, :, 2, 1]
            n1 = a2 * b3 - a3 * b2
            n2 = a3 * b1 - a1 * b3
            n3 = a1 * b2 - a2 * b1
            jac = np.sqrt(n1 * n1 + n2 * n2 + n3 * n3)
            nl[:, :, 0] = n1 / jac
            nl[:, :, 1] = n2 / jac
            nl[:, :, 2] = n3 / jac
        return jac, nl

    # ------------------------------------------------------------ solution init
    def _init_solution(self):
        npe, nc, ncu, ne = self.npe, self.nc, self.ncu, self.ne
        udg = np.zeros((npe, nc, ne))
        if self.udg0.size == npe * nc * ne:
            udg = _F(self.udg0, (npe, nc, ne)).copy()
        elif self.udg0.size == npe * ncu * ne:
            udg[:, :ncu] = _F(self.udg0, (npe, ncu, ne))
        else:
            xs = self.xdg.transpose(0, 2, 1).reshape(-1, self.ncx)
            u0 = self.model.initu(xs, self.param)                         # [npe*ne, ncu]
            udg[:, :ncu] = u0.reshape(npe, ne, ncu).transpose(0, 2, 1)
        self.udg = udg
        if self.uh0.size == ncu * self.npf * self.nf:
            self.uh = _F(self.uh0, (ncu, self.npf, self.nf)).copy()
        else:
            self.uh = self.get_face_nodes(self.udg)

    def get_face_nodes(self, udg):
        """uh from the first element of each face (kokkosimpl.h:901-915)."""
        e1, l1 = self.f2e[0], self.f2e[1]
        m = self.perm[:, l1]                                             # [npf, nf]
        return np.transpose(udg[m, :self.ncu, e1[None, :]], (2, 0, 1)).copy()   # [ncu, npf, nf]

    # --------------------------------------------------------------- q-equation
    def _qequation(self):
        """Minv*C and Minv*E per element and dimension (qequation.cpp:66-170, 255-338)."""
        nd, npe, npf, nfe, ne = self.nd, self.npe, self.npf, self.nfe, self.ne
        sgw, sgt = self.shapegw, self.shapegt
        # shapegwdotshapeg[j, i, g, d] = shapegw[j, g, d] * shapegt[g, i] (setstructs.cpp:495-505)
        sgds = np.einsum("jgd,gi->jigd", sgw, sgt[:, :, 0])
        mass = np.einsum("jig,ge->jie", sgds[:, :, :, 0], self.jac)
        self.Minv = _inverse(mass)
        C = np.zeros((npe, npe, ne, nd))
        for d in range(nd):
            w = np.zeros((npe, npe, ne))
            for r in range(nd):
                w += np.einsum("jig,ge->jie", sgds[:, :, :, 1 + r], self.Xx[:, d + nd * r])
            C[:, :, :, d] = np.einsum("ike,kje->ije", self.Minv, w)
        self.MinvC = C
        sfds = np.einsum("jg,gi->jig", self.shapfgw[:, :, 0], self.shapfgt[:, :, 0])   # [npf, npf, ngf]
        E = np.zeros((npe, npf * nfe, ne, nd))
        for d in range(nd):
            tg = self.nlf[:, :, d] * self.jacf                              # [ngf, nfe, ne]
            Etmp = np.einsum("kig,gle->kile", sfds, tg)                     # [npf, npf, nfe, ne]
            work = np.zeros((npe, npf, nfe, ne))
            for l in range(nfe):
                np.add.at(work, (self.perm[:, l], slice(None), l), Etmp[:, :, l])
            E[:, :, :, d] = np.einsum("ike,kje->ije", self.Minv, work.reshape(npe, npf * nfe, ne, order="F"))
        self.MinvE = E

    def get_q(self, udg, uh):
        """q = Minv*C*u - Minv*E*uhat per dimension (qequation.cpp:372-470)."""
        ncu, nd = self.ncu, self.nd
        u = udg[:, :ncu]                                                  # [npe, ncu, ne]
        uhe = self.gather_uh(uh, opt=1)                                   # [ndf, ncu, ne]
        for d in range(nd):
            q = np.einsum("ije,jce->ice", self.MinvC[:, :, :, d], u)
            q -= np.einsum("ije,jce->ice", self.MinvE[:, :, :, d], uhe)
            udg[:, ncu * (1 + d):ncu * (2 + d)] = q
        return udg

    def gather_uh(self, uh, opt):
        """GetElementFaceNodes through elemcon (kokkosimpl.h:999-1030).

        opt 0 -> [ndf, ne, ncu]; opt 1 -> [ndf, ncu, ne]; opt 2 -> [ncu, ndf, ne].
        """
        flat = uh.reshape(self.ncu, -1, order="F")                         # [ncu, npf*nf]
        g = flat[:, self.elemcon]                                          # [ncu, ndf, ne]
        if opt == 0:
            return np.transpose(g, (1, 2, 0))
        if opt == 1:
            return np.transpose(g, (1, 0, 2))
        return g

    # ----------------------------------------------------------------- assembly
    def _volume(self, udg, jacobian=True):
        """Volume quadrature of Ru (and D, B) (uequation.cpp:45-203, 790-880)."""
        nd, npe, nge, ne, ncu, nc = self.nd, self.npe, self.nge, self.ne, self.ncu, self.nc
        uqg = np.einsum("gj,jce->gec", self.shapegt[:, :, 0], udg)         # [nge, ne, nc]
        xg = np.transpose(self.xg, (0, 2, 1))                             # [nge, ne, ncx]
        X = xg.reshape(-1, self.ncx)
        UQ = uqg.reshape(-1, nc)
        s, s_uq = self.model.source(X, UQ, self.param, self.time)
        f, f_uq = self.model.flux(X, UQ, self.param, self.time)
        if self.tdep:
            sdgg = self.sdgg.reshape(-1, ncu)
            fg = sdgg - self.dtfactor * UQ[:, :ncu]
            td = self.model.tdfunc(X, UQ, self.param, self.time) if self.tdfunc == 1 else np.ones_like(fg)
            s = s + fg * td
            s_uq = s_uq.copy()
            for m in range(ncu):
                s_uq[:, m, m] += -self.dtfactor * td[:, m]
        s = s.reshape(nge, ne, ncu)
        f = f.reshape(nge, ne, ncu, nd)
        jac = self.jac                                                    # [nge, ne]
        Xx = self.Xx                                                      # [nge, nd*nd, ne]
        # ApplyXxJac (kokkosimpl.h:2105-2128): rg[g, 0] = s*jac, rg[g, 1+m] = sum_j f_j Xx[g, j+nd*m]
        rg = np.zeros((nge, nd + 1, ne, ncu))
        rg[:, 0] = s * jac[:, :, None]
        for m in range(nd):
            acc = f[:, :, :, 0] * Xx[:, 0 + nd * m, :, None]
            for j in range(1, nd):
                acc = acc + f[:, :, :, j] * Xx[:, j + nd * m, :, None]
            rg[:, 1 + m] = acc
        Ru = np.einsum("igd,gdek->iek", self.shapegw, rg)                  # [npe, ne, ncu]
        if not jacobian:
            return Ru, None, None
        s_uq = s_uq.reshape(nge, ne, ncu, nc)
        f_uq = f_uq.reshape(nge, ne, ncu, nd, nc)
        rj = np.zeros((nge, nd + 1, ne, ncu, nc))
        rj[:, 0] = s_uq * jac[:, :, None, None]
        for m in range(nd):
            acc = f_uq[:, :, :, 0] * Xx[:, 0 + nd * m, :, None, None]
            for j in range(1, nd):
                acc = acc + f_uq[:, :, :, j] * Xx[:, j + nd * m, :, None, None]
            rj[:, 1 + m] = acc
        # Gauss2Node with shapegwdotshapeg (setstructs.cpp:495-505), negated
        sgds = np.einsum("jgd,gi->jigd", self.shapegw, self.shapegt[:, :, 0])
        W = sgds.reshape(npe * npe, nge * (nd + 1), order="F")
        R = rj.reshape(nge * (nd + 1), ne * ncu * nc, order="F")
        DB = -(W @ R).reshape(npe, npe, ne, ncu, nc, order="F")
        D = DB[:, :, :, :, :ncu]
        B = DB[:, :, :, :, ncu:]
        return Ru, D, B

    def _faces(self, udg, uh, jacobian=True):
        """Element-face quadrature, numerical flux and boundary conditions (uequation.cpp:206-557)."""
        nd, npe, npf, ngf, nfe, ne, ncu, nc = (self.nd, self.npe, self.npf, self.ngf, self.nfe,
                                                self.ne, self.ncu, self.nc)
        perm = self.perm
        uhe = self.gather_uh(uh, opt=0).reshape(npf, nfe, ne, ncu, order="F")          # [npf, nfe, ne, ncu]
        ufe = udg[perm.ravel(order="F")].reshape(npf, nfe, nc, ne, order="F")
        uhg = np.einsum("gj,jlek->glek", self.shapfgt[:, :, 0], uhe)         # [ngf, nfe, ne, ncu]
        ug = np.einsum("gj,jlce->glec", self.shapfgt[:, :, 0], ufe)          # [ngf, nfe, ne, nc]
        xg = np.transpose(self.xgf, (0, 1, 3, 2))                           # [ngf, nfe, ne, ncx]
        nl = np.transpose(self.nlf, (0, 1, 3, 2))                           # [ngf, nfe, ne, nd]
        jac = self.jacf                                                     # [ngf, nfe, ne]
        npt = ngf * nfe * ne
        X = xg.reshape(npt, -1)
        UG = ug.reshape(npt, nc)
        UH = uhg.reshape(npt, ncu)
        NL = nl.reshape(npt, nd)
        # FhatDriver (ModelDrivers.cpp:789-849): flux at (uhat, q), dotted with n, + tau (u - uhat)
        UQh = UG.copy()
        UQh[:, :ncu] = UH
        f, f_uq = self.model.flux(X, UQh, self.param, self.time)
        fh = np.einsum("pkd,pd->pk", f, NL)
        fh_uq = np.einsum("pkdc,pd->pkc", f_uq, NL)
        fh_uh = fh_uq[:, :, :ncu].copy()
        fh_uq[:, :, :ncu] = 0.0
        tau = self.tau[0]
        fh = fh + tau * (UG[:, :ncu] - UH)
        for m in range(ncu):
            fh_uq[:, m, m] += tau
            fh_uh[:, m, m] -= tau
        jf = jac.reshape(npt)
        fh = fh * jf[:, None]
        fh_uq = fh_uq * jf[:, None, None]
        fh_uh = fh_uh * jf[:, None, None]
        fh = fh.reshape(ngf, nfe, ne, ncu)
        fh_uq = fh_uq.reshape(ngf, nfe, ne, ncu, nc)
        fh_uh = fh_uh.reshape(ngf, nfe, ne, ncu, ncu)
        w0 = self.shapfgw[:, :, 0]                                          # [npf, ngf]
        sfds = np.einsum("jg,gi->jig", w0, self.shapfgt[:, :, 0])           # [npf, npf, ngf]
        Rutmp = np.einsum("ig,glek->ilek", w0, fh)                          # [npf, nfe, ne, ncu]
        # Ru -= face terms on all faces (assembleRu, kokkosimpl.h:1650-1659)
        Ru_face = np.zeros((npe, ne, ncu))
        for l in range(nfe):
            np.add.at(Ru_face, perm[:, l], Rutmp[:, l])
        out = {"Ru_face": Ru_face}
        if jacobian:
            Dtmp = np.einsum("ijg,glekc->ijlekc", sfds, fh_uq)                 # [npf,npf,nfe,ne,ncu,nc]
            Ftmp = np.einsum("ijg,glekc->ijlekc", sfds, fh_uh)                 # [npf,npf,nfe,ne,ncu,ncu]
            Dface = np.zeros((npe, npe, ne, ncu, nc))
            Fface = np.zeros((npe, npf, nfe, ne, ncu, ncu))
            for l in range(nfe):
                p = perm[:, l]
                idx = np.ix_(p, p)
                Dface[idx[0], idx[1]] += Dtmp[:, :, l]
                np.add.at(Fface[:, :, l], p, Ftmp[:, :, l])
            out["Dface"] = Dface
            out["Fface"] = Fface.reshape(npe, npf * nfe, ne, ncu, ncu, order="F")
        # boundary faces: the trace equation uses Fbou instead (uequation.cpp:346-431)
        for ib in np.unique(self.bf[self.bf > 0]):
            ls, es = np.nonzero(self.bf == ib)
            Xb = xg[:, ls, es].reshape(-1, self.ncx)
            Ub = ug[:, ls, es].reshape(-1, nc)
            Hb = uhg[:, ls, es].reshape(-1, ncu)
            Nb = nl[:, ls, es].reshape(-1, nd)
            fb, fb_uq, fb_uh = self.model.fbou(int(ib), Xb, Ub, Hb, Nb, self.tau, self.param, self.time)
            jb = jac[:, ls, es].reshape(-1)
            nb = ls.size
            fb = (fb * jb[:, None]).reshape(ngf, nb, ncu)
            Rutmp[:, ls, es] = np.einsum("ig,gbk->ibk", w0, fb)
            if jacobian:
                fb_uq = (fb_uq * jb[:, None, None]).reshape(ngf, nb, ncu, nc)
                fb_uh = (fb_uh * jb[:, None, None]).reshape(ngf, nb, ncu, ncu)
                Dtmp[:, :, ls, es] = np.einsum("ijg,gbkc->ijbkc", sfds, fb_uq)
                Ftmp[:, :, ls, es] = np.einsum("ijg,gbkc->ijbkc", sfds, fb_uh)
        out["Rh"] = -Rutmp.reshape(npf * nfe, ne, ncu, order="F")                          # [ndf, ne, ncu]
        if jacobian:
            ndf = npf * nfe
            KG = np.zeros((npf, nfe, npe, ne, ncu, nc))
            H = np.zeros((npf, nfe, npf, nfe, ne, ncu, ncu))
            for l in range(nfe):
                p = perm[:, l]
                # assembleMatrixGK (kokkosimpl.h:1680-1695): K[(i,l), perm[j,l]] += Dtmp[i,j,l]
                np.add.at(KG, (slice(None), l, p), Dtmp[:, :, l])
                # assembleMatrixH (kokkosimpl.h:1714-1730): block-diagonal per face
                H[:, l, :, l] += Ftmp[:, :, l]
            out["KG"] = KG.reshape(ndf, npe, ne, ncu, nc, order="F")
            out["H"] = H.reshape(ndf, ndf, ne, ncu, ncu, order="F")
        return out

    def assemble(self, udg=None, uh=None):
        """A1-A3: returns H [m,m,ne], Rh [m,ne], DinvF [n,m,ne], Ru [n,ne] (Schur-condensed)."""
        udg = self.udg if udg is None else udg
        uh = self.uh if uh is None else uh
        nd, npe, npf, nfe, ne, ncu, nc, ncq = (self.nd, self.npe, self.npf, self.nfe, self.ne,
                                                self.ncu, self.nc, self.ncq)
        ndf = npf * nfe
        n, m = npe * ncu, ndf * ncu
        Ru, D, B = self._volume(udg)
        fc = self._faces(udg, uh)
        Ru = Ru - fc["Ru_face"]
        D = D + fc["Dface"][:, :, :, :, :ncu]
        B = B + fc["Dface"][:, :, :, :, ncu:]
        F = fc["Fface"]                                                    # [npe, ndf, ne, ncu, ncu]
        K = fc["KG"][:, :, :, :, :ncu]
        G = fc["KG"][:, :, :, :, ncu:]
        H = fc["H"]
        Rh = fc["Rh"]
        # reorder to (npe*ncu) and (ncu*ndf) blocks (kokkosimpl.h:1797-2020)
        D2 = np.transpose(D, (0, 3, 1, 4, 2)).copy()                         # [npe, ncu, npe, ncu, ne]
        F2 = np.transpose(F, (0, 3, 4, 1, 2)).copy()                         # [npe, ncu, ncu, ndf, ne]
        K2 = np.transpose(K, (3, 0, 1, 4, 2)).copy()                         # [ncu, ndf, npe, ncu, ne]
        H2 = np.transpose(H, (3, 0, 4, 1, 2)).copy()                         # [ncu, ndf, ncu, ndf, ne]
        if ncq > 0:
            for d in range(nd):
                Bd = B[:, :, :, :, ncu * d:ncu * (d + 1)]                     # [npe, npe, ne, ncu, ncu]
                Gd = G[:, :, :, :, ncu * d:ncu * (d + 1)]                     # [ndf, npe, ne, ncu, ncu]
                C = self.MinvC[:, :, :, d]
                E = self.MinvE[:, :, :, d]
                D2 += np.einsum("ikemn,kje->imjne", Bd, C)
                F2 -= np.einsum("ikeab,kje->iabje", Bd, E)
                K2 += np.einsum("ikemn,kje->mijne", Gd, C)
                H2 -= np.einsum("ikemn,kje->minje", Gd, E)
        Dm = D2.reshape(n, n, ne, order="F")
        Fm = F2.reshape(n, m, ne, order="F")
        Km = K2.reshape(m, n, ne, order="F")
        Hm = H2.reshape(m, m, ne, order="F")
        Dinv = _inverse(Dm)
        DinvF = -np.einsum("ike,kje->ije", Dinv, Fm)
        Ruv = np.transpose(Ru, (0, 2, 1)).reshape(n, ne, order="F")          # schurVectorRu
        Ruv = np.einsum("ike,ke->ie", Dinv, Ruv)
        Hm = Hm + np.einsum("ike,kje->ije", Km, DinvF)
        Rhv = np.transpose(Rh, (2, 0, 1)).reshape(m, ne, order="F")          # schurVectorRh
        Rhv = Rhv - np.einsum("ike,ke->ie", Km, Ruv)
        self.H, self.Rh, self.DinvF, self.Ru = Hm, Rhv, DinvF, Ruv
        self.K, self.Dinv = Km, Dinv  # the condensation factors (the mixed refinement reuses them)
        return Hm, Rhv, DinvF, Ruv

    def residual(self, udg=None, uh=None):
        """A5: Ru [n, ne] and Rh [m, ne] without Jacobians (uequation.cpp:790-1088)."""
        udg = self.udg if udg is None else udg
        uh = self.uh if uh is None else uh
        ncu, npe, ne = self.ncu, self.npe, self.ne
        Ru, _, _ = self._volume(udg, jacobian=False)
        fc = self._faces(udg, uh, jacobian=False)
        Ru = Ru - fc["Ru_face"]
        Ruv = np.transpose(Ru, (0, 2, 1)).reshape(npe * ncu, ne, order="F")
        Rhv = np.transpose(fc["Rh"], (2, 0, 1)).reshape(-1, ne, order="F")
        return Ruv, Rhv

    # ------------------------------------------------------------ linear system
    def assemble_rhs(self, Rh):
        """Element trace residuals -> face vector (matvec.cpp:103-117, kokkosimpl.h:1032-1065)."""
        return self.scatter(Rh)

    def scatter(self, we):
        """PutElementFaceNodes: first element writes, second element (interior faces) adds."""
        ncu, npf, nfe, nf, nf0 = self.ncu, self.npf, self.nfe, self.nf, self.nf0
        W = we.reshape(ncu, npf, nfe, -1, order="F")
        e1, l1, e2, l2 = self.f2e
        w = np.transpose(W[:, :, l1, e1], (0, 1, 2)).copy()                  # [ncu, npf, nf]
        fi = np.arange(nf0)
        inner = fi[e2[:nf0] >= 0]
        ii = self.elemcon[np.arange(npf)[:, None] + npf * l2[inner][None, :], e2[inner][None, :]] \
            - npf * inner[None, :]
        w[:, :, inner] += W[:, ii, l2[inner][None, :], e2[inner][None, :]]
        return w

    def gather(self, v):
        return self.gather_uh(v, opt=2).reshape(self.ncu * self.npf * self.nfe, self.ne, order="F")

    def matvec(self, v, A=None):
        """w = sum_e scatter(H_e gather(v)) (matvec.cpp:240-389)."""
        A = self.H if A is None else A
        ve = self.gather(v)
        we = np.einsum("ije,je->ie", A, ve)
        return self.scatter(we)

    def build_precond(self):
        ncu, npf, nfe, nf, nf0 = self.ncu, self.npf, self.nfe, self.nf, self.nf0
        ncf = ncu * npf
        A = self.H.reshape(ncf, nfe, ncf, nfe, self.ne, order="F")
        e1, l1, e2, l2 = self.f2e
        if self.preconditioner == 0:
            # BlockJacobi (kokkosimpl.h:1067-1111) then inverse per face
            BE = A[:, l1, :, l1, e1].transpose(1, 2, 0).copy()               # [ncf, ncf, nf]
            for f in range(nf0):
                if e2[f] < 0:
                    continue
                c = self.elemcon[np.arange(npf) + npf * l2[f], e2[f]] - npf * f
                dm = (np.arange(ncu)[:, None] + ncu * c[None, :]).ravel(order="F")
                BE[:, :, f] += A[:, l2[f], :, l2[f], e2[f]][np.ix_(dm, dm)]
            self.P = _inverse(BE)
        elif self.preconditioner == 1:
            # ElementalAdditiveSchwarz (kokkosimpl.h:1113-1143) then inverse per element
            BE = A.copy()
            for f in range(nf):
                if e2[f] < 0:
                    continue
                c = self.elemcon[np.arange(npf) + npf * l2[f], e2[f]] - npf * f
                dm = (np.arange(ncu)[:, None] + ncu * c[None, :]).ravel(order="F")
                blk2 = A[:, l2[f], :, l2[f], e2[f]][np.ix_(dm, dm)]
                tm = A[:, l1[f], :, l1[f], e1[f]] + blk2
                BE[:, l1[f], :, l1[f], e1[f]] = tm
                sub = BE[:, l2[f], :, l2[f], e2[f]]
                sub[np.ix_(dm, dm)] = tm
                BE[:, l2[f], :, l2[f], e2[f]] = sub
            self.P = _inverse(BE.reshape(ncf * nfe, ncf * nfe, self.ne, order="F"))
        else:
            # super-element additive Schwarz with block ILU(0) (matvec.cpp:119-166)
            from oracle.bilu0 import BlockILU0
            if self.cartgridpart.size == 0:
                raise ValueError("block ILU(0) needs cartgridpart in mesh.bin")
            self.bilu = BlockILU0(self.cartgridpart, self.f2e, self.elemcon, ncu, npf, nfe)
            m = ncf * nfe
            self.P = self.bilu.factor(self.bilu.assemble(self.H.reshape(m, m, self.ne, order="F")))

    def apply_precond(self, x):
        if self.preconditioner == 0:
            X = x.reshape(self.ncu * self.npf, self.nf, order="F")
            y = np.einsum("ijf,jf->if", self.P, X)
            return y.reshape(x.shape, order="F")
        if self.preconditioner == 2:
            X = x.reshape(self.ncu * self.npf, self.nf, order="F")
            return self.bilu.apply(self.P, X).reshape(x.shape, order="F")
        return self.matvec(x, self.P)

    # -------------------------------------------------------------------- GMRES
    def gmres(self, b, x=None):
        """Restarted left-preconditioned GMRES with MGS/CGS (gmres.cpp:361-597)."""
        N = b.size
        bv = b.ravel(order="F")
        x = np.zeros(N) if x is None else x.ravel(order="F").copy()
        shape = b.shape
        mv = lambda v: self.matvec(v.reshape(shape, order="F")).ravel(order="F")
        pc0 = lambda v: self.apply_precond(v.reshape(shape, order="F")).ravel(order="F")
        pc = pc0
        if self.ppdegree > 1:
            # getPoly (getpoly.cpp:208-247) with the Ritz post-processing (gmres.cpp:385-398), then
            # the preconditioner followed by ApplyPoly (gmres.cpp:319-357) wherever P is applied
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
            self.poly_sr, self.poly_si = sr, si

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
        nrest, maxit = self.restart, self.gmres_maxit
        n1 = nrest + 1
        nrmb = np.sqrt(np.dot(bv, bv))
        if nrmb < self.newton_tol:
            return np.zeros(shape), GmresInfo(0, 0.0, 0.0)
        scalar = np.sqrt(np.dot(x, x))
        if scalar > 1e-12:
            r = bv - mv(x)
            nrmr = np.sqrt(np.dot(r, r))
        else:
            r = bv.copy()
            nrmr = nrmb
        tol = min(0.1, self.gmres_tol * nrmb / nrmr)
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
                    return x.reshape(shape, order="F"), GmresInfo(j + 1, relerr, tol)
                i += 1
                j += 1
            x = x + V[:, :i] @ _backsolve(Hh, s, i - 1)
            r = pc(bv - mv(x))
            nrmr = np.sqrt(np.dot(r, r))
            relerr = nrmr / nrmb
            if relerr < tol:
                return x.reshape(shape, order="F"), GmresInfo(j, relerr, tol)
        return x.reshape(shape, order="F"), GmresInfo(j, relerr, tol)

    # ------------------------------------------------------------------- Newton
    def residual_norm(self):
        Ru, Rh = self.residual()
        b = self.assemble_rhs(Rh)
        return np.linalg.norm(b) + np.linalg.norm(Ru), b

    def newton(self, maxit=None, tol=None):
        """Damped Newton on [Ru; Rh] (solution.cpp:125-243); returns (iterations, norms)."""
        maxit = self.newton_maxit if maxit is None else maxit
        tol = self.newton_tol if tol is None else tol
        if self.ncq > 0:
            self.get_q(self.udg, self.uh)
        nrmr, _ = self.residual_norm()
        norms = [nrmr]
        self.gmres_log = []
        for it in range(maxit):
            self.assemble()
            b = self.assemble_rhs(self.Rh)
            self.build_precond()
            x, info = self.gmres(b, self._rb_guess(b))
            self.gmres_log.append(info)
            alpha = 1.0
            u = self.uh + alpha * x
            self.uh = u.copy()
            ve = self.gather(x)
            du = self.Ru + np.einsum("ije,je->ie", self.DinvF, ve)          # hdgGetDUDG
            dU = du.reshape(self.npe, self.ncu, self.ne, order="F")
            self.udg[:, :self.ncu] += alpha * dU
            if self.ncq > 0:
                self.get_q(self.udg, self.uh)
            nrm0 = nrmr
            nrmr, _ = self.residual_norm()
            while (nrmr > nrm0 and alpha > 0.1) or np.isnan(nrmr):
                alpha = alpha / 2.0
                u = u - alpha * x
                self.uh = u.copy()
                self.udg[:, :self.ncu] -= alpha * dU
                if self.ncq > 0:
                    self.get_q(self.udg, self.uh)
                nrmr, _ = self.residual_norm()
            norms.append(nrmr)
            if self.RBdim > 0:
                self._rb_update(alpha * x)
            if self.verbose:
                print(f"Newton {it + 1}: alpha {alpha} norm {nrmr:.6e} gmres {info}")
            if nrmr < tol:
                return it + 1, norms
        return maxit, norms

    def newton_mixed(self, inner_tol=1e-4, rtol=1e-8, maxit=30):
        """The mixed-precision form of the solve (no counterpart in the reference): the
        condensed blocks H, D^-1 F, K, D^-1 and the preconditioner of one assembly rounded to
        FP32 (the CUDA path forms them with 3xTF32 tensor-core products, about FP32
        accuracy), then refinement steps: GMRES on the FP32 operator to inner_tol, the Newton
        update, the FP64 residual, and its condensation through the FP32 factors, until the
        residual norm |b| + |Ru| has fallen by rtol or stops falling below the Newton
        tolerance.  Vectors and accumulation stay FP64.  Returns (steps, norms)."""
        f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
        if self.ncq > 0:
            self.get_q(self.udg, self.uh)
        nrm0, _ = self.residual_norm()
        norms = [nrm0]
        if not nrm0 > 0.0:
            return 0, norms
        self.assemble()
        self.H, self.DinvF, self.K, self.Dinv = f32(self.H), f32(self.DinvF), f32(self.K), f32(self.Dinv)
        # the FP64 residual condensed through the FP32 factors
        Ru, Rh = self.residual()
        self.Ru = np.einsum("ike,ke->ie", self.Dinv, Ru)
        self.Rh = Rh - np.einsum("ike,ke->ie", self.K, self.Ru)
        self.build_precond()
        self.P = f32(self.P)
        gtol, ntol = self.gmres_tol, self.newton_tol
        self.gmres_log = []
        prev = nrm0
        steps = 0
        for steps in range(1, maxit + 1):
            b = self.assemble_rhs(self.Rh)
            self.gmres_tol, self.newton_tol = inner_tol, 0.0
            try:
                x, info = self.gmres(b)
            finally:
                self.gmres_tol, self.newton_tol = gtol, ntol
            self.gmres_log.append(info)
            self.uh = self.uh + x
            du = self.Ru + np.einsum("ije,je->ie", self.DinvF, self.gather(x))
            self.udg[:, :self.ncu] += du.reshape(self.npe, self.ncu, self.ne, order="F")
            if self.ncq > 0:
                self.get_q(self.udg, self.uh)
            Ru, Rh = self.residual()
            nrm = np.linalg.norm(self.assemble_rhs(Rh)) + np.linalg.norm(Ru)
            norms.append(nrm)
            if nrm <= rtol * nrm0:
                break
            if nrm < ntol and nrm > 0.5 * prev:  # the FP64 round-off floor
                break
            prev = nrm
            self.Ru = np.einsum("ike,ke->ie", self.Dinv, Ru)
            self.Rh = Rh - np.einsum("ike,ke->ie", self.K, self.Ru)
        return steps, norms

    def _rb_guess(self, b):
        """ComputeInitialGuessAndPreconditioner (preconditioner.cpp:133-181): U_i = A W_i for the
        newest basis vector under the current Jacobian, c = (U^T U)^-1 U^T b, x0 = W c; None
        (zero guess) without a basis or with a singular U^T U."""
        if self.RBdim <= 0 or self.rb_cur == 0:
            return None
        shape = b.shape
        cur = self.rb_cur
        i = self.rb_removed - 1 if self.rb_removed > 0 else cur - 1
        self.rb_U[:, i] = self.matvec(self.rb_W[:, i].reshape(shape, order="F")).ravel(order="F")
        U, W = self.rb_U[:, :cur], self.rb_W[:, :cur]
        H = U.T @ U
        try:
            c = np.linalg.inv(H) @ (U.T @ b.ravel(order="F"))
        except np.linalg.LinAlgError:
            return None
        return (W @ c).reshape(shape, order="F")

    def _rb_update(self, x):
        """UpdateRB (ptcsolver.cpp:484-500): the scaled Newton update replaces the oldest vector."""
        xv = x.ravel(order="F")
        if self.rb_W is None:
            self.rb_W = np.zeros((xv.size, self.RBdim))
            self.rb_U = np.zeros((xv.size, self.RBdim))
        if np.sqrt(np.dot(xv, xv)) > 0.0:
            self.rb_W[:, self.rb_removed] = xv
            self.rb_cur = min(self.rb_cur + 1, self.RBdim)
            self.rb_removed = (self.rb_removed + 1) % self.RBdim

    # --------------------------------------------------------------------- DIRK
    def dirk_solve(self, nsteps=None, on_stage=None):
        """DIRK time stepping around Newton (exasim.hpp:413-482); returns per-stage Newton counts."""
        npe, ncu, nc, ne = self.npe, self.ncu, self.nc, self.ne
        c, dvec, tt = dirk_coeff(self.nstage, self.torder)
        S = self.nstage
        dd = dvec  # column-major [S, S]: d[i + S*j]
        nsteps = len(self.dt) if nsteps is None else nsteps
        time = self.factor[0]
        counts = []
        for istep in range(nsteps):
            dt = self.dt[istep]
            udgprev = self.udg[:, :ncu].copy()                              # PreviousSolutions
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
                its, norms = self.newton()
                counts.append(its)
                utmp = utmp + c[j] * self.udg[:, :ncu]
                if on_stage is not None:
                    on_stage(istep, j, self)
            self.udg[:, :ncu] = utmp
            time = time + dt
        return counts


def _givens(H, s, cs, sn, i):
    """cpuApplyGivensRotation (cpuimpl.h:167-196)."""
    for k in range(i):
        temp = cs[k] * H[k] + sn[k] * H[k + 1]
        H[k + 1] = -sn[k] * H[k] + cs[k] * H[k + 1]
        H[k] = temp
    if H[i + 1] == 0.0:
        cs[i] = 1.0
        sn[i] = 0.0
    elif abs(H[i + 1]) > abs(H[i]):
        temp = H[i] / H[i + 1]
        sn[i] = 1.0 / np.sqrt(1.0 + temp * temp)
        cs[i] = temp * sn[i]
    else:
        temp = H[i + 1] / H[i]
        cs[i] = 1.0 / np.sqrt(1.0 + temp * temp)
        sn[i] = temp * cs[i]
    temp = cs[i] * s[i]
    s[i + 1] = -sn[i] * s[i]
    s[i] = temp
    H[i] = cs[i] * H[i] + sn[i] * H[i + 1]
    H[i + 1] = 0.0


def _backsolve(H, s, i):
    """cpuBackSolve (cpuimpl.h:198-208) on the (i+1)x(i+1) upper triangle."""
    y = s[:i + 1].copy()
    for j in range(i, -1, -1):
        y[j] = y[j] / H[j, j]
        for k in range(j - 1, -1, -1):
            y[k] = y[k] - H[k, j] * y[j]
    return y

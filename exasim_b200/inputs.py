"""Exasim input files (``datain/{app,master,mesh,sol}.bin``): readers, writers and
synthetic-case generators.

Exasim's preprocessor (``text2code``) turns ``pdeapp.txt`` + a mesh into four
binary files of float64 words.  The HDG solver in this package consumes exactly
those files, so this module restates the parts of the preprocessor that produce
them for structured synthetic meshes, and reads/writes the formats:

* ``app.bin``    writer ``writepde``         text2code/text2code/readpdeapp.cpp:820-918,
                 reader ``readappstruct``    backend/Discretization/readbinaryfiles.cpp:65-152
* ``master.bin`` builder ``initializeMaster`` text2code/text2code/makemaster.cpp:1019-1146,
                 reader ``readmasterstruct`` backend/Discretization/readbinaryfiles.cpp:208-268
* ``mesh.bin``   writer ``writemesh``        text2code/text2code/writebinaryfiles.cpp:155-295
                 (the "raw t" form whose connectivity the solver builds itself)
* ``sol.bin``    writer ``writesol``         text2code/text2code/writebinaryfiles.cpp:50-137

Reference-element node sets and quadrature rules come from the table copied out of
Exasim's ``masternodes.bin``/``gaussnodes.bin`` (``data/master_tables.npz``).
Nodal shape functions are computed the way ``mkshape`` does
(text2code/text2code/makemaster.cpp:774-846): evaluate a polynomial basis and its
derivatives at the points, divide by the basis' Vandermonde matrix at the nodes.
A different (but equivalent) polynomial basis is used, so shape tables agree with
the preprocessor's to rounding (~1e-14), not bit for bit.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

_TABLES = None


def _tables():
    global _TABLES
    if _TABLES is None:
        fn = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "master_tables.npz")
        _TABLES = dict(np.load(fn))
    return _TABLES


def _node_block(elemtype, dim, porder, name):
    t = _tables()
    v = t[f"n_{elemtype}_{dim}_{porder}_{name}"]
    s1, s2 = t[f"n_{elemtype}_{dim}_{porder}_{name}_shape"]
    return v, (int(s1), int(s2))


def _gauss_block(elemtype, dim, pgauss):
    t = _tables()
    x = t[f"g_{elemtype}_{dim}_{pgauss}_x"]
    w = t[f"g_{elemtype}_{dim}_{pgauss}_w"]
    return x, w


# ----------------------------------------------------------------------------------
# binary helpers (every word is a float64; integer arrays are stored as doubles)
# ----------------------------------------------------------------------------------

def _write_blob(fn, nsize: Sequence[float], parts: Sequence[np.ndarray]):
    os.makedirs(os.path.dirname(os.path.abspath(fn)), exist_ok=True)
    with open(fn, "wb") as f:
        np.array([len(nsize)], dtype=np.float64).tofile(f)
        np.asarray(nsize, dtype=np.float64).tofile(f)
        for p in parts:
            np.asarray(p, dtype=np.float64).ravel(order="F").tofile(f)


def read_blob(fn_or_bytes) -> List[np.ndarray]:
    """Split an Exasim ``*.bin`` file into ``[nsize, part0, part1, ...]``."""
    if isinstance(fn_or_bytes, (bytes, bytearray, memoryview)):
        a = np.frombuffer(fn_or_bytes, dtype=np.float64)
    else:
        a = np.fromfile(fn_or_bytes, dtype=np.float64)
    ls = int(a[0])
    nsize = a[1:1 + ls].astype(np.int64)
    out = [nsize]
    o = 1 + ls
    for n in nsize:
        out.append(a[o:o + n])
        o += n
    return out


# ----------------------------------------------------------------------------------
# polynomial bases on the reference element [0,1]^d or the unit simplex
# ----------------------------------------------------------------------------------

def _legendre01(x, p):
    """Shifted Legendre polynomials on [0,1] and their x-derivatives, shape [npts, p+1]."""
    t = 2.0 * x - 1.0
    L = np.zeros((x.size, p + 1))
    dL = np.zeros((x.size, p + 1))
    L[:, 0] = 1.0
    if p >= 1:
        L[:, 1] = t
        dL[:, 1] = 1.0
    for n in range(1, p):
        L[:, n + 1] = ((2 * n + 1) * t * L[:, n] - n * L[:, n - 1]) / (n + 1)
        dL[:, n + 1] = dL[:, n - 1] + (2 * n + 1) * L[:, n]
    return L, 2.0 * dL


def _basis(pts, porder, elemtype, nd):
    """Basis values and first derivatives at pts [npts, nd] -> [nd+1, npts, nbasis].

    Tensor elements span Q_p (all products with each index <= p); simplices span P_p
    (products with total degree <= p).  Either spans the same space as Exasim's
    Koornwinder / tensor-Legendre basis, so the nodal shape functions agree.
    """
    pts = np.asarray(pts, dtype=np.float64).reshape(-1, nd)
    npts = pts.shape[0]
    Ls, dLs = [], []
    for d in range(nd):
        L, dL = _legendre01(pts[:, d], porder)
        Ls.append(L)
        dLs.append(dL)
    idx = []
    if nd == 1:
        idx = [(i,) for i in range(porder + 1)]
    elif nd == 2:
        idx = [(i, j) for j in range(porder + 1) for i in range(porder + 1)
               if elemtype == 1 or i + j <= porder]
    elif nd == 3:
        idx = [(i, j, k) for k in range(porder + 1) for j in range(porder + 1) for i in range(porder + 1)
               if elemtype == 1 or i + j + k <= porder]
    nb = len(idx)
    out = np.zeros((nd + 1, npts, nb))
    for b, ijk in enumerate(idx):
        v = np.ones(npts)
        for d in range(nd):
            v = v * Ls[d][:, ijk[d]]
        out[0, :, b] = v
        for r in range(nd):
            dv = np.ones(npts)
            for d in range(nd):
                dv = dv * (dLs[d][:, ijk[d]] if d == r else Ls[d][:, ijk[d]])
            out[1 + r, :, b] = dv
    return out


def mkshape(plocal, pts, elemtype, porder, nd):
    """Nodal shape functions and derivatives at pts: returns shap [numNodes, npts, nd+1].

    Follows text2code/text2code/makemaster.cpp:774-846 (mkshape): basis at points times
    the inverse Vandermonde matrix of the basis at the nodes.
    """
    plocal = np.asarray(plocal, dtype=np.float64).reshape(-1, nd)
    nf = _basis(pts, porder, elemtype, nd)          # [nd+1, npts, nb]
    A = _basis(plocal, porder, elemtype, nd)[0]     # [numNodes, nb]
    Ainv = np.linalg.inv(A)                          # column n: coefficients of nodal function n
    shap = np.einsum("dpb,bn->dpn", nf, Ainv)       # [nd+1, npts, numNodes]
    return np.ascontiguousarray(np.transpose(shap, (2, 1, 0)))  # [numNodes, npts, nd+1]


# ----------------------------------------------------------------------------------
# master element
# ----------------------------------------------------------------------------------

@dataclass
class Master:
    nd: int
    elemtype: int
    porder: int
    pgauss: int
    nodetype: int
    xpe: np.ndarray      # [npe, nd]
    telem: np.ndarray
    xpf: np.ndarray      # [npf, nd-1]
    tface: np.ndarray
    perm: np.ndarray     # [npf, nfe] 0-based
    gpe: np.ndarray
    gwe: np.ndarray
    gpf: np.ndarray
    gwf: np.ndarray
    shapegt: np.ndarray  # [nge, npe, nd+1]
    shapegw: np.ndarray  # [npe, nge, nd+1]
    shapfgt: np.ndarray  # [ngf, npf, nd]
    shapfgw: np.ndarray  # [npf, ngf, nd]
    shapent: np.ndarray
    shapen: np.ndarray
    shapfnt: np.ndarray
    shapfn: np.ndarray
    xp1d: np.ndarray
    gp1d: np.ndarray
    gw1d: np.ndarray
    shap1dgt: np.ndarray
    shap1dgw: np.ndarray
    shap1dnt: np.ndarray
    shap1dn: np.ndarray

    @property
    def npe(self):
        return self.xpe.shape[0]

    @property
    def npf(self):
        return self.perm.shape[0]

    @property
    def nge(self):
        return self.gwe.size

    @property
    def ngf(self):
        return self.gwf.size

    @property
    def nfe(self):
        return self.perm.shape[1]


def _shapes_t_w(shap, w, nd1):
    """shap [nn, ng, nd1] -> (shapt [ng, nn, nd1], shapw [nn, ng, nd1]) as makemaster.cpp:1061-1066."""
    shapt = np.ascontiguousarray(np.transpose(shap, (1, 0, 2)))
    shapw = shap * w[None, :, None]
    return shapt, shapw


def make_master(nd: int, elemtype: int, porder: int, pgauss: int, nodetype: int = 1) -> Master:
    """Reference element data as ``initializeMaster`` builds it (makemaster.cpp:1019-1146)."""
    xpe, s = _node_block(elemtype, nd, porder, "xpe")
    xpe = xpe.reshape(s, order="F")
    telem, s2 = _node_block(elemtype, nd, porder, "telem")
    telem = (telem.reshape(s2, order="F") - 1).astype(np.int64)
    xpf, s3 = _node_block(elemtype, nd, porder, "xpf")
    tface, s4 = _node_block(elemtype, nd, porder, "tface")
    perm, s5 = _node_block(elemtype, nd, porder, "perm")
    perm = (perm.reshape(s5, order="F") - 1).astype(np.int64)
    if nd == 1:
        xpf = np.zeros((1, 1))
        tface = np.zeros((1, 1), dtype=np.int64)
    else:
        xpf = xpf.reshape(s3, order="F")
        tface = (tface.reshape(s4, order="F") - 1).astype(np.int64)
    gx, gw = _gauss_block(elemtype, nd, pgauss)
    gpe = gx.reshape(-1, nd, order="F")
    gwe = gw.ravel()
    if nd > 1:
        fx, fw = _gauss_block(elemtype, nd - 1, pgauss)
        gpf = fx.reshape(-1, nd - 1, order="F")
        gwf = fw.ravel()
    else:
        gpf = np.zeros((1, 1))
        gwf = np.ones(1)

    shapeg = mkshape(xpe, gpe, elemtype, porder, nd)         # [npe, nge, nd+1]
    shapen = mkshape(xpe, xpe, elemtype, porder, nd)         # [npe, npe, nd+1]
    shapegt, shapegw = _shapes_t_w(shapeg, gwe, nd + 1)
    shapent = np.ascontiguousarray(np.transpose(shapen, (1, 0, 2)))
    if nd > 1:
        shapfg = mkshape(xpf, gpf, elemtype, porder, nd - 1)  # [npf, ngf, nd]
        shapfn = mkshape(xpf, xpf, elemtype, porder, nd - 1)
    else:
        shapfg = np.ones((1, 1, 1))
        shapfn = np.ones((1, 1, 1))
    shapfgt, shapfgw = _shapes_t_w(shapfg, gwf, nd)
    shapfnt = np.ascontiguousarray(np.transpose(shapfn, (1, 0, 2)))

    xp1d, s6 = _node_block(elemtype, 1, porder, "xpe")
    xp1d = xp1d.reshape(-1, 1)
    g1x, g1w = _gauss_block(elemtype, 1, pgauss)
    gp1d = g1x.reshape(-1, 1)
    gw1d = g1w.ravel()
    shap1dg = mkshape(xp1d, gp1d, elemtype, porder, 1)
    shap1dn = mkshape(xp1d, xp1d, elemtype, porder, 1)
    shap1dgt, shap1dgw = _shapes_t_w(shap1dg, gw1d, 2)
    shap1dnt = np.ascontiguousarray(np.transpose(shap1dn, (1, 0, 2)))

    return Master(nd=nd, elemtype=elemtype, porder=porder, pgauss=pgauss, nodetype=nodetype,
                  xpe=xpe, telem=telem, xpf=xpf, tface=tface, perm=perm, gpe=gpe, gwe=gwe,
                  gpf=gpf, gwf=gwf, shapegt=shapegt, shapegw=shapegw, shapfgt=shapfgt,
                  shapfgw=shapfgw, shapent=shapent, shapen=shapen, shapfnt=shapfnt,
                  shapfn=shapfn, xp1d=xp1d, gp1d=gp1d, gw1d=gw1d, shap1dgt=shap1dgt,
                  shap1dgw=shap1dgw, shap1dnt=shap1dnt, shap1dn=shap1dn)


_MASTER_FIELDS = ["shapegt", "shapegw", "shapfgt", "shapfgw", "shapent", "shapen", "shapfnt",
                  "shapfn", "xpe", "gpe", "gwe", "xpf", "gpf", "gwf", "shap1dgt", "shap1dgw",
                  "shap1dnt", "shap1dn", "xp1d", "gp1d", "gw1d"]


def write_master_bin(fn: str, m: Master):
    """Write master.bin in the layout readmasterstruct expects (readbinaryfiles.cpp:208-268)."""
    ndims = np.zeros(20)
    ndims[:11] = [m.nd, m.elemtype, m.nodetype, m.porder, m.pgauss, m.npe, m.npf, m.nge, m.ngf,
                  m.xp1d.shape[0], m.gw1d.size]
    parts = [ndims] + [np.asarray(getattr(m, k)) for k in _MASTER_FIELDS]
    nsize = [p.size for p in parts]
    _write_blob(fn, nsize, parts)


def read_master_bin(fn) -> Dict[str, np.ndarray]:
    """Read master.bin into flat arrays keyed by the reference's field names."""
    b = read_blob(fn)
    out = {"ndims": b[1].astype(np.int64)}
    for k, v in zip(_MASTER_FIELDS, b[2:]):
        out[k] = v
    return out


# ----------------------------------------------------------------------------------
# app.bin
# ----------------------------------------------------------------------------------

@dataclass
class PDEApp:
    """The ``pdeapp.txt`` keys that reach ``app.bin`` (defaults as readpdeapp.cpp:336-439)."""
    nd: int = 2
    ncu: int = 1
    model: str = "ModelD"          # ModelD carries q = grad u (nc = ncu*(nd+1)); ModelC has no q
    mpiprocs: int = 1
    hybrid: int = 1
    tdep: int = 0
    wave: int = 0
    linearproblem: int = 0
    debugmode: int = 0
    matvecorder: int = 1
    GMRESortho: int = 0
    preconditioner: int = 0
    precMatrixType: int = 0
    NLMatrixType: int = 0
    runmode: int = 0
    tdfunc: int = 1
    sourcefunc: int = 1
    modelnumber: int = 0
    extFhat: int = 0
    extUhat: int = 0
    extStab: int = 0
    subproblem: int = 0
    temporalscheme: int = 0
    torder: int = 1
    nstage: int = 1
    NewtonIter: int = 20
    GMRESiter: int = 200
    GMRESrestart: int = 25
    RBdim: int = 5
    ppdegree: int = 0
    saveSolFreq: int = 1
    saveSolOpt: int = 1
    AVsmoothingIter: int = 2
    frozenAVflag: int = 1
    time: float = 0.0
    NewtonTol: float = 1e-6
    GMREStol: float = 1e-3
    matvectol: float = 1e-3
    NLparam: float = 0.0
    dt: List[float] = field(default_factory=list)
    tau: List[float] = field(default_factory=lambda: [1.0])
    physicsparam: List[float] = field(default_factory=list)
    externalparam: List[float] = field(default_factory=list)

    @property
    def nc(self):
        return self.ncu * (self.nd + 1) if self.model in ("ModelD", "modelD", "ModelW", "modelW") else self.ncu

    @property
    def ncq(self):
        return self.nc - self.ncu


def write_app_bin(fn: str, pde: PDEApp):
    """Write app.bin in the layout of ``writepde`` (readpdeapp.cpp:820-918)."""
    tdep = pde.tdep
    if len(pde.dt) > 0 and pde.dt[0] > 0:
        tdep = 1
    ndims = np.zeros(40)
    ndims[0] = pde.mpiprocs
    ndims[1] = pde.nd
    ndims[5] = pde.nc
    ndims[6] = pde.ncu
    ndims[7] = pde.ncq
    ndims[10] = pde.ncu     # nch
    ndims[11] = pde.nd      # ncx
    flag = [tdep, pde.wave, pde.linearproblem, pde.debugmode, pde.matvecorder, pde.GMRESortho,
            pde.preconditioner, pde.precMatrixType, pde.NLMatrixType, pde.runmode, pde.tdfunc,
            pde.sourcefunc, pde.modelnumber, pde.extFhat, pde.extUhat, pde.extStab, pde.subproblem]
    problem = [pde.hybrid, 0, pde.temporalscheme, pde.torder, pde.nstage, 0, 0, 0, 0, 0, 0, 0,
               0, pde.NewtonIter, pde.GMRESiter, pde.GMRESrestart, pde.RBdim, pde.saveSolFreq,
               pde.saveSolOpt, 0, 0, 0, 0, 0, 0, pde.AVsmoothingIter, pde.frozenAVflag,
               pde.ppdegree, 0, 0, 0, 0]
    factor = [pde.time, 1.0, 0.0, 0.0, 0.0]
    solversparam = [pde.NewtonTol, pde.GMREStol, pde.matvectol, pde.NLparam]
    parts = [ndims, flag, problem, pde.externalparam, pde.dt, factor, pde.physicsparam,
             solversparam, pde.tau]
    nsize = np.zeros(30)
    for i, p in enumerate(parts):
        nsize[i] = len(p)
    _write_blob(fn, nsize, parts)


def read_app_bin(fn) -> Dict[str, np.ndarray]:
    b = read_blob(fn)
    names = ["ndims", "flag", "problem", "uinf", "dt", "factor", "physicsparam", "solversparam",
             "tau", "stgdata", "stgparam", "stgib", "vindx", "dae_dt", "interfacefluxmap", "avparam"]
    return {k: v for k, v in zip(names, b[1:])}


# ----------------------------------------------------------------------------------
# meshes
# ----------------------------------------------------------------------------------

def elem_faces(dim: int, elemtype: int) -> np.ndarray:
    """Local vertex lists of each face, [nvf, nfe] 0-based (connectivity.cpp:1010-1105)."""
    if dim == 1:
        f = [[1], [2]]
    elif dim == 2 and elemtype == 0:
        f = [[2, 3], [3, 1], [1, 2]]
    elif dim == 2:
        f = [[1, 2], [2, 3], [3, 4], [4, 1]]
    elif elemtype == 0:
        f = [[2, 3, 4], [1, 4, 3], [1, 2, 4], [1, 3, 2]]
    else:
        f = [[1, 4, 3, 2], [5, 6, 7, 8], [1, 2, 6, 5], [3, 4, 8, 7], [2, 3, 7, 6], [4, 1, 5, 8]]
    return np.array(f, dtype=np.int64).T - 1


@dataclass
class Grid:
    """``grid.bin`` content: vertices p [nd, np] and elements t [nve, ne] (0-based).

    ``tp``, when set, is t with the vertices of periodic boundaries identified (the vertex on
    the far side replaced by its image on the near side), as the preprocessor's
    ``setperiodicfaces`` leaves it (makemesh.cpp:593-760): connectivity is built from tp,
    so periodic faces join their two elements, while the element nodes (xdg) come from t."""
    p: np.ndarray
    t: np.ndarray
    elemtype: int
    tp: Optional[np.ndarray] = None

    @property
    def tconn(self):
        return self.t if self.tp is None else self.tp

    @property
    def nd(self):
        return self.p.shape[0]

    @property
    def ne(self):
        return self.t.shape[1]


def read_grid_bin(fn: str) -> Grid:
    """grid.bin = [nd, np, nve, ne, p (nd x np), t (nve x ne, 1-based)] (readmesh.cpp:83-98)."""
    g = np.fromfile(fn, dtype=np.float64)
    nd, npv, nve, ne = (int(v) for v in g[:4])
    p = g[4:4 + nd * npv].reshape((nd, npv), order="F")
    t = g[4 + nd * npv:4 + nd * npv + nve * ne].reshape((nve, ne), order="F").astype(np.int64) - 1
    elemtype = 0 if nve == nd + 1 else 1
    return Grid(p=p, t=t, elemtype=elemtype)


def square_tri_grid(n: int, perturb: float = 0.0, seed: int = 0) -> Grid:
    """Unit square, (n+1)^2 vertices, each square split into two triangles.

    Interior vertices are moved by U(-perturb*h, perturb*h) in x and y (seeded).
    """
    h = 1.0 / n
    xs = np.linspace(0.0, 1.0, n + 1)
    X, Y = np.meshgrid(xs, xs, indexing="ij")     # vertex (i,j) -> i + (n+1)*j
    p = np.vstack([X.ravel(order="F"), Y.ravel(order="F")])
    if perturb > 0:
        rng = np.random.default_rng(seed)
        inner = np.zeros((n + 1, n + 1), dtype=bool)
        inner[1:-1, 1:-1] = True
        inner = inner.ravel(order="F")
        d = rng.uniform(-perturb * h, perturb * h, size=(2, p.shape[1]))
        p[:, inner] += d[:, inner]
    t = []
    for j in range(n):
        for i in range(n):
            v0 = i + (n + 1) * j
            v1 = v0 + 1
            v2 = v0 + (n + 1) + 1
            v3 = v0 + (n + 1)
            t.append([v0, v1, v2])
            t.append([v0, v2, v3])
    return Grid(p=p, t=np.array(t, dtype=np.int64).T, elemtype=0)


def square_quad_grid(n: int, L: float = 1.0) -> Grid:
    """Square of n^2 quadrilaterals, element i + n*j (vertices counter-clockwise)."""
    xs = np.linspace(0.0, L, n + 1)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    p = np.vstack([X.ravel(order="F"), Y.ravel(order="F")])
    m = n + 1
    t = []
    for j in range(n):
        for i in range(n):
            v0 = i + m * j
            t.append([v0, v0 + 1, v0 + 1 + m, v0 + m])
    return Grid(p=p, t=np.array(t, dtype=np.int64).T, elemtype=1)


def _periodic_ids(t, n, nd):
    """Structured vertex ids i + (n+1) j (+ (n+1)^2 k) with every coordinate index taken mod n."""
    m = n + 1
    idx = [t % m, (t // m) % m] + ([t // (m * m)] if nd == 3 else [])
    out = np.zeros_like(t)
    s = 1
    for k in range(nd):
        out += (idx[k] % n) * s
        s *= m
    return out


def periodic_square_quad_grid(n: int, x0: float = 0.0, L: float = 1.0) -> Grid:
    """n^2 quadrilaterals on [x0, x0+L]^2, periodic in x and y."""
    g = square_quad_grid(n, L)
    g.p = g.p + x0
    g.tp = _periodic_ids(g.t, n, 2)
    return g


def periodic_cube_hex_grid(n: int, x0: float = 0.0, L: float = 1.0) -> Grid:
    """n^3 hexahedra on [x0, x0+L]^3, periodic in x, y and z."""
    g = cube_hex_grid(n, L)
    g.p = g.p + x0
    g.tp = _periodic_ids(g.t, n, 3)
    return g


def cube_hex_grid(n: int, L: float = 1.0) -> Grid:
    """Unit cube of n^3 hexahedra (vertex order of Exasim's hex: bottom face CCW, then top)."""
    xs = np.linspace(0.0, L, n + 1)
    X, Y, Z = np.meshgrid(xs, xs, xs, indexing="ij")
    p = np.vstack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")])
    m = n + 1
    t = []
    for k in range(n):
        for j in range(n):
            for i in range(n):
                v0 = i + m * j + m * m * k
                b = [v0, v0 + 1, v0 + 1 + m, v0 + m]
                t.append(b + [v + m * m for v in b])
    return Grid(p=p, t=np.array(t, dtype=np.int64).T, elemtype=1)


def boundary_faces(grid: Grid) -> np.ndarray:
    """bool [nfe, ne]: True where the local face is not shared with another element."""
    nd, et = grid.nd, grid.elemtype
    lf = elem_faces(nd, et)
    nvf, nfe = lf.shape
    keys = np.sort(grid.tconn[lf.T.reshape(-1)].reshape(nfe, nvf, grid.ne), axis=1)   # [nfe, nvf, ne]
    keys = np.transpose(keys, (2, 0, 1)).reshape(-1, nvf)                      # (e, l) rows
    _, inv, cnt = np.unique(keys, axis=0, return_inverse=True, return_counts=True)
    shared = cnt[inv.ravel()] > 1
    return (~shared).reshape(grid.ne, nfe).T


def assign_bf(grid: Grid, exprs: Sequence[Callable[[np.ndarray], bool]], bcs: Sequence[int]) -> np.ndarray:
    """Boundary code per local face, [nfe, ne] (0 = interior).

    As ``assignboundaryfaces`` + ``apply_bcm`` (makemesh.cpp:216-257, connectivity.cpp:285-299):
    the first expression true at the face's vertices 0, 1 and nvf-1 gives the face expression
    index k, and the stored code is ``bcs[k]``.
    """
    nd, et = grid.nd, grid.elemtype
    lf = elem_faces(nd, et)
    nvf, nfe = lf.shape
    isb = boundary_faces(grid)
    bf = np.zeros((nfe, grid.ne), dtype=np.int64)
    ind2 = 0 if nvf == 1 else 1
    for e, l in zip(*np.nonzero(isb.T)):
        for k, ex in enumerate(exprs):
            ok = True
            for i in (0, ind2, nvf - 1):
                if not ex(grid.p[:, grid.t[lf[i, l], e]]):
                    ok = False
                    break
            if ok:
                bf[l, e] = bcs[k]
                break
    return bf


def write_mesh_bin(fn: str, grid: Grid, master: Master, bf: np.ndarray, bcs: Sequence[int],
                   cartgridpart: Sequence[int] = ()):
    """mesh.bin in the raw form (facecon empty, t present) that the solver connects itself."""
    ne = grid.ne
    nve = grid.t.shape[0]
    ndims = np.zeros(20)
    ndims[0] = grid.nd
    ndims[1] = ne
    ndims[3] = int(grid.tconn.max()) + 1
    ndims[4] = master.nfe
    nsize = np.zeros(50)
    nsize[0] = 20
    nsize[9] = ne
    nsize[10] = 1
    nsize[23] = master.perm.size
    nsize[24] = bf.size
    nsize[25] = len(cartgridpart)
    nsize[26] = ne * nve
    nsize[27] = len(bcs)
    nsize[28] = 4
    parts = [ndims, np.arange(ne), [ne], master.perm, bf, list(cartgridpart), grid.tconn,
             list(bcs), [ne, 0, 0, 0]]
    _write_blob(fn, nsize, parts)


def phielem(master: Master) -> np.ndarray:
    """Vertex (linear) basis at the element nodes, [npe, nve] (makemaster.cpp:848-938)."""
    x = master.xpe
    nd, et = master.nd, master.elemtype
    if nd == 1:
        return np.stack([1.0 - x[:, 0], x[:, 0]], axis=1)
    if nd == 2 and et == 0:
        return np.stack([1.0 - x[:, 0] - x[:, 1], x[:, 0], x[:, 1]], axis=1)
    if nd == 2:
        xi, eta = x[:, 0], x[:, 1]
        return np.stack([(1.0 - xi) * (1.0 - eta), xi * (1.0 - eta), xi * eta, (1.0 - xi) * eta], axis=1)
    if et == 0:
        return np.stack([1.0 - x[:, 0] - x[:, 1] - x[:, 2], x[:, 0], x[:, 1], x[:, 2]], axis=1)
    xi, eta, zeta = x[:, 0], x[:, 1], x[:, 2]
    return np.stack([(1.0 - xi) * (1.0 - eta) * (1.0 - zeta), xi * (1.0 - eta) * (1.0 - zeta),
                     xi * eta * (1.0 - zeta), (1.0 - xi) * eta * (1.0 - zeta),
                     (1.0 - xi) * (1.0 - eta) * zeta, xi * (1.0 - eta) * zeta, xi * eta * zeta,
                     (1.0 - xi) * eta * zeta], axis=1)


def dgnodes(grid: Grid, master: Master) -> np.ndarray:
    """xdg [npe, nd, ne]: vertex basis applied to vertex coordinates, summed over vertices in
    order as ``compute_dgnodes`` does (makemesh.cpp:809-827)."""
    phi = phielem(master)
    nve = grid.t.shape[0]
    x = np.zeros((master.npe, grid.nd, grid.ne))
    for node in range(nve):
        x += phi[:, node][:, None, None] * grid.p[:, grid.t[node]][None, :, :]
    return x


def write_sol_bin(fn: str, xdg: np.ndarray, udg: Optional[np.ndarray] = None,
                  uh: Optional[np.ndarray] = None, nc: int = 0, ncu: int = 0):
    """sol.bin as ``writesol`` (writebinaryfiles.cpp:50-137): xdg, then optional udg / uhat."""
    npe, nd, ne = xdg.shape
    ndims = np.zeros(12)
    ndims[0] = ne
    ndims[3] = npe
    ndims[5] = nc
    ndims[6] = ncu
    ndims[11] = nd
    nsize = np.zeros(20)
    nsize[0] = 12
    nsize[1] = xdg.size
    parts = [ndims, xdg]
    if udg is not None:
        nsize[2] = udg.size
        parts.append(udg)
    if uh is not None:
        nsize[5] = uh.size
        parts.append(uh)
    _write_blob(fn, nsize, parts)


def read_sol_bin(fn) -> Dict[str, np.ndarray]:
    b = read_blob(fn)
    names = ["ndims", "xdg", "udg", "odg", "wdg", "uh", "xcg"]
    return {k: v for k, v in zip(names, b[1:])}

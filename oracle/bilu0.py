"""Oracle (test infrastructure only): restatement of Exasim's super-element additive Schwarz
preconditioner with block ILU(0) (preconditioner = 2), used by tests/ to check the CUDA
path.  Nothing in the product imports it.

* Cartesian sub-domains      backend/Common/cpuimpl.h:1332-1496 (gridpartition2d/3d)
* face ordering in a domain  backend/Common/cpuimpl.h:1266-1330 (crs_faceordering) with its
                             helpers mke2f :440, mkf2f :459, mkfelem :529, mkf2eelem :562,
                             facereorder :1118, sortinteriorfaces :946, sortrecurrence :1024,
                             crs_array :1198, mkface :1254
* block assembly             backend/Common/kokkosimpl.h:1264-1341 (AssembleBlockILU0)
* factorization              backend/Discretization/matvec.cpp:119-166 (hdgBlockILU0),
                             index maps cpuimpl.h:1498-1625 (crs_indexingilu0)
* application                backend/Preconditioning/preconditioner.cpp:184-271 (ApplyBlockILU0)
                             and :296-325 (gather to sub-domains, sum back)

All index arrays are 0-based; f2e is [4, nf] (e1, l1, e2, l2) as in the oracle's HDG code.
"""
from __future__ import annotations

import numpy as np


# ---------------------------------------------------------------- sub-domains
def partition(cgp):
    """elem [nse, nese]: the elements of each Cartesian sub-domain (cpuimpl.h:1332-1496)."""
    cgp = [int(v) for v in cgp]
    dim = cgp[0]
    if dim == 2:
        N, M, opt = cgp[1:3], cgp[3:5], cgp[5]
    else:
        N, M, opt = cgp[1:4], cgp[4:7], cgp[7]
    if any(n % m for n, m in zip(N, M)):
        raise ValueError("grid sizes must be multiples of the block sizes")
    nb = [n // m for n, m in zip(N, M)]

    def cell_id(g):
        if opt == 0:   # lexicographic, x fastest
            r, s = 0, 1
            for k in range(dim):
                r += g[k] * s
                s *= N[k]
            return r
        r, s = 0, 1    # last coordinate fastest
        for k in reversed(range(dim)):
            r += g[k] * s
            s *= N[k]
        return r

    # block order: opt 0 walks blocks x fastest, opt 1 walks them last coordinate fastest
    if opt == 0:
        blocks = [b for b in np.ndindex(*reversed(nb))]
        blocks = [tuple(reversed(b)) for b in blocks]
    else:
        blocks = [b for b in np.ndindex(*nb)]
    cells = [tuple(reversed(c)) for c in np.ndindex(*reversed(M))]   # x fastest within a block
    elem = np.zeros((len(blocks), len(cells)), dtype=np.int64)
    for r, b in enumerate(blocks):
        for c, off in enumerate(cells):
            elem[r, c] = cell_id([b[k] * M[k] + off[k] for k in range(dim)])
    return elem


# ---------------------------------------------------------------- face graph helpers
def e2f_of(f2e, nfe, ne):
    e2f = -np.ones((nfe, ne), dtype=np.int64)
    for i in range(f2e.shape[1]):
        e1, l1, e2, l2 = f2e[:, i]
        e2f[l1, e1] = i
        if e2 >= 0:
            e2f[l2, e2] = i
    return e2f


def f2f_of(f2e, e2f, nfe):
    """Neighbour faces of each face: the other faces of e1, then those of e2."""
    nbf = 2 * (nfe - 1)
    nf = f2e.shape[1]
    f2f = -np.ones((nbf, nf), dtype=np.int64)
    for i in range(nf):
        e1, l1, e2, l2 = f2e[:, i]
        nbrs = [e2f[l, e1] for l in range(nfe) if l != l1]
        if e2 >= 0:
            nbrs += [e2f[l, e2] for l in range(nfe) if l != l2]
        f2f[:len(nbrs), i] = nbrs
    return f2f


def stable_argsort(a):
    return np.argsort(np.asarray(a), kind="stable")


def order_by_recurrence(a):
    """Indices of a: first the values that occur once (ascending), then those occurring twice
    (ascending, ties in index order), and so on (sortrecurrence, cpuimpl.h:1024-1080)."""
    a = np.asarray(a)
    rec = np.array([np.sum(a == v) for v in a], dtype=np.int64)
    out = []
    for k in range(1, int(rec.max()) + 1 if a.size else 1):
        idx = np.nonzero(rec == k)[0]
        out += list(idx[stable_argsort(a[idx])])
    return np.array(out, dtype=np.int64)


def reorder_faces(f2e):
    """Boundary faces of the domain (l2 = -1) first, by recurrence of their element; then the
    interior faces, repeatedly moving to the front those with the fewest not-yet-ordered
    neighbours (facereorder / sortinteriorfaces, cpuimpl.h:946-1165)."""
    f2e = f2e.copy()
    nf = f2e.shape[1]
    ind0 = np.nonzero(f2e[3] == -1)[0]
    ind0 = ind0[order_by_recurrence(f2e[0, ind0])]
    ind1 = np.setdiff1d(np.arange(nf), ind0)
    f2e = f2e[:, np.concatenate([ind0, ind1])]
    ne = int(max(f2e[0].max(), f2e[2].max())) + 1
    nfe = int(max(f2e[1].max(), f2e[3].max())) + 1
    nbf = 2 * (nfe - 1)
    done = len(ind0)
    while done < nf:
        f2f = f2f_of(f2e, e2f_of(f2e, nfe, ne), nfe)
        rest = np.arange(done, nf)
        cnt = np.array([np.sum(f2f[:, f] >= done) for f in rest], dtype=np.int64)
        a = stable_argsort(cnt)
        f2e[:, rest] = f2e[:, rest[a]]
        done += int(np.sum(cnt[a] < nbf))
    return f2e


def face_ordering(elem, f2e, nfe):
    """row_ptr, col_ind (face graph of one sub-domain in CRS, diagonal first) and
    face [nse, nfse] (global face of each local face of each sub-domain)."""
    nse, nese = elem.shape
    ne_tot = int(f2e[0].max()) + 1
    e2f = e2f_of(f2e, nfe, max(ne_tot, int(f2e[2].max()) + 1))
    el0 = elem[0]
    felem = []
    for e in el0:
        for l in range(nfe):
            f = e2f[l, e]
            if f not in felem:
                felem.append(f)
    felem = np.array(felem, dtype=np.int64)
    loc = {int(e): j for j, e in enumerate(el0)}
    f2el = f2e[:, felem].copy()
    for i in range(f2el.shape[1]):
        e1, l1, e2, l2 = f2el[:, i]
        in1, in2 = int(e1) in loc, int(e2) in loc
        if in1:
            f2el[0, i] = loc[int(e1)]
        if in2:
            f2el[2, i] = loc[int(e2)]
        if not in1 and in2:
            f2el[:, i] = [loc[int(e2)], l2, -1, -1]
        if not in2:
            f2el[2:, i] = -1
    f2el = reorder_faces(f2el)
    nfse = f2el.shape[1]
    f2f = f2f_of(f2el, e2f_of(f2el, nfe, nese), nfe)
    row_ptr, col_ind = [0], []
    for i in range(nfse):
        nb = sorted(int(v) for v in f2f[:, i] if v >= 0)
        col_ind += [i] + nb
        row_ptr.append(len(col_ind))
    face = np.zeros((nse, nfse), dtype=np.int64)
    for r in range(nse):
        for i in range(nfse):
            e, l = f2el[0, i], f2el[1, i]
            face[r, i] = e2f[l, elem[r, e]]
    return np.array(row_ptr), np.array(col_ind), face


# ---------------------------------------------------------------- ILU(0)
class BlockILU0:
    """Block ILU(0) of the sub-domain face matrices (one per sub-domain, same pattern)."""

    def __init__(self, cgp, f2e, elemcon, ncu, npf, nfe):
        self.elem = partition(cgp)
        self.row_ptr, self.col_ind, self.face = face_ordering(self.elem, f2e, nfe)
        self.f2e = f2e
        self.elemcon = np.asarray(elemcon).reshape(npf, nfe, -1, order="F")   # [npf, nfe, ne]
        self.ncu, self.npf, self.nfe = ncu, npf, nfe
        self.ncf = ncu * npf
        self.nse, self.nfse = self.face.shape
        self.pos = {}
        for i in range(self.nfse):
            for t in range(self.row_ptr[i], self.row_ptr[i + 1]):
                self.pos[(i, int(self.col_ind[t]))] = t

    def _perm(self, f, e, l):
        """Trace-row index within face f of the rows of element e's local face l."""
        npf, ncu = self.npf, self.ncu
        a = self.elemcon[:, l, e] - npf * f          # [npf]
        return np.array([c + ncu * a[b] for b in range(npf) for c in range(ncu)])

    def assemble(self, H):
        """Blocks [nse, nnz, ncf, ncf] from the element matrices H [m, m, ne]
        (AssembleBlockILU0, kokkosimpl.h:1264-1341)."""
        ncf, npf, ncu = self.ncf, self.npf, self.ncu
        nnz = len(self.col_ind)
        BE = np.zeros((self.nse, nnz, ncf, ncf))
        for r in range(self.nse):
            for i in range(self.nfse):
                fi = int(self.face[r, i])
                e1, l1, e2, l2 = (int(v) for v in self.f2e[:, fi])
                # local order (a, c) -> element row index c + ncu * perm
                m1 = self._perm(fi, e1, l1)
                blk = H[:, :, e1][np.ix_(l1 * ncf + m1, l1 * ncf + m1)]
                if e2 >= 0:
                    m2 = self._perm(fi, e2, l2)
                    blk = blk + H[:, :, e2][np.ix_(l2 * ncf + m2, l2 * ncf + m2)]
                t0 = self.row_ptr[i]
                BE[r, t0] = blk
                for t in range(t0 + 1, self.row_ptr[i + 1]):
                    j = int(self.col_ind[t])
                    fj = int(self.face[r, j])
                    je1, jl1, je2, jl2 = (int(v) for v in self.f2e[:, fj])
                    if je1 == e1:
                        e, k1, k2 = e1, l1, jl1
                    elif je1 == e2:
                        e, k1, k2 = e2, l2, jl1
                    elif je2 == e1:
                        e, k1, k2 = e1, l1, jl2
                    else:
                        e, k1, k2 = e2, l2, jl2
                    mi = self._perm(fi, e, k1)
                    nj = self._perm(fj, e, k2)
                    BE[r, t] = H[:, :, e][np.ix_(k1 * ncf + mi, k2 * ncf + nj)]
        return BE

    def factor(self, BE):
        """In place: diagonal blocks replaced by their inverses, L blocks multiplied by the
        inverse diagonal, U blocks updated (hdgBlockILU0, matvec.cpp:119-166)."""
        for i in range(self.nfse):
            d = self.pos[(i, i)]
            BE[:, d] = np.linalg.inv(BE[:, d])
            for t in range(self.row_ptr[i], self.row_ptr[i + 1]):
                j = int(self.col_ind[t])
                if j <= i or (j, i) not in self.pos:
                    continue
                ji = self.pos[(j, i)]
                BE[:, ji] = BE[:, ji] @ BE[:, d]
                for t2 in range(self.row_ptr[i], self.row_ptr[i + 1]):
                    ell = int(self.col_ind[t2])
                    if ell <= i or (j, ell) not in self.pos:
                        continue
                    BE[:, self.pos[(j, ell)]] -= BE[:, ji] @ BE[:, t2]
        return BE

    def apply(self, BE, x):
        """y = P x for a trace vector x [ncf, nf]: gather to the sub-domains, forward and
        backward sweeps, sum back (preconditioner.cpp:184-325)."""
        y = x[:, self.face]                          # [ncf, nse, nfse]
        y = np.transpose(y, (1, 2, 0)).copy()        # [nse, nfse, ncf]
        for i in range(self.nfse):
            for t in range(self.row_ptr[i], self.row_ptr[i + 1]):
                j = int(self.col_ind[t])
                if j < i:
                    y[:, i] -= np.einsum("rab,rb->ra", BE[:, t], y[:, j])
        z = np.zeros_like(y)
        for i in reversed(range(self.nfse)):
            for t in range(self.row_ptr[i], self.row_ptr[i + 1]):
                ell = int(self.col_ind[t])
                if ell > i:
                    y[:, i] -= np.einsum("rab,rb->ra", BE[:, t], z[:, ell])
            z[:, i] = np.einsum("rab,rb->ra", BE[:, self.pos[(i, i)]], y[:, i])
        out = np.zeros_like(x)
        for r in range(self.nse):
            for i in range(self.nfse):
                out[:, self.face[r, i]] += z[r, i]
        return out

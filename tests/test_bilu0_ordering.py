"""CPU checks of the block-ILU(0) set-up: the oracle's restatement of the Cartesian
sub-domain partition and of the sub-domain face ordering (CRS pattern and face map) against
the reference's own routines (backend/Common/cpuimpl.h:1266-1496), compiled from the
reference tree by oracle/build_ref.sh when the tree is present; and the product's host
ordering (C ABI exa_bilu0_ordering) against the oracle."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from exasim_b200 import inputs as I
from oracle.bilu0 import face_ordering, partition

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFSO = os.path.join(ROOT, "oracle", "_ref", "libref_bilu0.so")


def cube_f2e(nd, n, tmp):
    """Face connectivity (reference order) of an n^nd Cartesian grid, from the oracle."""
    from exasim_b200 import cases
    from oracle.hdg import HDGOracle
    from oracle.models import MODELS
    d = os.path.join(tmp, f"g{nd}_{n}")
    if nd == 2:
        cases.poisson2d_quad(d, n=n, porder=1)
        return HDGOracle(d, MODELS["poisson2d"]()).f2e
    cases.convdiff3d_hex(d, n=n, porder=1, nsteps=1)
    return HDGOracle(d, MODELS["convdiff3d"]()).f2e


def ref_lib():
    if not os.path.exists(REFSO):
        ref = os.environ.get("EXASIM_REF", "")
        if not os.path.isdir(os.path.join(ref, "backend")):
            pytest.skip("reference tree absent (EXASIM_REF): the reference ordering cannot be built")
        subprocess.run(["sh", os.path.join(ROOT, "oracle", "build_ref.sh"), ref], check=True)
    L = ctypes.CDLL(REFSO)
    P = ctypes.c_void_p
    L.ref_partition.argtypes = [ctypes.c_int, P, ctypes.POINTER(P), ctypes.POINTER(ctypes.c_int),
                                ctypes.POINTER(ctypes.c_int)]
    L.ref_faceordering.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, ctypes.c_int, P,
                                   ctypes.c_int, P, ctypes.c_int]
    L.ref_free.argtypes = [P]
    return L


def ref_partition(L, cgp):
    c = np.ascontiguousarray(cgp, dtype=np.int32)
    p, nse, nese = ctypes.c_void_p(), ctypes.c_int(), ctypes.c_int()
    L.ref_partition(int(cgp[0]), c.ctypes.data, ctypes.byref(p), ctypes.byref(nse), ctypes.byref(nese))
    n = nse.value * nese.value
    out = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_int)), shape=(n,)).copy()
    L.ref_free(p)
    return out.reshape(nse.value, nese.value, order="F")


CASES = [(2, 8, (2, 8, 8, 4, 4, 0)), (2, 8, (2, 8, 8, 2, 4, 1)), (2, 6, (2, 6, 6, 3, 2, 0)),
         (3, 4, (3, 4, 4, 4, 2, 2, 2, 0)), (3, 4, (3, 4, 4, 4, 2, 4, 2, 1))]


@pytest.mark.parametrize("nd,n,cgp", CASES)
def test_partition_and_ordering_match_reference(tmp_path, nd, n, cgp):
    L = ref_lib()
    elem = partition(cgp)
    assert np.array_equal(elem, ref_partition(L, cgp))
    f2e = cube_f2e(nd, n, str(tmp_path))
    nfe = 2 * nd
    row_ptr, col_ind, face = face_ordering(elem, f2e, nfe)
    nse, nese = elem.shape
    cap = 64 * nese * nfe
    rp = np.zeros(cap, dtype=np.int32)
    ci = np.zeros(cap * 8, dtype=np.int32)
    fc = np.zeros(cap * nse, dtype=np.int32)
    el = np.ascontiguousarray(elem.ravel(order="F"), dtype=np.int32)
    fe = np.ascontiguousarray(f2e.ravel(order="F"), dtype=np.int32)
    nfse = L.ref_faceordering(el.ctypes.data, fe.ctypes.data, nse, nese, nfe, f2e.shape[1], rp.ctypes.data, cap,
                              ci.ctypes.data, ci.size, fc.ctypes.data, fc.size)
    assert nfse == len(row_ptr) - 1
    assert np.array_equal(row_ptr, rp[:nfse + 1])
    assert np.array_equal(col_ind, ci[:rp[nfse]])
    assert np.array_equal(face, fc[:nse * nfse].reshape(nse, nfse, order="F"))


@pytest.mark.parametrize("nd,n,cgp", CASES)
def test_product_ordering_matches_oracle(tmp_path, nd, n, cgp):
    from exasim_b200 import build as B, load_library
    B.build(["poisson2d"])
    L = load_library("poisson2d")
    f2e = cube_f2e(nd, n, str(tmp_path))
    nfe = 2 * nd
    ne = n ** nd
    row_ptr, col_ind, face = face_ordering(partition(cgp), f2e, nfe)
    c = np.ascontiguousarray(cgp, dtype=np.int32)
    fe = np.ascontiguousarray(f2e.ravel(order="F"), dtype=np.int32)
    cap = 64 * ne * nfe
    rp, ci, fc = np.zeros(cap, np.int32), np.zeros(8 * cap, np.int32), np.zeros(cap, np.int32)
    nse = ctypes.c_int()
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    nfse = L.exa_bilu0_ordering(P(c), len(cgp), P(fe), f2e.shape[1], nfe, ne, P(rp), rp.size, P(ci), ci.size, P(fc),
                                fc.size, ctypes.byref(nse))
    assert nfse == len(row_ptr) - 1, L.exa_last_error()
    assert np.array_equal(rp[:nfse + 1], row_ptr) and np.array_equal(ci[:row_ptr[-1]], col_ind)
    assert np.array_equal(fc[:nse.value * nfse].reshape(nse.value, nfse, order="F"), face)


def ilu_pattern_error(fac, orig, row_ptr, col_ind):
    """Block ILU(0) property, the dense check of the reference's test_block_ilu0.m in
    substance: with L unit lower (stored L blocks) and U upper (inverted stored diagonal,
    stored U blocks), (L U)_jk equals the assembled A_jk on every stored block (j, k)."""
    nfse = len(row_ptr) - 1
    ncf = fac.shape[-1]
    n = nfse * ncf
    L, U, A = np.eye(n), np.zeros((n, n)), np.zeros((n, n))
    blk = lambda i: slice(i * ncf, (i + 1) * ncf)
    for i in range(nfse):
        for t in range(row_ptr[i], row_ptr[i + 1]):
            j = int(col_ind[t])
            A[blk(i), blk(j)] = orig[t]
            if j == i:
                U[blk(i), blk(i)] = np.linalg.inv(fac[t])
            elif j > i:
                U[blk(i), blk(j)] = fac[t]
            else:
                L[blk(i), blk(j)] = fac[t]
    LU = L @ U
    err = 0.0
    for i in range(nfse):
        for t in range(row_ptr[i], row_ptr[i + 1]):
            j = int(col_ind[t])
            err = max(err, np.abs(LU[blk(i), blk(j)] - A[blk(i), blk(j)]).max())
    return err / np.abs(A).max()


@pytest.mark.parametrize("nd", [2, 3])
def test_oracle_block_ilu0_reproduces_the_matrix_on_its_pattern(tmp_path, nd):
    from exasim_b200 import cases
    from oracle.bilu0 import BlockILU0
    from oracle.hdg import HDGOracle
    from oracle.models import MODELS
    if nd == 2:
        d = cases.poisson2d_quad(str(tmp_path / "q"), n=4, porder=1, preconditioner=2, cartgridpart=(2, 4, 4, 2, 2, 0))
        o = HDGOracle(d, MODELS["poisson2d"]())
    else:
        d = cases.convdiff3d_hex(str(tmp_path / "h"), n=2, porder=1, nsteps=1, preconditioner=2,
                                 cartgridpart=(3, 2, 2, 2, 2, 2, 2, 0))
        o = HDGOracle(d, MODELS["convdiff3d"]())
    rng = np.random.default_rng(nd)
    m = o.ncu * o.npf * o.nfe
    H = rng.standard_normal((m, m, o.ne)) + 4.0 * m * np.eye(m)[:, :, None]
    b = BlockILU0(o.cartgridpart, o.f2e, o.elemcon, o.ncu, o.npf, o.nfe)
    orig = b.assemble(H)
    fac = b.factor(orig.copy())
    for r in range(b.nse):
        assert ilu_pattern_error(fac[r], orig[r], b.row_ptr, b.col_ind) < 1e-12

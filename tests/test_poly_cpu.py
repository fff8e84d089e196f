"""The polynomial preconditioner's host part (exa_poly_ritz, host code of the C ABI, no GPU)
against its numpy restatement (oracle/poly.py): harmonic Ritz values of the Hessenberg
matrix of m Arnoldi steps, Leja-ordered (getpoly.cpp:111-173, 226-247; gmres.cpp:385-398).
The C library finds the eigenvalues by the Francis QR iteration and numpy by LAPACK, so the
values agree to 1e-9 of their scale and come in the same order, up to which member of a
conjugate pair comes first."""
import ctypes

import numpy as np
import pytest

from exasim_b200 import build as B, load_library
from oracle.poly import poly_ritz


def ritz(L, H):
    m = H.shape[1]
    Hf = np.asfortranarray(H, dtype=np.float64)
    sr, si = np.zeros(m), np.zeros(m)
    st = L.exa_poly_ritz(Hf.ctypes.data_as(ctypes.c_void_p), m, sr.ctypes.data_as(ctypes.c_void_p),
                         si.ctypes.data_as(ctypes.c_void_p))
    assert st == 0, L.exa_last_error().decode()
    return sr, si


def hessenberg(rng, m, shift):
    H = np.triu(rng.standard_normal((m + 1, m)), -1)
    H[:m, :m] += shift * np.eye(m)
    return H


@pytest.mark.parametrize("m,shift,seed", [(2, 3.0, 0), (3, 3.0, 1), (5, 2.0, 2), (8, 4.0, 3), (10, 0.5, 4),
                                          (16, 6.0, 5)])
def test_ritz_values_match_restatement(m, shift, seed):
    B.build(["poisson2d"])
    L = load_library("poisson2d")
    H = hessenberg(np.random.default_rng(seed), m, shift)
    sr, si = ritz(L, H)
    rr, ri = poly_ritz(H)
    scale = np.abs(rr + 1j * ri).max()
    # within a conjugate pair the two members tie in the Leja order; which comes first does not
    # change the polynomial (ApplyPoly uses the pair's real part and modulus only)
    assert np.abs(sr - rr).max() <= 1e-9 * scale and np.abs(np.abs(si) - np.abs(ri)).max() <= 1e-9 * scale


def test_all_real_ritz_values_become_spread_points():
    B.build(["poisson2d"])
    L = load_library("poisson2d")
    # upper triangular Hm: real eigenvalues, so the points are spread over [lmin, lmax]
    m = 4
    H = np.zeros((m + 1, m))
    H[:m, :m] = np.triu(np.arange(1.0, 1.0 + m * m).reshape(m, m)) * 0.1 + np.diag([1.0, 2.0, 3.0, 4.0])
    H[m, m - 1] = 0.0
    sr, si = ritz(L, H)
    rr, ri = poly_ritz(H)
    assert np.all(si == 0.0) and np.allclose(sr, rr, rtol=1e-12, atol=0.0)

"""Numpy restatement of the polynomial preconditioner's host part (test infrastructure).

getPoly's eigH and LejaSort (backend/Solver/getpoly.cpp:111-173, 226-247) and the Ritz-value
post-processing in GMRES (backend/Solver/gmres.cpp:385-398): from the Hessenberg matrix of m
Arnoldi steps, the harmonic Ritz values Hm + beta^2 (Hm^-T e_m) e_m^T, their Leja order, and
the spread of real points that replaces them when all are real.
"""
import numpy as np

_TINY = np.finfo(float).tiny


def leja_sort(lr, li):
    """LejaSort (getpoly.cpp:130-173)."""
    n = len(lr)
    sr, si = np.zeros(n), np.zeros(n)
    sr[0], si[0] = lr[0], li[0]
    for i in range(1, n):
        if np.hypot(lr[i], li[i]) > np.hypot(sr[0], si[0]):
            sr[0], si[0] = lr[i], li[i]
    j = 1
    if abs(si[0]) > 1e-10:
        if n > 1:
            sr[1], si[1] = sr[0], -si[0]
        j = 2
    else:
        si[0] = 0.0
    while j < n:
        prod = np.array([1.0 + sum(np.log(max(np.hypot(lr[i] - sr[k], li[i] - si[k]), _TINY)) for k in range(j))
                         for i in range(n)])
        best = 0
        for i in range(1, n):
            if prod[i] > prod[best]:
                best = i
        sr[j], si[j] = lr[best], li[best]
        if abs(si[j]) > 1e-10:
            if j + 1 < n:
                sr[j + 1], si[j + 1] = sr[j], -si[j]
            j += 1
        else:
            si[j] = 0.0
        j += 1
    return sr, si


def poly_ritz(H):
    """H [(m+1), m] -> (sr, si): the Leja-ordered roots of the preconditioning polynomial."""
    m = H.shape[1]
    Hm = H[:m, :m]
    em = np.zeros(m)
    em[-1] = 1.0
    work = np.linalg.solve(Hm.T, em)
    A = Hm.copy()
    A[:, -1] += H[m, m - 1] ** 2 * work
    ev = np.linalg.eigvals(A)
    sr, si = leja_sort(ev.real.copy(), ev.imag.copy())
    if np.abs(si).max() == 0.0:
        lmin, lmax = sr.min(), sr.max()
        i = np.arange(1, m + 1)
        lam = lmin + (lmax - lmin) * (0.5 - 0.5 * np.cos((2 * i - 1) * np.pi / (2 * m)) / np.cos(np.pi / (2 * m)))
        sr, si = leja_sort(lam, np.zeros(m))
    return sr, si

"""The TF32 tensor-core batched GEMM (tcgen05) through the C ABI.

Reference: the same product in FP64 numpy with the operands first rounded the way the
kernel rounds them (FP64 -> FP32 to nearest, then to TF32 to nearest with ties away from
zero), so the only difference left is FP32 accumulation: max |gpu - ref| <= 2e-5 * max |ref|.
"""
import ctypes

import numpy as np
import pytest

from exasim_b200 import build as B, load_library

pytestmark = pytest.mark.gpu


def tf32(x):
    f = np.asarray(x, dtype=np.float64).astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x1000) & 0xFFFFE000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


@pytest.mark.parametrize("M,N,K,a64", [(125, 125, 375, True), (150, 150, 125, False), (125, 150, 375, True),
                                       (150, 125, 375, True), (25, 25, 25, False), (64, 256, 40, False)])
def test_tf32_gemm_matches_rounded_reference(M, N, K, a64):
    import torch
    B.build(["poisson2d"])
    L = load_library("poisson2d")
    rng = np.random.default_rng(M * 1000 + N + K)
    nb = 37
    lda, ldb, ldc = M + 3, K + 1, M + 2
    A = rng.standard_normal((nb, K, lda))
    Bm = rng.standard_normal((nb, N, ldb)).astype(np.float32)
    C0 = rng.standard_normal((nb, N, ldc)).astype(np.float32)
    alpha, beta = -1.5, 0.75
    dev = "cuda"
    At = torch.tensor(A, dtype=torch.float64 if a64 else torch.float32, device=dev)
    Bt = torch.tensor(Bm, device=dev)
    Ct = torch.tensor(C0, device=dev)
    flag = torch.zeros(1, dtype=torch.int32, device=dev)
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = L.exa_gemm_tf32_batched(M, N, K, alpha, P(At), int(a64), lda, K * lda, P(Bt), 0, ldb, N * ldb, beta, P(Ct),
                                 0, ldc, N * ldc, nb, P(flag), None)
    assert rc == 0, L.exa_last_error().decode()
    torch.cuda.synchronize()
    assert int(flag.item()) == 0
    got = Ct.cpu().numpy().astype(np.float64)
    Ar = tf32(A if a64 else A.astype(np.float32))
    Br = tf32(Bm)
    for b in range(nb):
        ref = alpha * Ar[b, :, :M].T @ Br[b, :, :K].T + beta * C0[b, :, :M].T.astype(np.float64)
        g = got[b, :, :M].T
        assert np.abs(g - ref).max() <= 2e-5 * np.abs(ref).max(), (b, np.abs(g - ref).max(), np.abs(ref).max())
        # padding rows of C untouched
        assert np.array_equal(got[b, :, M:], C0[b, :, M:].astype(np.float64))


@pytest.mark.parametrize("M,N,K,a64,nb", [(125, 125, 375, True, 29), (150, 150, 125, False, 29),
                                          (125, 150, 375, True, 29), (150, 125, 375, True, 29), (10, 12, 20, True, 29),
                                          (64, 256, 40, False, 29), (150, 480, 320, True, 29), (96, 300, 40, False, 29),
                                          (125, 125, 100, True, 700), (150, 150, 60, False, 400),
                                          (64, 256, 40, False, 640)])
def test_3xtf32_gemm_matches_fp64(M, N, K, a64, nb):
    """hi*hi + hi*lo + lo*hi drops the lo*lo term (2^-22 relative) and the tensor cores add the
    products in FP32 without round-to-nearest on every step: within 1e-5 of max |C| at K <= 375
    (1xTF32 is about 1e-3 there).  Batches of 400 and more as well as 29."""
    import torch
    B.build(["poisson2d"])
    L = load_library("poisson2d")
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    lda, ldb, ldc = M + 1, K + 3, M + 2
    A = rng.standard_normal((nb, K, lda))
    Bm = rng.standard_normal((nb, N, ldb))
    C0 = rng.standard_normal((nb, N, ldc)).astype(np.float32)
    alpha, beta = 0.5, -1.0
    dev = "cuda"
    At = torch.tensor(A, dtype=torch.float64 if a64 else torch.float32, device=dev)
    Bt = torch.tensor(Bm, dtype=torch.float64, device=dev)
    Ct = torch.tensor(C0, device=dev)
    flag = torch.zeros(1, dtype=torch.int32, device=dev)
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = L.exa_gemm_3xtf32_batched(M, N, K, alpha, P(At), int(a64), lda, K * lda, P(Bt), 1, ldb, N * ldb, beta, P(Ct),
                                   ldc, N * ldc, nb, P(flag), None)
    assert rc == 0, L.exa_last_error().decode()
    assert int(flag.item()) == 0
    got = Ct.cpu().numpy().astype(np.float64)
    Aref = A if a64 else A.astype(np.float32).astype(np.float64)
    for b in range(nb):
        ref = alpha * Aref[b, :, :M].T @ Bm[b, :, :K].T + beta * C0[b, :, :M].T.astype(np.float64)
        g = got[b, :, :M].T
        assert np.abs(g - ref).max() <= 1e-5 * np.abs(ref).max(), (b, np.abs(g - ref).max(), np.abs(ref).max())
        assert np.array_equal(got[b, :, M:], C0[b, :, M:].astype(np.float64))

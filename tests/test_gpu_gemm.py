"""The FP64 batched GEMM on the DMMA tensor cores (exa_dgemm_batched, the reference's
PGEMNMStridedBached, backend/Common/pblas.h:695) against numpy, on the element-block
shapes of the assembly, before and after the tile autotuner (exa_dgemm_tune) has picked
the shape's fastest tile.  Every tile sums each entry over k in the same order, so the two
results must be equal bit for bit; against numpy the tolerance is 1e-13 of max |C|."""
import ctypes

import numpy as np
import pytest

from exasim_b200 import build as B, load_library

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    B.build(["poisson2d"])
    return load_library("poisson2d")


def run(lib, A, Bm, C0, alpha, beta):
    import torch
    batch, M, K = A.shape
    N = Bm.shape[2]
    dev = lambda X: torch.tensor(np.ascontiguousarray(np.transpose(X, (0, 2, 1))).ravel(), dtype=torch.float64,
                                 device="cuda")
    a, b, c = dev(A), dev(Bm), dev(C0)
    st = lib.exa_dgemm_batched(M, N, K, alpha, ctypes.c_void_p(a.data_ptr()), M, M * K, ctypes.c_void_p(b.data_ptr()),
                               K, K * N, beta, ctypes.c_void_p(c.data_ptr()), M, M * N, batch, None)
    assert st == 0, lib.exa_last_error().decode()
    torch.cuda.synchronize()
    return np.transpose(c.cpu().numpy().reshape(batch, N, M), (0, 2, 1))


@pytest.mark.parametrize("M,N,K", [(125, 125, 375), (125, 150, 375), (150, 125, 375), (150, 150, 375),
                                   (125, 150, 125), (150, 150, 125), (64, 96, 48), (64, 4000, 64),
                                   (64, 3000, 256)])
def test_dgemm_tuned_equals_untuned_and_numpy(lib, M, N, K):
    rng = np.random.default_rng(M * N + K)
    batch = 40
    A = rng.standard_normal((batch, M, K))
    Bm = rng.standard_normal((batch, K, N))
    C0 = rng.standard_normal((batch, M, N))
    before = run(lib, A, Bm, C0, -1.0, 1.0)
    tile = ctypes.c_int(-1)
    assert lib.exa_dgemm_tune(M, N, K, 64, None, ctypes.byref(tile)) == 0, lib.exa_last_error().decode()
    assert 0 <= tile.value < 6
    after = run(lib, A, Bm, C0, -1.0, 1.0)
    assert np.array_equal(before, after)
    ref = C0 - A @ Bm
    assert np.abs(after - ref).max() / np.abs(ref).max() < 1e-13

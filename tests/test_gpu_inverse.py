"""The batched explicit inverse (exa_dinverse_batched, the reference's Inverse,
backend/Common/pblas.h:163) against LAPACK through numpy, for every kernel shape: one warp
per matrix (n <= 32), the register-tiled kernel (n <= 160) and the 2 x 2 blocked form
(n <= 320).  Matrices are diagonally weighted random blocks with cond ~ 1e2; tolerance
1e-12 of max |inverse| (Gauss-Jordan with partial pivoting against getrf + getri).  A
singular block sets the flag."""
import ctypes

import numpy as np
import pytest

from exasim_b200 import build as B, load_library

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    B.build(["poisson2d"])
    return load_library("poisson2d")


@pytest.mark.parametrize("n", [1, 5, 25, 32, 33, 64, 96, 125, 128, 150, 160, 200, 320])
def test_inverse_matches_lapack(lib, n):
    import torch
    rng = np.random.default_rng(n)
    batch = 37
    A = rng.standard_normal((batch, n, n)) + np.eye(n) * (2.0 * np.sqrt(n))
    # column-major blocks spaced n^2 apart
    dev = torch.tensor(np.ascontiguousarray(np.transpose(A, (0, 2, 1))).ravel(), dtype=torch.float64, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib.exa_dinverse_batched(ctypes.c_void_p(dev.data_ptr()), n, n * n, batch, ctypes.c_void_p(flag.data_ptr()),
                                  None)
    assert st == 0, lib.exa_last_error().decode()
    torch.cuda.synchronize()
    got = np.transpose(dev.cpu().numpy().reshape(batch, n, n), (0, 2, 1))
    ref = np.linalg.inv(A)
    assert int(flag.item()) == 0
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-12, err


@pytest.mark.parametrize("n", [25, 125, 160, 170, 201, 250, 320])
def test_fp32_inverse_matches_lapack(lib, n):
    """exa_sinverse_batched, the mixed form's FP32 inverse: register kernels up to 160, the
    recursive blocked form with 3xTF32 tensor-core products above (one level at 170, two at
    201, 250 and 320; 170, 201 and 250 have halves that are not multiples of 16, so the
    packed operands carry padding).  FP32 rounding of the input and of the elimination:
    within 2e-5 of max |inverse| at cond ~ 1e2."""
    import torch
    rng = np.random.default_rng(1000 + n)
    batch = 37
    A = (rng.standard_normal((batch, n, n)) + np.eye(n) * (2.0 * np.sqrt(n))).astype(np.float32)
    dev = torch.tensor(np.ascontiguousarray(np.transpose(A, (0, 2, 1))).ravel(), dtype=torch.float32, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(2):  # the second call reuses the stream-ordered workspace memory
        d = dev.clone()
        st = lib.exa_sinverse_batched(ctypes.c_void_p(d.data_ptr()), n, n * n, batch,
                                      ctypes.c_void_p(flag.data_ptr()), None)
        assert st == 0, lib.exa_last_error().decode()
        torch.cuda.synchronize()
        assert int(flag.item()) == 0
        got = np.transpose(d.cpu().numpy().reshape(batch, n, n), (0, 2, 1)).astype(np.float64)
        ref = np.linalg.inv(A.astype(np.float64))
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < 2e-5, err


@pytest.mark.parametrize("n", [125, 250])
def test_fp32_singular_block_sets_flag(lib, n):
    """A zero pivot column in the block (the leading diagonal block of the blocked form at
    250) sets the flag in the FP32 inverse as in the FP64 one."""
    import torch
    A = np.eye(n, dtype=np.float32)
    A[3, 3] = 0.0
    dev = torch.tensor(A.T.ravel(), dtype=torch.float32, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.exa_sinverse_batched(ctypes.c_void_p(dev.data_ptr()), n, n * n, 1, ctypes.c_void_p(flag.data_ptr()),
                                    None) == 0
    torch.cuda.synchronize()
    assert int(flag.item()) == 1


@pytest.mark.parametrize("n", [8, 125])
def test_singular_block_sets_flag(lib, n):
    import torch
    A = np.eye(n)
    A[3, 3] = 0.0
    dev = torch.tensor(A.T.ravel(), dtype=torch.float64, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.exa_dinverse_batched(ctypes.c_void_p(dev.data_ptr()), n, n * n, 1, ctypes.c_void_p(flag.data_ptr()),
                                    None) == 0
    torch.cuda.synchronize()
    assert int(flag.item()) == 1


@pytest.mark.parametrize("fp64", [0, 1])
def test_every_tuned_shape_gives_the_same_bits(lib, fp64):
    """exa_inverse_autotune picks one of the column-by-warp shapes per order; whatever it
    picks, the inverse is the same to the bit, because every shape performs the same
    operations with the same pivots.  The same blocks of orders 96 and 125 are inverted with
    the untuned default shape and again after tuning: the results must be identical.  (In a
    session where an earlier test already tuned the order, both runs use the tuned shape and
    the check holds trivially.)"""
    import torch
    dt, inv = (torch.float64, lib.exa_dinverse_batched) if fp64 else (torch.float32, lib.exa_sinverse_batched)
    for n in (96, 125):
        rng = np.random.default_rng(100 + n)
        batch = 300
        # diagonally weighted (cond ~ 1e2), then the rows shuffled, so partial pivoting has to
        # find the permutation
        A = rng.standard_normal((batch, n, n)) + np.eye(n) * (2.0 * np.sqrt(n))
        A = np.stack([a[rng.permutation(n)] for a in A])
        host = np.ascontiguousarray(np.transpose(A, (0, 2, 1))).ravel()
        outs = []
        for tune in (False, True):
            if tune:
                v = ctypes.c_int(-2)
                assert lib.exa_inverse_autotune(n, fp64, batch, None, ctypes.byref(v)) == 0, lib.exa_last_error().decode()
                assert 0 <= v.value <= 3
                w = ctypes.c_int(-2)
                assert lib.exa_inverse_autotune(n, fp64, batch, None, ctypes.byref(w)) == 0
                assert w.value == v.value                       # kept after the first call
            dev = torch.tensor(host, dtype=dt, device="cuda")
            flag = torch.zeros(1, dtype=torch.int32, device="cuda")
            st = inv(ctypes.c_void_p(dev.data_ptr()), n, n * n, batch, ctypes.c_void_p(flag.data_ptr()), None)
            assert st == 0, lib.exa_last_error().decode()
            torch.cuda.synchronize()
            outs.append(dev.cpu().numpy())
        assert np.array_equal(outs[0], outs[1])
        ref = np.linalg.inv(A)
        got = np.transpose(outs[1].reshape(batch, n, n), (0, 2, 1))
        tol = 1e-12 if fp64 else 1e-4
        assert np.abs(got - ref).max() / np.abs(ref).max() < tol
    v = ctypes.c_int(-2)
    assert lib.exa_inverse_autotune(200, fp64, 8, None, ctypes.byref(v)) == 0 and v.value == -1

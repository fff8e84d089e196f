"""Failure detection through the C ABI, in the forms that fault and hang no GPU.

* A NaN in the state: the reference's damped Newton loop halves the step while the residual
  is NaN (backend/Solution/solution.cpp:211-225, with no exit); here the solve ends with
  status 7 (EXA_ERR_NAN) once the step length falls below 1e-12, and the context stays usable.
* GMRES stopped by its iteration cap above its tolerance: the reference prints a warning with
  the relative error (backend/Solver/gmres.cpp:586-594); the standalone call returns status 6
  (EXA_ERR_NOTCONV) with that error in its message, while a Newton step goes on as the
  reference's does.
* A bounded wait inside the tensor-core GEMM that runs out: a test hook sets the main-loop
  waits of the 3xTF32 kernel to give up at once.  The kernel then drains the bulk copies and
  MMAs it started (at the normal limit), frees its tensor memory and sets its flag to 2; the
  mixed-form solver reports status 3.  With the normal limit back, the same calls succeed.
"""
import ctypes
import os

import numpy as np
import pytest

from exasim_b200 import ExaError, HDGSolver, build as B, cases, load_library

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build(["poisson2d"])


def _set_problem_entry(datain, index, value):
    """Entry `index` of app.bin's problem part (13 NewtonIter, 14 GMRESiter, 15 GMRESrestart;
    layout of readpdeapp.cpp:820-918)."""
    fn = os.path.join(datain, "app.bin")
    a = np.fromfile(fn, dtype=np.float64)
    ls = int(a[0])
    ns = a[1:1 + ls].astype(np.int64)
    a[1 + ls + int(ns[0] + ns[1]) + index] = value
    a.tofile(fn)


def test_nan_state_returns_nan_status_and_context_recovers(tmp_path):
    d = cases.poisson2d_tri(str(tmp_path / "datain"), n=3)
    _set_problem_entry(d, 14, 60)   # a short GMRES cap: GMRES cannot converge on NaN
    s = HDGSolver(d, "poisson2d")
    udg = s.get("udg")
    udg[7] = np.nan
    s.set("udg", udg)
    with pytest.raises(ExaError) as e:
        s.NewtonSolver()
    assert e.value.code == 7, str(e.value)
    s.set("udg", np.zeros_like(udg))
    s.set("uh", np.zeros(s.field_size("uh")))
    _, nrm = s.NewtonSolver()
    assert nrm < 1e-6
    s.close()


def test_gmres_iteration_cap_returns_not_converged(tmp_path):
    d = cases.poisson2d_tri(str(tmp_path / "datain"), n=4)
    _set_problem_entry(d, 14, 3)
    s = HDGSolver(d, "poisson2d")
    s.hdgGetQ()
    s.hdgAssembleLinearSystem()
    with pytest.raises(ExaError) as e:
        s.GMRES()
    assert e.value.code == 6, str(e.value)
    assert "within 3 iterations" in str(e.value) and "relative error" in str(e.value)
    # inside Newton the unconverged step goes on, as in the reference: one step, not converged
    its, nrm = s.NewtonSolver()
    assert its == 1 and nrm > 1e-10
    s.close()


def test_tensor_core_wait_timeout_sets_flag_and_recovers(tmp_path):
    import torch
    L = load_library("poisson2d")
    M = N = 125
    K, nb = 375, 9
    rng = np.random.default_rng(5)
    A = torch.tensor(rng.standard_normal((nb, K, M)), dtype=torch.float64, device="cuda")
    Bm = torch.tensor(rng.standard_normal((nb, N, K)), dtype=torch.float64, device="cuda")
    C = torch.zeros((nb, N, M), dtype=torch.float32, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    P = lambda t: ctypes.c_void_p(t.data_ptr())

    def gemm():
        return L.exa_gemm_3xtf32_batched(M, N, K, 1.0, P(A), 1, M, K * M, P(Bm), 1, K, N * K, 0.0, P(C), M, N * M,
                                         nb, P(flag), None)

    try:
        L.exa_debug_umma_wait_polls(0)
        assert gemm() == 0, L.exa_last_error().decode()
        torch.cuda.synchronize()
        assert int(flag.item()) == 2
        # the mixed form reports the run-out wait as status 3 (EXA_ERR_CUDA)
        d = cases.poisson2d_tri(str(tmp_path / "datain"), n=3)
        s = HDGSolver(d, "poisson2d")
        s.set_precision(1, 1e-4, 1e-8)
        with pytest.raises(ExaError) as e:
            s.NewtonSolver()
        assert e.value.code == 3, str(e.value)
    finally:
        L.exa_debug_umma_wait_polls(-1)
    flag.zero_()
    assert gemm() == 0, L.exa_last_error().decode()
    torch.cuda.synchronize()
    assert int(flag.item()) == 0
    ref = torch.einsum("bkm,bnk->bnm", A, Bm)
    assert float((C.double() - ref).abs().max() / ref.abs().max()) < 1e-5
    s2 = HDGSolver(d, "poisson2d")
    s2.set_precision(1, 1e-4, 1e-8)
    s2.set("udg", np.zeros(s2.field_size("udg")))
    _, nrm = s2.NewtonSolver()
    r0, r1 = s2.last_residual()
    assert r1 <= 1e-8 * r0
    s.close()
    s2.close()

"""The fixed-scratch column-norm entry point (exa_dnrm2_cols_fixed), called through the C
ABI.  Its norms must reproduce the residual norm that exa_residual reports (|b| + |Ru|,
computed with the context's own allocated partials), on two calls in a row, and it must
refuse more columns than its fixed scratch holds.  The file sorts last so the entry point
also runs after every other GPU test of the session."""
import ctypes

import numpy as np
import pytest

from exasim_b200 import HDGSolver, build as B, cases

pytestmark = pytest.mark.gpu
TOL = 1e-14


def test_fixed_scratch_norms_match_residual_norm(tmp_path):
    import torch
    B.build(["poisson2d"])
    d = str(tmp_path / "datain")
    cases.poisson2d_tri(d, n=4)
    s = HDGSolver(d, "poisson2d")
    L = s.lib
    st = ctypes.c_void_p(s.stream())
    torch.cuda.set_device(0)
    nrm = s.hdgAssembleResidual()
    b, nb = s.field_ptr("b")
    ru, nru = s.field_ptr("Ru")
    out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
    results = []
    for _ in range(2):
        for k, (p, n) in enumerate(((b, nb), (ru, nru))):
            rc = L.exa_dnrm2_cols_fixed(ctypes.c_void_p(p), n, n, 1, ctypes.c_void_p(out.data_ptr() + 8 * k), st)
            assert rc == 0, L.exa_last_error().decode()
        assert L.exa_synchronize(s.h) == 0
        v = out.cpu().numpy()
        results.append(v[0] + v[1])
    assert results[0] == results[1]
    assert abs(results[0] - nrm) <= TOL * nrm, (results, nrm)
    # several columns in one call: the field copies side by side, against numpy
    X = torch.zeros((3, nru), dtype=torch.float64, device="cuda")
    ru_host = s.get("Ru")
    for j in range(3):
        X[j].copy_(torch.from_numpy(ru_host * (j + 1)))
    torch.cuda.synchronize()
    for _ in range(2):
        out.fill_(-1.0)
        torch.cuda.synchronize()
        rc = L.exa_dnrm2_cols_fixed(ctypes.c_void_p(X.data_ptr()), nru, nru, 3, ctypes.c_void_p(out.data_ptr()),
                                    None)
        assert rc == 0, L.exa_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()[:3]
        ref = np.linalg.norm(ru_host) * np.arange(1, 4)
        assert np.abs(got - ref).max() <= TOL * ref.max() * 10, (got, ref)
        assert out.cpu().numpy()[3] == -1.0
    # more columns than the fixed scratch holds: refused on the host, nothing launched
    before = L.exa_launch_count()
    rc = L.exa_dnrm2_cols_fixed(ctypes.c_void_p(X.data_ptr()), 1, 1, 65, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1 and "65" in L.exa_last_error().decode()
    assert L.exa_launch_count() == before
    s.close()


def test_fixed_scratch_norms_at_its_limits():
    """The full 64 columns, strided (ldx > n), of a vector long enough that the grid-stride
    loop runs more than once per block (n > 296 * 256), and n = 0, whose norms are 0; each on
    two calls in a row."""
    import torch
    B.build(["poisson2d"])
    from exasim_b200 import load_library
    L = load_library("poisson2d")
    n, ldx, nc = 200_003, 200_011, 64
    rng = np.random.default_rng(9)
    X = torch.tensor(rng.standard_normal((nc, ldx)), dtype=torch.float64, device="cuda")
    out = torch.full((nc + 1,), -1.0, dtype=torch.float64, device="cuda")
    ref = np.linalg.norm(X.cpu().numpy()[:, :n], axis=1)
    for _ in range(2):
        rc = L.exa_dnrm2_cols_fixed(ctypes.c_void_p(X.data_ptr()), n, ldx, nc, ctypes.c_void_p(out.data_ptr()), None)
        assert rc == 0, L.exa_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.abs(got[:nc] - ref).max() <= 1e-13 * ref.max()
        assert got[nc] == -1.0
    for _ in range(2):
        out.fill_(-1.0)
        rc = L.exa_dnrm2_cols_fixed(ctypes.c_void_p(X.data_ptr()), 0, ldx, 3, ctypes.c_void_p(out.data_ptr()), None)
        assert rc == 0, L.exa_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(got[:3] == 0.0) and got[3] == -1.0

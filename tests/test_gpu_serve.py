"""Serving (continuous batching of independent solves, exa_server_* in the C ABI) on the
served stream's model: 2D convection-diffusion with parametrised kappa, velocity and source.

Every reduction of a solve runs in a fixed order whatever else shares the device, so a
request's result in the mix must equal its result alone: the test compares them entry by
entry (tolerance 0), for plain and mixed-precision requests, with contexts created fresh
and reused.  Admission by memory budget is checked through the server's counters."""
import numpy as np
import pytest

from exasim_b200 import ExaError, HDGSolver, build as B
from exasim_b200.serve import CaseCache, Server, stream_requests, with_params

pytestmark = pytest.mark.gpu
MODEL = "cdsin2d"


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build([MODEL])


@pytest.fixture(scope="module")
def cache():
    return CaseCache()


def requests(cache, count, seed, n_range=(8, 14)):
    out = []
    for _, n, p, params in stream_requests(count, 0.0, seed=seed, n_range=n_range):
        b = cache.get(n, p)
        out.append([with_params(b[0], params)] + b[1:])
    return out


def alone(blobs, precision=0):
    s = HDGSolver("", MODEL, blobs=blobs)
    if precision:
        s.set_precision(1, inner_tol=1e-4, rtol=1e-10)
    s.NewtonSolver()
    r = s.get("udg"), s.get("uh")
    s.close()
    return r


@pytest.mark.parametrize("precision", [0, 1])
def test_results_in_the_mix_equal_results_alone(cache, precision):
    reqs = requests(cache, 16, seed=3 + precision)
    ref = [alone(b, precision) for b in reqs]
    with Server(MODEL, slots=6, hbm_budget=8 << 30) as srv:
        # two passes: the second reuses the contexts the first left resident
        for rep in range(2):
            ids = [srv.submit(b, precision=precision, inner_tol=1e-4, rtol=1e-10) for b in reqs]
            res = [srv.wait(i) for i in ids]
            for (u_ref, h_ref), r in zip(ref, res):
                assert np.array_equal(r.udg, u_ref) and np.array_equal(r.uh, h_ref)
                assert r.latency_ms >= r.run_ms >= 0.0
            if rep == 1:
                assert all(r.reused for r in res)
        st = srv.stats()
        assert st["done"] == 2 * len(reqs) and st["failed"] == 0
        assert st["contexts_reused"] >= len(reqs)


def test_admission_by_memory_budget(cache):
    reqs = requests(cache, 10, seed=7, n_range=(16, 24))
    ref = [alone(b) for b in reqs]
    # a budget smaller than any one context: requests run one at a time, nothing is kept
    with Server(MODEL, slots=4, hbm_budget=1) as srv:
        ids = [srv.submit(b) for b in reqs]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    for (u_ref, h_ref), r in zip(ref, res):
        assert np.array_equal(r.uh, h_ref)
    assert st["done"] == len(reqs)
    biggest = max(r.run_ms for r in res)
    assert biggest > 0
    # one context at a time: each later request reuses the resident one (same mesh) or evicts it
    assert st["contexts_evicted"] + st["contexts_reused"] == len(reqs) - 1
    assert st["contexts_idle"] == 1 and st["bytes_held"] <= st["peak_bytes_held"]


def test_failed_request_does_not_stop_the_server(cache):
    good = requests(cache, 2, seed=11)
    bad = [b.copy() for b in good[0]]
    bad[0] = with_params(bad[0], [1.0, 0.0, 0.0, 1.0, 1.0])
    # an app asking for a polynomial preconditioner of higher degree than the GMRES restart,
    # which this path refuses
    ls = int(bad[0][0])
    nsize = bad[0][1:1 + ls].astype(np.int64)
    off = 1 + ls + int(nsize[:2].sum()) + 27
    bad[0][off] = 1000.0
    with Server(MODEL, slots=2) as srv:
        with pytest.raises(ExaError) as e:
            srv.wait(srv.submit(bad))
        assert e.value.code == 2
        r = srv.wait(srv.submit(good[1]))
        u_ref, h_ref = alone(good[1])
        assert np.array_equal(r.uh, h_ref)
        with pytest.raises(ExaError):
            srv.submit([bad[0][:3]] + bad[1:])

"""Batched Krylov steps across served solves (exa_server_set_batching): the GMRES calls of
all running requests share one set of launches per Arnoldi step.

Each job's reductions keep a fixed partition and order that depend on its own sizes only, so
a request's result must not depend on what else is in the batch: solved with 12 requests in
flight it must equal, entry by entry, its result through the same batched server one at a
time.  Against the unbatched solve of the same request (whose matvec sums in another order)
the trace solution must agree within the GMRES tolerance of the request (1e-11 plain; the
mixed form's refinement target 1e-10 for its residual ratio)."""
import numpy as np
import pytest

from exasim_b200 import HDGSolver, build as B
from exasim_b200.serve import CaseCache, Server, stream_requests, with_params

pytestmark = pytest.mark.gpu
MODEL = "cdsin2d"


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build([MODEL])


@pytest.fixture(scope="module")
def cache():
    return CaseCache()


def requests(cache, count, seed, n_range=(8, 20)):
    out = []
    for _, n, p, params in stream_requests(count, 0.0, seed=seed, n_range=n_range):
        b = cache.get(n, p)
        out.append([with_params(b[0], params)] + b[1:])
    return out


def unbatched(blobs, precision):
    s = HDGSolver("", MODEL, blobs=blobs)
    if precision:
        s.set_precision(1, inner_tol=1e-4, rtol=1e-10)
    s.NewtonSolver()
    uh = s.get("uh")
    s.close()
    return uh


@pytest.mark.parametrize("precision", [0, 1])
def test_batched_results_do_not_depend_on_the_batch(cache, precision):
    reqs = requests(cache, 12, seed=21 + precision)
    kw = dict(precision=precision, inner_tol=1e-4, rtol=1e-10)
    with Server(MODEL, slots=1, hbm_budget=8 << 30, batch=16) as one:
        solo = [one.wait(one.submit(b, **kw)) for b in reqs]
    with Server(MODEL, slots=12, hbm_budget=8 << 30, batch=16) as srv:
        ids = [srv.submit(b, **kw) for b in reqs]
        mix = [srv.wait(i) for i in ids]
        bs = srv.batch_stats()
    for a, b in zip(solo, mix):
        assert np.array_equal(a.uh, b.uh) and np.array_equal(a.udg, b.udg)
        assert a.gmres == b.gmres
    assert bs["gmres_calls"] >= len(reqs) and bs["steps"] > 0
    assert bs["matvec_elements_per_warp"] in (1, 2, 4, 8)
    # the same requests unbatched: the same solution within the solve's tolerance
    for b, r in zip(reqs, mix):
        ref = unbatched(b, precision)
        assert np.linalg.norm(r.uh - ref) / np.linalg.norm(ref) < (1e-9 if precision == 0 else 1e-8)
        assert r.residual <= 1e-8 * r.residual0


def test_batched_steps_are_shared(cache):
    """12 requests in flight take far fewer batched steps than their GMRES iterations in all."""
    reqs = requests(cache, 12, seed=5)
    with Server(MODEL, slots=12, hbm_budget=8 << 30, batch=16) as srv:
        res = [srv.wait(i) for i in [srv.submit(b) for b in reqs]]
        bs = srv.batch_stats()
    total = sum(r.gmres for r in res)
    assert bs["steps"] < total / 2, (bs, total)

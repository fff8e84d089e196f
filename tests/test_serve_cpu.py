"""CPU checks of the served stream's request generation (exasim_b200.serve)."""
import numpy as np

from exasim_b200 import inputs as I
from exasim_b200.serve import CaseCache, stream_requests, with_params


def test_stream_distribution():
    rs = stream_requests(4000, 100.0, seed=1)
    t = np.array([r[0] for r in rs])
    assert np.all(np.diff(t) >= 0)
    assert abs(len(rs) / t[-1] - 100.0) < 10.0
    ns = np.array([r[1] for r in rs])
    ps = np.array([r[2] for r in rs])
    assert ns.min() == 8 and ns.max() == 64 and set(ps) == {2, 3, 4}
    kap = np.array([r[3][0] for r in rs])
    assert kap.min() >= 1e-3 and kap.max() <= 1.0 and abs(np.median(np.log10(kap)) + 1.5) < 0.1
    speed = np.hypot([r[3][1] for r in rs], [r[3][2] for r in rs])
    assert np.allclose(speed, 1.0)


def test_with_params_replaces_only_the_parameters():
    c = CaseCache()
    app = c.get(8, 2)[0]
    new = with_params(app, [0.5, 0.6, 0.8, 2.0, 3.0])
    a, b = I.read_blob(app.tobytes()), I.read_blob(new.tobytes())
    assert np.array_equal(b[7], [0.5, 0.6, 0.8, 2.0, 3.0])
    for i in range(len(a)):
        if i != 7:
            assert np.array_equal(a[i], b[i])

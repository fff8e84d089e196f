"""Serving many independent HDG solves on one GPU (continuous batching).

``Server`` wraps the library's request loop (``exa_server_*`` in include/exasim_b200.h): a
fixed number of slots, each a host thread driving one solve on its own context and CUDA
stream; requests are admitted in arrival order as slots and device memory (a byte budget)
free up, and contexts of finished requests stay resident for later requests on the same
mesh.  ``stream_requests`` makes the parametrised request stream of the served benchmark:
2D convection-diffusion on n x n quadrilaterals of the unit square, kappa log-uniform in
[1e-3, 1], velocity (cos theta, sin theta), p in {2, 3, 4}, n in {8, ..., 64}, source
sin(a pi x) sin(b pi y) with seeded integers a, b, and Poisson arrival times.
"""
from __future__ import annotations

import ctypes
import os
import tempfile
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import ExaError, _ptr, load_library, read_datain


@dataclass
class Result:
    udg: np.ndarray
    uh: np.ndarray
    queued_ms: float
    run_ms: float
    latency_ms: float
    newton: int
    gmres: int
    residual0: float
    residual: float
    reused: bool


class Server:
    def __init__(self, model: str, device: int = 0, hbm_budget: int = 16 << 30, slots: int = 8,
                 reuse_contexts: bool = True, batch: int = 0):
        """batch > 0: the running solves' GMRES calls share batched Arnoldi steps (that many job
        slots; exa_server_set_batching)."""
        self.lib = load_library(model)
        h = ctypes.c_void_p()
        self._check(self.lib.exa_server_create(device, int(hbm_budget), int(slots), int(bool(reuse_contexts)),
                                               ctypes.byref(h)))
        self.h = h
        if batch > 0:
            self._check(self.lib.exa_server_set_batching(self.h, int(batch)))

    def batch_stats(self) -> Dict[str, int]:
        out = (ctypes.c_longlong * 4)()
        self._check(self.lib.exa_server_batch_stats(self.h, out))
        return {k: int(v) for k, v in zip(["steps", "launches", "gmres_calls", "matvec_elements_per_warp"], out)}

    def _check(self, st: int):
        if st != 0:
            raise ExaError(st, self.lib.exa_last_error().decode())

    def submit(self, blobs: Sequence[np.ndarray], precision: int = 0, inner_tol: float = 1e-4,
               rtol: float = 0.0) -> int:
        b = [np.ascontiguousarray(x, dtype=np.float64) for x in blobs]
        rid = ctypes.c_longlong()
        self._check(self.lib.exa_server_submit(self.h, _ptr(b[0]), b[0].size, _ptr(b[1]), b[1].size, _ptr(b[2]),
                                               b[2].size, _ptr(b[3]), b[3].size, int(precision), float(inner_tol),
                                               float(rtol), ctypes.byref(rid)))
        return int(rid.value)

    def wait(self, rid: int, timeout: Optional[float] = None) -> Result:
        nu, nh = ctypes.c_longlong(), ctypes.c_longlong()
        st = self.lib.exa_server_wait(self.h, rid, -1.0 if timeout is None else float(timeout), ctypes.byref(nu),
                                      ctypes.byref(nh))
        if st != 0:
            msg = self.lib.exa_last_error().decode()
            if st != 9:  # a failed request is forgotten once reported
                self.lib.exa_server_fetch(self.h, rid, None, 0, None, 0, None)
            raise ExaError(st, msg)
        udg, uh = np.empty(nu.value), np.empty(nh.value)
        info = (ctypes.c_double * 8)()
        self._check(self.lib.exa_server_fetch(self.h, rid, _ptr(udg), udg.size, _ptr(uh), uh.size, info))
        return Result(udg, uh, info[0], info[1], info[2], int(info[3]), int(info[4]), info[5], info[6], bool(info[7]))

    def stats(self) -> Dict[str, int]:
        out = (ctypes.c_longlong * 10)()
        self._check(self.lib.exa_server_stats(self.h, out))
        names = ["queued", "running", "done", "failed", "bytes_held", "peak_bytes_held", "contexts_created",
                 "contexts_reused", "contexts_idle", "contexts_evicted"]
        return {k: int(v) for k, v in zip(names, out)}

    def close(self):
        if getattr(self, "h", None):
            self.lib.exa_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# ------------------------------------------------------------------ request stream
PARAM_PART = 6  # physicsparam is part 6 of app.bin (readappstruct)


def with_params(app: np.ndarray, params: Sequence[float]) -> np.ndarray:
    """A copy of an app.bin blob with its physical parameters replaced (same count)."""
    a = app.copy()
    ls = int(a[0])
    nsize = a[1:1 + ls].astype(np.int64)
    if int(nsize[PARAM_PART]) != len(params):
        raise ValueError(f"app.bin holds {nsize[PARAM_PART]} parameters, got {len(params)}")
    off = 1 + ls + int(nsize[:PARAM_PART].sum())
    a[off:off + len(params)] = params
    return a


class CaseCache:
    """Blobs of the served model's (n, p) meshes, written once per shape.  The GMRES tolerance
    1e-11 on the preconditioned residual brings the plain form's one Newton step to a true
    residual ratio below 1e-8 on every request of the stream."""

    def __init__(self, gmres_tol: float = 1e-11):
        self.tmp = tempfile.TemporaryDirectory()
        self.blobs: Dict[Tuple[int, int], List[np.ndarray]] = {}
        self.gmres_tol = gmres_tol

    def get(self, n: int, p: int) -> List[np.ndarray]:
        if (n, p) not in self.blobs:
            from . import cases
            d = os.path.join(self.tmp.name, f"n{n}p{p}")
            cases.cdsin2d_quad(d, n=n, porder=p, gmres_tol=self.gmres_tol)
            self.blobs[(n, p)] = read_datain(d)
        return self.blobs[(n, p)]


def stream_requests(count: int, rate: float, seed: int = 0, n_range=(8, 64), p_choices=(2, 3, 4)):
    """[(arrival time s, n, p, params)] of the served stream; params = [kappa, cx, cy, a, b]."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=count)) if rate > 0 else np.zeros(count)
    out = []
    for i in range(count):
        kappa = float(10.0 ** rng.uniform(-3.0, 0.0))
        th = float(rng.uniform(0.0, 2.0 * np.pi))
        p = int(rng.choice(p_choices))
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        a, b = int(rng.integers(1, 4)), int(rng.integers(1, 4))
        out.append((float(t[i]), n, p, [kappa, float(np.cos(th)), float(np.sin(th)), float(a), float(b)]))
    return out

"""B200-native HDG implicit solver with Exasim's inputs and model plugins.

Python mirror of the solver's host interface.  The numerical work runs in the CUDA
library ``lib/libexasim_b200_<model>.so`` (C ABI: ``include/exasim_b200.h``); this
module only loads it, passes Exasim's ``datain/*.bin`` files in, and exposes the
steps under the names of the reference's C++ methods
(``CDiscretization::hdgAssembleLinearSystem``, ``hdgAssembleResidual``, ``evalMatVec``,
``CPreconditioner::ApplyPreconditioner``, ``GMRES``, ``CSolution::NewtonSolver``, DIRK).
There is no CPU fallback: a missing library or device raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Optional, Sequence

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
_LIBS: Dict[str, ctypes.CDLL] = {}

STATUS = {0: "ok", 1: "bad argument", 2: "unsupported input", 3: "CUDA error", 4: "singular block",
          5: "mesh error", 6: "not converged", 7: "NaN residual", 8: "out of device memory",
          9: "wait timed out"}


class ExaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def lib_path(model: str) -> str:
    return os.path.join(PKG, "lib", f"libexasim_b200_{model}.so")


def load_library(model: str) -> ctypes.CDLL:
    """Load the compiled solver for `model` (built by ``python -m exasim_b200.build``)."""
    if model in _LIBS:
        return _LIBS[model]
    path = lib_path(model)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing; run `python -m exasim_b200.build {model}`")
    L = ctypes.CDLL(path)
    P, D, I, LL = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_longlong
    PD, PI, PLL = ctypes.POINTER(D), ctypes.POINTER(I), ctypes.POINTER(LL)
    sig = {
        "exa_last_error": ([], ctypes.c_char_p),
        "exa_create": ([P, LL, P, LL, P, LL, P, LL, I, ctypes.POINTER(P)], I),
        "exa_destroy": ([P], None),
        "exa_sizes": ([P, PLL], I),
        "exa_get_field": ([P, ctypes.c_char_p, P, LL], I),
        "exa_set_field": ([P, ctypes.c_char_p, P, LL], I),
        "exa_field_ptr": ([P, ctypes.c_char_p, ctypes.POINTER(P), PLL], I),
        "exa_get_connectivity": ([P, P, P], I),
        "exa_set_time": ([P, D, D], I),
        "exa_set_step_time": ([P, D], I),
        "exa_assemble": ([P], I),
        "exa_residual": ([P, PD], I),
        "exa_matvec": ([P, P, P], I),
        "exa_precond": ([P, P, P], I),
        "exa_gmres": ([P, PI, PD], I),
        "exa_getq": ([P], I),
        "exa_newton": ([P, PI, PD], I),
        "exa_dirk": ([P, I, P, I], I),
        "exa_solve": ([P, P, P, P, P, PI, PD], I),
        "exa_stats": ([P, PLL], I),
        "exa_synchronize": ([P], I),
        "exa_connectivity_host": ([P, P, P, P, I, I, I, I, I, P, P, PI], I),
        "exa_dirk_stage": ([P, I, I, PI, PD], I),
        "exa_stream": ([P, ctypes.POINTER(P)], I),
        "exa_launch_count": ([], LL),
        "exa_debug_umma_wait_polls": ([LL], None),
        "exa_poly_ritz": ([P, I, P, P], I),
        "exa_dgemm_batched": ([I, I, I, D, P, LL, LL, P, LL, LL, D, P, LL, LL, I, P], I),
        "exa_dinverse_batched": ([P, I, LL, I, P, P], I),
        "exa_sinverse_batched": ([P, I, LL, I, P, P], I),
        "exa_dgemm_tune": ([I, I, I, I, P, PI], I),
        "exa_inverse_autotune": ([I, I, I, P, PI], I),
        "exa_dnrm2_cols_fixed": ([P, LL, LL, I, P, P], I),
        "exa_gemm_tf32_batched": ([I, I, I, D, P, I, LL, LL, P, I, LL, LL, D, P, I, LL, LL, I, P, P], I),
        "exa_gemm_3xtf32_batched": ([I, I, I, D, P, I, LL, LL, P, I, LL, LL, D, P, LL, LL, I, P, P], I),
        "exa_profile": ([P, I], I),
        "exa_set_precision": ([P, I, D, D], I),
        "exa_bilu0_ordering": ([P, I, P, I, I, I, P, I, P, I, P, I, PI], I),
        "exa_last_residual": ([P, PD, PD], I),
        "exa_profile_read": ([P, I, PD, PLL, PD], I),
        "exa_server_create": ([I, LL, I, I, ctypes.POINTER(P)], I),
        "exa_server_submit": ([P, P, LL, P, LL, P, LL, P, LL, I, D, D, PLL], I),
        "exa_server_wait": ([P, LL, D, PLL, PLL], I),
        "exa_server_fetch": ([P, LL, P, LL, P, LL, PD], I),
        "exa_server_stats": ([P, PLL], I),
        "exa_server_destroy": ([P], None),
        "exa_server_set_batching": ([P, I], I),
        "exa_server_batch_stats": ([P, PLL], I),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIBS[model] = L
    return L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def read_datain(datain: str):
    """The four float64 blobs of an Exasim datain/ folder."""
    return [np.fromfile(os.path.join(datain, f + ".bin"), dtype=np.float64) for f in ("app", "master", "mesh", "sol")]


class HDGSolver:
    """One mesh + model on one GPU (a CDiscretization + CSolution of the reference)."""

    def __init__(self, datain: str, model: str, device: int = 0, blobs: Optional[Sequence[np.ndarray]] = None):
        self.model = model
        self.lib = load_library(model)
        b = [np.ascontiguousarray(x, dtype=np.float64) for x in (blobs or read_datain(datain))]
        h = ctypes.c_void_p()
        st = self.lib.exa_create(_ptr(b[0]), b[0].size, _ptr(b[1]), b[1].size, _ptr(b[2]), b[2].size,
                                 _ptr(b[3]), b[3].size, device, ctypes.byref(h))
        self._check(st)
        self.h = h
        s = (ctypes.c_longlong * 16)()
        self._check(self.lib.exa_sizes(self.h, s))
        names = ["ne", "nf", "nf0", "npe", "npf", "nfe", "nc", "ncu", "nd", "n", "m", "ndofuhat", "nge",
                 "ngf", "neb", "preconditioner"]
        self.sizes = {k: int(v) for k, v in zip(names, s)}

    def _check(self, st: int):
        if st != 0:
            raise ExaError(st, self.lib.exa_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.exa_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- data access
    def field_size(self, name: str) -> int:
        p, n = ctypes.c_void_p(), ctypes.c_longlong()
        self._check(self.lib.exa_field_ptr(self.h, name.encode(), ctypes.byref(p), ctypes.byref(n)))
        return int(n.value)

    def field_ptr(self, name: str):
        p, n = ctypes.c_void_p(), ctypes.c_longlong()
        self._check(self.lib.exa_field_ptr(self.h, name.encode(), ctypes.byref(p), ctypes.byref(n)))
        return p.value, int(n.value)

    def get(self, name: str) -> np.ndarray:
        a = np.empty(self.field_size(name), dtype=np.float64)
        self._check(self.lib.exa_get_field(self.h, name.encode(), _ptr(a), a.size))
        return a

    def set(self, name: str, values: np.ndarray):
        a = np.ascontiguousarray(values, dtype=np.float64).ravel(order="F")
        self._check(self.lib.exa_set_field(self.h, name.encode(), _ptr(a), a.size))

    def connectivity(self):
        nf, ne, ndf = self.sizes["nf"], self.sizes["ne"], self.sizes["npf"] * self.sizes["nfe"]
        f2e = np.empty(4 * nf, dtype=np.int32)
        ec = np.empty(ndf * ne, dtype=np.int32)
        self._check(self.lib.exa_get_connectivity(self.h, _ptr(f2e), _ptr(ec)))
        return f2e.reshape(4, nf, order="F"), ec.reshape(ndf, ne, order="F")

    def set_time(self, time: float, dtfactor: float):
        self._check(self.lib.exa_set_time(self.h, time, dtfactor))

    def set_step_time(self, time0: float):
        """Start time of the next DIRK step (a restart at step R: R dt[0])."""
        self._check(self.lib.exa_set_step_time(self.h, time0))

    # ---- the reference's steps
    def hdgAssembleLinearSystem(self):
        self._check(self.lib.exa_assemble(self.h))

    def hdgAssembleResidual(self) -> float:
        nrm = ctypes.c_double()
        self._check(self.lib.exa_residual(self.h, ctypes.byref(nrm)))
        return nrm.value

    def evalMatVec(self, v_dev: int, w_dev: int):
        """w = A v on device pointers (e.g. torch.Tensor.data_ptr())."""
        self._check(self.lib.exa_matvec(self.h, ctypes.c_void_p(v_dev), ctypes.c_void_p(w_dev)))

    def ApplyPreconditioner(self, v_dev: int, w_dev: int):
        self._check(self.lib.exa_precond(self.h, ctypes.c_void_p(v_dev), ctypes.c_void_p(w_dev)))

    def GMRES(self):
        it, re = ctypes.c_int(), ctypes.c_double()
        self._check(self.lib.exa_gmres(self.h, ctypes.byref(it), ctypes.byref(re)))
        return it.value, re.value

    def hdgGetQ(self):
        self._check(self.lib.exa_getq(self.h))

    def evalResidual(self) -> float:
        """LDG contexts (problem[0] = 0): R(u) of the current element states into the field
        "Ru", returning |R| (CDiscretization::evalResidual, discretization.cpp:604-612)."""
        return self.hdgAssembleResidual()

    def PTCsolver(self):
        """LDG contexts: the pseudo-transient solve of R(u) = 0 (ptcsolver.cpp:255-330);
        returns (PTC steps, |R|).  An HDG context runs its Newton solve."""
        return self.NewtonSolver()

    def NewtonSolver(self):
        it, nrm = ctypes.c_int(), ctypes.c_double()
        self._check(self.lib.exa_newton(self.h, ctypes.byref(it), ctypes.byref(nrm)))
        return it.value, nrm.value

    def DIRK(self, nsteps: int):
        its = np.zeros(max(1, nsteps * 8), dtype=np.int32)
        self._check(self.lib.exa_dirk(self.h, nsteps, _ptr(its), its.size))
        return its

    def DIRKStage(self, istep: int, stage: int):
        it, nrm = ctypes.c_int(), ctypes.c_double()
        self._check(self.lib.exa_dirk_stage(self.h, istep, stage, ctypes.byref(it), ctypes.byref(nrm)))
        return it.value, nrm.value

    def stream(self) -> int:
        p = ctypes.c_void_p()
        self._check(self.lib.exa_stream(self.h, ctypes.byref(p)))
        return int(p.value or 0)

    def solve(self, udg: Optional[np.ndarray] = None, uh: Optional[np.ndarray] = None,
              udg_out: Optional[np.ndarray] = None, uh_out: Optional[np.ndarray] = None):
        """One Newton solve with host buffers in and out (the end-to-end call)."""
        it, nrm = ctypes.c_int(), ctypes.c_double()
        P = lambda a: _ptr(a) if a is not None else None
        self._check(self.lib.exa_solve(self.h, P(udg), P(uh), P(udg_out), P(uh_out), ctypes.byref(it),
                                       ctypes.byref(nrm)))
        return it.value, nrm.value

    def set_precision(self, mode: int, inner_tol: float = 1e-4, rtol: float = 0.0):
        """0: plain FP64.  1: FP32/TF32 element elimination with FP64 residual refinement."""
        self._check(self.lib.exa_set_precision(self.h, int(mode), float(inner_tol), float(rtol)))

    def last_residual(self):
        """(initial, final) residual norm |b| + |Ru| of the last Newton solve."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.exa_last_residual(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    PHASES = ("volume", "face", "qelim", "inverse", "schur", "precond_build", "matvec", "precond_apply",
              "orthogonalize", "getq", "residual", "pack", "update")

    def profile(self, enable: bool):
        """Start (resetting the totals) or stop the per-phase device timers."""
        self._check(self.lib.exa_profile(self.h, 1 if enable else 0))

    def profile_read(self):
        """{phase: (ms, timed regions, algorithmic GEMM FLOPs)} accumulated since profile(True)."""
        n = len(self.PHASES)
        ms, cnt, fl = (ctypes.c_double * n)(), (ctypes.c_longlong * n)(), (ctypes.c_double * n)()
        self._check(self.lib.exa_profile_read(self.h, n, ms, cnt, fl))
        return {p: (float(ms[i]), int(cnt[i]), float(fl[i])) for i, p in enumerate(self.PHASES)}

    def stats(self):
        s = (ctypes.c_longlong * 4)()
        self._check(self.lib.exa_stats(self.h, s))
        return {"gmres_iters": int(s[0]), "newton_iters": int(s[1]), "gmres_total": int(s[2])}

"""The mixed-precision refinement restated on the CPU (oracle.hdg.HDGOracle.newton_mixed):
condensed blocks, factors and preconditioner of one assembly rounded to FP32, FP64 residual
refinement.  It reaches the FP64 residual ratio and the FP64 solution, as the CUDA path does
with its 3xTF32 tensor-core blocks (tests/test_gpu_mixed.py): ratio <= 1e-10, solution within
1e-6 (relative 2-norm) of the FP64 Newton solve, in a few refinement steps."""
import numpy as np
import pytest

from exasim_b200 import cases
from oracle.hdg import HDGOracle
from oracle.models import MODELS


def rel2(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


@pytest.mark.parametrize("case", ["poisson2d", "convdiff3d"])
def test_fp32_refinement_reaches_fp64_solution(tmp_path, case):
    d = str(tmp_path / "datain")
    if case == "poisson2d":
        cases.poisson2d_tri(d, n=6)
    else:
        cases.convdiff3d_hex(d, n=2, porder=3, nsteps=1)
    def oracle():
        o = HDGOracle(d, MODELS[case]())
        if o.tdep:  # a stage with a source and a time-derivative term, as a DIRK stage sets them
            rng = np.random.default_rng(5)
            o.sdg = rng.standard_normal((o.npe, o.ncu, o.ne))
            o.sdgg = np.einsum("gj,jce->gec", o.shapegt[:, :, 0], o.sdg)
            o.time, o.dtfactor = 0.01, 100.0
        return o

    o64 = oracle()
    o64.newton()
    o32 = oracle()
    steps, norms = o32.newton_mixed(inner_tol=1e-4, rtol=1e-10)
    assert norms[-1] <= 1e-10 * norms[0], norms
    assert steps <= 6, (steps, norms)
    assert rel2(o32.uh, o64.uh) < 1e-6
    assert rel2(o32.udg, o64.udg) < 1e-6

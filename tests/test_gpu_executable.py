"""The solver as an executable (exasim_b200/bin/exasim_b200_<model>, csrc/exa_main.cpp): the
reference's datain/ folder in, its dataout files out.  On the reference's Poisson3D example
the written outuhat_np0.bin must carry the reference's header and match its golden trace
solution to the tolerance of the library-level golden test (1e-10 relative); for a DIRK run
the last udg snapshot must equal the library's own DIRK result bit for bit."""
import os
import subprocess

import numpy as np
import pytest

from exasim_b200 import HDGSolver, build as B, cases
from tests.cases import poisson3d_datain

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    B.build(["poisson3d", "convdiff3d"])


def run(model, datain, prefix):
    r = subprocess.run([B.exe_path(model), datain, prefix], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    return r


def test_executable_reproduces_reference_golden_uhat(tmp_path):
    d, gold = poisson3d_datain(tmp_path)
    out = str(tmp_path / "dataout")
    os.makedirs(out)
    run("poisson3d", d, out + "/out")
    uh = np.fromfile(out + "/outuhat_np0.bin")
    assert np.array_equal(uh[:3], gold[:3])          # (ncu, npf, nf)
    assert uh.size == gold.size
    assert np.linalg.norm(uh[3:] - gold[3:]) / np.linalg.norm(gold[3:]) < 1e-10
    udg = np.fromfile(out + "/outudg_np0.bin")
    npe, nc, ne = (int(v) for v in udg[:3])
    assert udg.size == 3 + npe * nc * ne


def test_executable_dirk_snapshots(tmp_path):
    d = cases.convdiff3d_hex(str(tmp_path / "cd"), n=2, porder=2, nsteps=2)
    out = str(tmp_path / "o")
    run("convdiff3d", d, out)
    udg = np.fromfile(out + "udg_np0.bin")
    npe, nc, ne = (int(v) for v in udg[:3])
    snaps = udg[3:].reshape(-1, npe * nc * ne)
    assert snaps.shape[0] == 2                      # saveSolFreq 1: one snapshot per step
    s = HDGSolver(d, "convdiff3d")
    s.DIRK(2)
    assert np.array_equal(snaps[-1], s.get("udg"))
    s.close()

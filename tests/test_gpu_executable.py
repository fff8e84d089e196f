"""The solver as an executable (exasim_b200/bin/exasim_b200_<model>, csrc/exa_main.cpp): the
reference's datain/ folder in, its dataout files out.  On the reference's Poisson3D example
the written outuhat_np0.bin must carry the reference's header and match its golden trace
solution to the tolerance of the library-level golden test (1e-10 relative); for a DIRK run
the last udg snapshot must equal the library's own DIRK result bit for bit; and a run restarted
from a step's checkpoint files (ReadSolutions, backend/Solution/solution.cpp:804-828, with the
restart argument of backend/Main/exasim.hpp:338-348, 387-393) must end in the same state, bit
for bit, as the uninterrupted run; with --vtu, each saved step's VTK file holds that step's
udg and the .pvd series their times."""
import shutil
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


def run(model, datain, prefix, *extra):
    r = subprocess.run([B.exe_path(model), datain, prefix, *extra], capture_output=True, text=True, timeout=900)
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


def test_executable_restart_matches_uninterrupted_run(tmp_path):
    # four DIRK steps in one run, checkpointing every saved step
    da = cases.convdiff3d_hex(str(tmp_path / "a"), n=2, porder=2, nsteps=4)
    oa = str(tmp_path / "oa")
    run("convdiff3d", da, oa, "--checkpoint")
    udg = np.fromfile(oa + "udg_np0.bin")
    npe, nc, ne = (int(v) for v in udg[:3])
    full = udg[3:].reshape(-1, npe * nc * ne)
    uha = np.fromfile(oa + "uhat_np0.bin")[3:].reshape(4, -1)
    for k in range(1, 5):
        c = np.fromfile(oa + f"udg_t{k}_np0.bin")
        assert np.array_equal(c, full[k - 1])       # saveSolOpt 1: all of udg, raw
        assert np.array_equal(np.fromfile(oa + f"_uhat_t{k}_np0.bin"), uha[k - 1])
    # the same problem restarted at step 2 for the remaining two steps
    db = cases.convdiff3d_hex(str(tmp_path / "b"), n=2, porder=2, nsteps=2)
    ob = str(tmp_path / "ob")
    shutil.copy(oa + "udg_t2_np0.bin", ob + "udg_t2_np0.bin")
    shutil.copy(oa + "_uhat_t2_np0.bin", ob + "_uhat_t2_np0.bin")
    r = run("convdiff3d", db, ob, "2", "0", "--checkpoint")
    assert "restart at step 2" in r.stdout
    rest = np.fromfile(ob + "udg_np0.bin")[3:].reshape(-1, npe * nc * ne)
    assert rest.shape[0] == 2
    assert np.array_equal(rest[-1], full[-1])
    assert np.array_equal(np.fromfile(ob + "uhat_np0.bin")[3:].reshape(2, -1)[-1], uha[-1])
    assert os.path.exists(ob + "udg_t4_np0.bin")     # numbered by step + restart
    # a missing checkpoint is an error, not a fresh start
    r = subprocess.run([B.exe_path("convdiff3d"), db, str(tmp_path / "none"), "3"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 1 and "cannot open" in r.stderr


def test_executable_writes_vtu_snapshots(tmp_path):
    from tests.test_cpu_vtu import read_vtu
    d = cases.convdiff3d_hex(str(tmp_path / "cd"), n=2, porder=2, nsteps=2, dt=0.01)
    out = str(tmp_path / "o")
    run("convdiff3d", d, out, "--vtu")
    udg = np.fromfile(out + "udg_np0.bin")
    npe, nc, ne = (int(v) for v in udg[:3])
    snaps = udg[3:].reshape(-1, npe * nc * ne)
    for k in (1, 2):
        npts, ncell, a = read_vtu(out + f"vis_{k}.vtu")
        assert npts == npe * ne and ncell == 8 * ne       # p^3 hexahedra per element
        u = snaps[k - 1].reshape(npe, nc, ne, order="F")
        for q in range(nc):
            assert np.array_equal(a[f"udg{q}"], u[:, q, :].ravel(order="F").astype(np.float32))
    pvd = open(out + "vis.pvd").read()
    times = [float(t) for t in __import__("re").findall(r'timestep="([^"]+)"', pvd)]
    assert times == pytest.approx([0.01, 0.02]) and "vis_1.vtu" in pvd and "vis_2.vtu" in pvd


def test_executable_ldg_matches_reference_outudg(tmp_path):
    """An LDG datain (problem[0] = 0): the reference's outudg after its DIRK step, and no
    uhat file (the reference writes the trace field for HDG alone)."""
    from tests import ref_fixtures as RF
    B.build(["euler3d"])
    fx = RF.load("euler3d_hex3_p2_ldg_bnd")
    d = RF.write_datain(fx, str(tmp_path / "datain"))
    out = str(tmp_path / "dataout")
    os.makedirs(out)
    run("euler3d", d, out + "/out")
    udg = np.fromfile(out + "/outudg_np0.bin")
    ref = fx["outudg"]
    assert np.array_equal(udg[:3], ref[:3])
    nud = int(np.prod(ref[:3]))
    a, b = udg[3:].reshape(-1, nud)[-1], ref[3:].reshape(-1, nud)[-1]
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-8
    assert not os.path.exists(out + "/outuhat_np0.bin")

"""CPU checks of the drop-in boundary: the C-ABI libraries load and export every
declared entry point, the host connectivity matches the oracle's restatement of the
reference's face numbering, and the model transformer handles every case model."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from exasim_b200 import build as B
from exasim_b200 import cases, inputs as I, modelc
from exasim_b200 import load_library
from oracle.hdg import HDGOracle
from oracle.models import MODELS
from tests.cases import poisson3d_datain

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def libs():
    return B.build()


def declared_functions():
    with open(os.path.join(ROOT, "include", "exasim_b200.h")) as f:
        txt = f.read()
    return sorted(set(re.findall(r"\b(exa_\w+)\s*\(", txt)))


def test_every_declared_symbol_is_exported(libs):
    names = declared_functions()
    assert len(names) >= 18
    for so in libs:
        out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True).stdout
        exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
        missing = [n for n in names if n not in exported]
        assert not missing, (so, missing)
        L = ctypes.CDLL(so)
        for n in names:
            assert hasattr(L, n)


def _conn_both(datain, model):
    o = HDGOracle(datain, MODELS[model]())
    L = load_library(model)
    t = np.ascontiguousarray(o.t.ravel(order="F"), dtype=np.int32)
    bf = np.ascontiguousarray(o.bf.ravel(order="F"), dtype=np.int32)
    perm = np.ascontiguousarray(o.perm.ravel(order="F"), dtype=np.int32)
    xpf = np.ascontiguousarray(o.xpf.ravel(order="F"), dtype=np.float64)
    f2e = np.zeros(4 * o.nfe * o.ne, dtype=np.int32)
    ec = np.zeros(o.npf * o.nfe * o.ne, dtype=np.int32)
    nf0 = ctypes.c_int()
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    nf = L.exa_connectivity_host(P(t), P(bf), P(perm), P(xpf), int(o.nd), int(o.elemtype), int(o.ne), int(o.npe),
                                 int(o.npf), P(f2e), P(ec), ctypes.byref(nf0))
    return o, nf, f2e[:4 * nf].reshape(4, nf, order="F"), ec.reshape(-1, o.ne, order="F"), nf0.value


@pytest.mark.parametrize("case", ["poisson2d", "convdiff3d"])
def test_host_connectivity_matches_oracle(libs, tmp_path, case):
    d = str(tmp_path / "datain")
    if case == "poisson2d":
        cases.poisson2d_tri(d, n=6)
    else:
        cases.convdiff3d_hex(d, n=3, porder=2, nsteps=1)
    o, nf, f2e, ec, nf0 = _conn_both(d, case)
    assert nf == o.nf and nf0 == o.nf0
    assert np.array_equal(f2e, o.f2e)
    assert np.array_equal(ec, o.elemcon)


def test_host_connectivity_on_reference_poisson3d_mesh(libs, tmp_path):
    d, _ = poisson3d_datain(tmp_path)
    o, nf, f2e, ec, nf0 = _conn_both(d, "poisson3d")
    assert (nf, nf0) == (50688, 47616)
    assert np.array_equal(f2e, o.f2e) and np.array_equal(ec, o.elemcon)


def test_modelc_generates_device_functions_for_all_models():
    for name in B.available_models():
        txt = modelc.generate(os.path.join(B.MODELS, name), name)
        for fn in ("HdgFlux_pt", "HdgSource_pt", "HdgFbou_pt", "HdgFbouonly_pt", "KokkosFlux_pt", "KokkosSource_pt",
                   "KokkosTdfunc_pt"):
            assert f"void {fn}(const size_t i," in txt, (name, fn)
        assert "Kokkos::" not in txt


def test_master_generator_matches_reference_tet_master():
    """Nodal shapes at the quadrature points agree with the preprocessor's (p=2 tetrahedron)."""
    z = np.load(os.path.join(ROOT, "tests", "golden", "poisson3d.npz"))
    import tempfile
    with tempfile.TemporaryDirectory() as t:
        fn = os.path.join(t, "master.bin")
        z["master"].tofile(fn)
        ref = I.read_master_bin(fn)
    m = I.make_master(3, 0, 2, 4)
    for k in ("shapegt", "shapegw", "xpe", "gpe", "gwe", "xpf", "gpf", "gwf", "shap1dgt", "shap1dgw"):
        a = np.asarray(getattr(m, k)).ravel(order="F")
        assert np.abs(a - ref[k]).max() < 1e-13, k
    # face shapes differ by ~5e-8: the preprocessor's simplex basis clamps y to 0.99999999 at the
    # face vertex (text2code/text2code/makemaster.cpp:451-455); the tables here do not
    assert np.abs(m.shapfgt.ravel(order="F") - ref["shapfgt"]).max() < 1e-6


def test_executable_reports_usage_and_missing_input(tmp_path):
    """The executable starts without a GPU far enough to check its arguments and inputs."""
    import subprocess
    from exasim_b200 import build as B
    exe = B.exe_path("poisson2d")
    assert os.path.exists(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "usage" in r.stderr
    r = subprocess.run([exe, str(tmp_path / "nowhere"), str(tmp_path / "out")], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 1 and "cannot open" in r.stderr
    # the restart argument must be a non-negative step number (exasim.hpp:341-347 refuses others)
    for bad in ("x", "-1", "2a"):
        r = subprocess.run([exe, str(tmp_path / "nowhere"), str(tmp_path / "out"), bad], capture_output=True,
                           text=True, timeout=60)
        assert r.returncode == 1 and "invalid restart value" in r.stderr, (bad, r.stderr)

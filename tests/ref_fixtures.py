"""Access to the reference-run fixtures (tests/golden/ref_<case>.npz, written by
tests/golden/make_ref_fixtures.py from the reference's own cput2cEXASIM).

Each fixture holds the case's four datain files byte for byte, arrays the reference wrote in
debug mode at its first Newton step (whole, or as per-block products with a seeded vector,
key proj_<name>), and the outputs of a normal run (outuhat, outudg, Newton norms, GMRES counts).
"""
from __future__ import annotations

import glob
import os
from typing import Dict, Optional, Tuple

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(os.path.basename(f)[4:-4] for f in glob.glob(os.path.join(GOLDEN, "ref_*.npz")))


def load(name: str) -> Dict[str, np.ndarray]:
    with np.load(os.path.join(GOLDEN, f"ref_{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def write_datain(fx: Dict[str, np.ndarray], path: str) -> str:
    os.makedirs(path, exist_ok=True)
    for k in ("app", "master", "mesh", "sol"):
        fx[k].tofile(os.path.join(path, k + ".bin"))
    return path


def projection_vector(cols: int, nblocks: int, seed: int) -> np.ndarray:
    """The seeded vector of tests/golden/make_ref_fixtures.py (one column per block)."""
    return np.random.default_rng(int(seed)).standard_normal((cols, nblocks))


def reference_view(fx, key: str, mine: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """(mine, reference) in comparable form: whole arrays, or per-block products with the
    fixture's seeded vector when the fixture stores only those."""
    mine = np.asarray(mine, dtype=np.float64).ravel(order="F")
    if key in fx:
        return mine, fx[key]
    r, c, nb = (int(v) for v in fx["shape_" + key])
    v = projection_vector(c, nb, fx["seed"])
    return np.einsum("ijk,jk->ik", mine.reshape(r, c, nb, order="F"), v), fx["proj_" + key]


def rel_err(fx, key: str, mine: np.ndarray) -> float:
    a, b = reference_view(fx, key, mine)
    a, b = np.ravel(a), np.ravel(b)
    assert a.shape == b.shape, (key, a.shape, b.shape)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def has(fx, key: str) -> bool:
    return key in fx or ("proj_" + key) in fx


def first_stage_state(datain: str) -> Optional[Tuple[float, float, np.ndarray]]:
    """For a time-dependent case: (time, dtfactor, sdg) of stage 1 of step 1, the state the
    reference assembles its first Newton step in (UpdateSource, updatesource.cpp:32-50:
    sdg = u d_11 / dt at time t0 + c_1 dt).  None for a steady case."""
    from exasim_b200 import inputs as I
    from oracle.hdg import dirk_coeff
    app = I.read_app_bin(os.path.join(datain, "app.bin"))
    dt = app["dt"]
    if dt.size == 0 or dt[0] <= 0:
        return None
    prob = app["problem"].astype(int)
    torder, nstage = prob[3], prob[4]
    c, d, tt = dirk_coeff(nstage, torder)
    t0 = app["factor"][0]
    sol = I.read_sol_bin(os.path.join(datain, "sol.bin"))
    nds = sol["ndims"].astype(int)
    ne, npe, nc, ncu = nds[0], nds[3], nds[5], nds[6]
    u = sol["udg"]
    if u.size == npe * nc * ne:
        u = u.reshape(npe, nc, ne, order="F")[:, :ncu]
    else:
        u = u.reshape(npe, ncu, ne, order="F")
    return t0 + dt[0] * tt[0], d[0] / dt[0], u * (d[0] / dt[0])

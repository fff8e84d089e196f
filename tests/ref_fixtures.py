"""Access to the reference-run fixtures (tests/golden/ref_<case>.npz, written by
tests/golden/make_ref_fixtures.py from the reference's own cput2cEXASIM).

Each fixture holds the case's four datain files byte for byte, arrays the reference wrote in
debug mode at its first Newton step (whole, or as per-block products with a seeded vector,
key proj_<name>), and the outputs of a normal run (outuhat, outudg, Newton norms, GMRES counts).
"""
from __future__ import annotations

import ctypes
import glob
import os
from typing import Dict, Optional, Tuple

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    """The HDG cases."""
    return sorted(n for n in _all() if "_ldg" not in n)


def ldg_names():
    """The LDG cases (pseudo-transient solver): PTC norms, outudg and one residual dump."""
    return sorted(n for n in _all() if "_ldg" in n)


def _all():
    return [os.path.basename(f)[4:-4] for f in glob.glob(os.path.join(GOLDEN, "ref_*.npz"))]


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


def reference_randvect(oracle, faces: bool = True) -> np.ndarray:
    """The start vector of the reference's polynomial preconditioner, made as it makes it
    (backend/Solver/setsysstruct.cpp:54-81, 84-203, 338-352): rand_normal draws (the polar
    Box-Muller method on C's rand(), from its default seed) on the element nodes [npe, ncu, ne],
    each component averaged over the element nodes that share a point (ArrayDG2CG), the values
    of each face's first element at its nodes (GetFaceNodes; with faces=False, the LDG form, the
    element-node field itself), normalised.  The libc of this
    process supplies rand(), reseeded with srand(1) first."""
    libc = ctypes.CDLL("libc.so.6")
    libc.rand.restype = ctypes.c_int
    libc.srand(1)
    rmax = 2147483647.0
    npe, ncu, ne = oracle.npe, oracle.ncu, oracle.ne
    n = npe * ncu * ne
    vals = np.empty(n)
    cached = None
    for i in range(n):
        if cached is not None:
            vals[i], cached = cached, None
            continue
        while True:
            x = 2.0 * libc.rand() / rmax - 1.0
            y = 2.0 * libc.rand() / rmax - 1.0
            r = x * x + y * y
            if r != 0.0 and r <= 1.0:
                break
        d = np.sqrt(-2.0 * np.log(r) / r)
        vals[i], cached = x * d, y * d
    u = vals.reshape(npe, ncu, ne, order="F")
    # points shared by element nodes: the nodes' coordinates, rounded
    xs = oracle.xdg.transpose(2, 0, 1).reshape(ne * npe, -1)   # row j + npe * e
    key = np.round(xs / max(np.abs(xs).max(), 1.0) * 1e9).astype(np.int64)
    _, cg = np.unique(key, axis=0, return_inverse=True)
    cg = cg.ravel()
    out = np.empty_like(u)
    for k in range(ncu):
        dg = u[:, k, :].ravel(order="F")                   # index j + npe * e
        sums = np.zeros(cg.max() + 1)
        cnt = np.zeros(cg.max() + 1)
        np.add.at(sums, cg, dg)
        np.add.at(cnt, cg, 1.0)
        out[:, k, :] = (sums / cnt)[cg].reshape(npe, ne, order="F")
    if not faces:
        # the LDG form keeps the element-node field itself (setsysstruct.cpp:338-341)
        v = out.ravel(order="F")
        return v / np.sqrt(np.dot(v, v))
    uh = oracle.get_face_nodes(out).ravel(order="F")
    return uh / np.sqrt(np.dot(uh, uh))

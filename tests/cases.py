"""Input cases for the tests: the reference's Poisson3D example and seeded synthetic
meshes with the shapes of the benchmark configurations (smaller sizes)."""
import os
import types

import numpy as np

from exasim_b200 import inputs as I

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def poisson3d_datain(tmpdir):
    """datain/ of examples/Poisson/poisson3d (byte-identical) plus sol.bin rebuilt from
    grid.bin with the preprocessor's compute_dgnodes.  Returns (dir, golden uhat)."""
    z = np.load(os.path.join(GOLDEN, "poisson3d.npz"))
    d = os.path.join(str(tmpdir), "datain")
    os.makedirs(d, exist_ok=True)
    for name in ("app", "master", "mesh"):
        z[name].tofile(os.path.join(d, name + ".bin"))
    gfn = os.path.join(str(tmpdir), "grid.bin")
    z["grid"].tofile(gfn)
    g = I.read_grid_bin(gfn)
    m = I.read_master_bin(os.path.join(d, "master.bin"))
    npe = int(m["ndims"][5])
    ms = types.SimpleNamespace(xpe=m["xpe"].reshape(npe, 3, order="F"), nd=3, elemtype=0, npe=npe)
    I.write_sol_bin(os.path.join(d, "sol.bin"), I.dgnodes(g, ms), nc=4, ncu=1)
    gold = np.frombuffer(z["outuhat"].tobytes(), dtype=np.float64)
    return d, gold

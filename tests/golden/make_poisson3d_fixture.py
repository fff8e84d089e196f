"""Pack the reference's own Poisson3D example into a test fixture.

examples/Poisson/poisson3d holds the only end-to-end golden output the reference
ships for its HDG path: datain/{app,master,mesh}.bin written by its preprocessor,
the vertex grid (grid.bin) and the solved trace field dataout/outuhat_np0.bin
(3D Poisson, p=2 tetrahedra, 24,576 elements, elemental additive Schwarz,
GMRES(50) to 1e-8).  sol.bin is not shipped; tests rebuild it from grid.bin and the
master's nodes exactly as the preprocessor's compute_dgnodes does.

The .bin files are stored byte for byte.  Usage:
    python tests/golden/make_poisson3d_fixture.py [/path/to/Exasim/examples/Poisson/poisson3d]
(default: $EXASIM_REF/examples/Poisson/poisson3d)
"""
import os
import sys

import numpy as np

src = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.environ["EXASIM_REF"], "examples/Poisson/poisson3d")
out = {}
for name in ("app", "master", "mesh"):
    out[name] = np.fromfile(os.path.join(src, "datain", name + ".bin"), dtype=np.uint8)
out["grid"] = np.fromfile(os.path.join(src, "grid.bin"), dtype=np.uint8)
out["outuhat"] = np.fromfile(os.path.join(src, "dataout", "outuhat_np0.bin"), dtype=np.uint8)
dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "poisson3d.npz")
np.savez_compressed(dst, **out)
print("wrote", dst, os.path.getsize(dst))

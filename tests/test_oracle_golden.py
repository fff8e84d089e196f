"""Pin the oracle to the reference's own golden output (examples/Poisson/poisson3d):
3D Poisson on 24,576 p=2 tetrahedra, elemental additive Schwarz, GMRES(50) to 1e-8,
one Newton step.  The reference reproduced this file to ~6e-12 relative; the oracle
must land within the same GMRES-limited band and on the same face numbering."""
import numpy as np

from oracle.hdg import HDGOracle
from oracle.models import Poisson
from tests.cases import poisson3d_datain


def test_oracle_reproduces_poisson3d_golden_uhat(tmp_path):
    d, gold = poisson3d_datain(tmp_path)
    ncu, npf, nf = (int(v) for v in gold[:3])
    o = HDGOracle(d, Poisson(3))
    assert (o.ncu, o.npf, o.nf) == (ncu, npf, nf)
    its, norms = o.newton()
    assert its == 1 and norms[-1] < 1e-6
    ref = gold[3:]
    mine = o.uh.ravel(order="F")
    rel = np.linalg.norm(mine - ref) / np.linalg.norm(ref)
    assert rel < 1e-10, rel
    assert np.abs(mine - ref).max() < 1e-10

"""bench.py's accounting on the CPU: the algorithmic bytes behind the q-elimination roofline,
the per-solve phase table and the workload description of the benchmark configuration."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def sizes(n=16, p=4):
    npe = (p + 1) ** 3
    npf = (p + 1) ** 2
    return {"n": npe, "m": 6 * npf, "npe": npe, "nd": 3, "ne": n ** 3, "npf": npf, "nfe": 6,
            "ndofuhat": npf * 3 * n * n * (n + 1)}


def test_packed_operand_size():
    # 125 rows in 8-row groups (16 groups), 375 k in chunks of 16 (24 chunks), 128 floats each
    assert bench.pack_floats(125, 375) == 16 * 24 * 128
    assert bench.pack_floats(8, 16) == 128


def test_qelim_bytes_of_the_benchmark_assembly():
    """Four 3xTF32 products per assembly at 16^3 hexahedra, p = 4 (n = 125, m = 150, K = 375):
    FP32 operands read once, FP64 Cin read, FP32 results written (F packed, K plain and packed)."""
    per_elem = bench.qelim_mixed_bytes(sizes()) / 16 ** 3
    d = 4 * (125 * 375 + 375 * 125) + 8 * 125 * 125 + 4 * 125 * 125
    f = 4 * (125 * 375 + 375 * 150) + 8 * 125 * 150 + 4 * 125 * 150
    k = 4 * (150 * 375 + 375 * 125) + 8 * 150 * 125 + 8 * 150 * 125
    h = 4 * (150 * 375 + 375 * 150) + 8 * 150 * 150 + 4 * 150 * 150
    assert per_elem == d + f + k + h == 2632500


def test_phase_table_per_solve():
    prof = {"qelim": (36.0, 40, 4.0e12), "matvec": (19.5, 420, 0.0), "getq": (0.0, 0, 0.0)}
    out = bench.phases_of(prof, 10)
    assert out["qelim"]["ms_per_solve"] == 3.6 and out["qelim"]["regions"] == 40
    assert abs(out["qelim"]["tflops"] - 4.0e12 / 36.0e-3 / 1e12) < 1e-9
    assert "tflops" not in out["matvec"]
    assert "getq" not in out  # phases that never ran are left out


def test_workload_description():
    c = bench.config(16)
    assert c["elements"] == 4096 and c["porder"] == 4
    assert c["ndofuhat"] == 326400
    assert "one DIRK-stage Newton solve" == c["step"]

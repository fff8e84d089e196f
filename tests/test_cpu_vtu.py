"""The executable's VTK writer (exasim_b200/csrc/exa_vtu.h), compiled here into a small driver
on the CPU: for each element type and order the file must parse as a VTK XML UnstructuredGrid
with raw appended UInt64-headed blocks, hold one point per DG node with the udg components as
Float32 point data, and cut every element into linear cells that tile it exactly (their
volumes add up to the element's: 1 for the unit square and cube, 1/2 and 1/6 for the
simplices)."""
import os
import re
import subprocess

import numpy as np
import pytest

from exasim_b200 import inputs as I

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = r'''
#include <cstdio>
#include <vector>
#include "exa_vtu.h"
int main(int argc, char** argv) {
  int nd, et, p, npe, ne, ncx, nc;
  std::FILE* f = std::fopen(argv[1], "rb");
  if (std::fread(&nd, 4, 1, f) != 1 || std::fread(&et, 4, 1, f) != 1 || std::fread(&p, 4, 1, f) != 1 ||
      std::fread(&npe, 4, 1, f) != 1 || std::fread(&ne, 4, 1, f) != 1 || std::fread(&ncx, 4, 1, f) != 1 ||
      std::fread(&nc, 4, 1, f) != 1) return 2;
  std::vector<double> xpe((size_t)npe * nd), xdg((size_t)npe * ncx * ne), udg((size_t)npe * nc * ne);
  if (std::fread(xpe.data(), 8, xpe.size(), f) != xpe.size() || std::fread(xdg.data(), 8, xdg.size(), f) != xdg.size() ||
      std::fread(udg.data(), 8, udg.size(), f) != udg.size()) return 2;
  std::fclose(f);
  return exa_vtu::write(argv[2], nd, et, p, npe, xpe.data(), ne, ncx, xdg.data(), nc, udg.data()) ? 0 : 1;
}
'''


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("vtu")
    src = d / "drv.cpp"
    src.write_text(DRIVER)
    exe = str(d / "drv")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "exasim_b200", "csrc"), str(src), "-o", exe],
                   check=True)
    return exe


def read_vtu(fn):
    raw = open(fn, "rb").read()
    head, data = raw.split(b"<AppendedData encoding=\"raw\">", 1)
    data = data[data.index(b"_") + 1:]
    head = head.decode()
    npts = int(re.search(r'NumberOfPoints="(\d+)"', head).group(1))
    ncell = int(re.search(r'NumberOfCells="(\d+)"', head).group(1))
    arrays = {}
    for m in re.finditer(r'<DataArray type="(\w+)" Name="(\w+)"[^>]*offset="(\d+)"', head):
        t, name, off = m.group(1), m.group(2), int(m.group(3))
        n = int(np.frombuffer(data[off:off + 8], dtype="<u8")[0])
        dt = {"Float32": "<f4", "Int32": "<i4", "UInt8": "u1"}[t]
        arrays[name] = np.frombuffer(data[off + 8:off + 8 + n], dtype=dt)
    assert raw.rstrip().endswith(b"</VTKFile>")
    return npts, ncell, arrays


def cell_volume(pts, conn, typ):
    P = pts[conn]
    if typ == 3:
        return np.linalg.norm(P[1] - P[0])
    if typ in (5, 9):     # triangle, or quadrilateral as two triangles
        tri = [(0, 1, 2)] if typ == 5 else [(0, 1, 2), (0, 2, 3)]
        return sum(0.5 * abs(np.cross(P[b] - P[a], P[c] - P[a])[2]) for a, b, c in tri)
    if typ == 10:
        return abs(np.linalg.det(np.stack([P[1] - P[0], P[2] - P[0], P[3] - P[0]]))) / 6.0
    # hexahedron as six tetrahedra around the diagonal 0-6
    tets = [(0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)]
    return sum(abs(np.linalg.det(np.stack([P[b] - P[a], P[c] - P[a], P[d] - P[a]]))) / 6.0 for a, b, c, d in tets)


@pytest.mark.parametrize("nd,et,p", [(1, 1, 3), (2, 1, 1), (2, 1, 3), (2, 0, 1), (2, 0, 3), (3, 1, 1), (3, 1, 2),
                                     (3, 0, 1), (3, 0, 2), (3, 0, 3), (3, 0, 4)])
def test_vtu_tiles_each_element(driver, tmp_path, nd, et, p):
    m = I.make_master(nd, et, p, 2 * p)
    xpe = np.asarray(m.xpe, dtype=np.float64).reshape(-1, nd, order="F")
    npe, ne, nc = xpe.shape[0], 2, 3
    # two copies of the master element, the second shifted by 2 in x
    xdg = np.zeros((npe, nd, ne))
    xdg[:, :, 0] = xpe
    xdg[:, :, 1] = xpe + np.eye(nd)[0] * 2.0
    udg = np.random.default_rng(nd * 10 + p).standard_normal((npe, nc, ne))
    blob = tmp_path / "in.bin"
    with open(blob, "wb") as f:
        np.array([nd, et, p, npe, ne, nd, nc], dtype=np.int32).tofile(f)
        xpe.ravel(order="F").tofile(f)
        xdg.ravel(order="F").tofile(f)
        udg.ravel(order="F").tofile(f)
    out = str(tmp_path / "o.vtu")
    subprocess.run([driver, str(blob), out], check=True)
    npts, ncell, a = read_vtu(out)
    assert npts == npe * ne and ncell == p ** nd * ne
    pts = a["points"].reshape(-1, 3).astype(np.float64)
    assert np.allclose(pts[:npe, :nd], xpe, atol=1e-7)
    for q in range(nc):
        assert np.array_equal(a[f"udg{q}"], udg[:, q, :].ravel(order="F").astype(np.float32))
    offs, types, conn = a["offsets"], a["types"], a["connectivity"]
    full = {1: 1.0, 2: 1.0 if et == 1 else 0.5, 3: 1.0 if et == 1 else 1.0 / 6.0}[nd]
    start = 0
    vols = np.zeros(ne)
    for i in range(ncell):
        cc = conn[start:offs[i]]
        start = offs[i]
        e = int(cc[0]) // npe
        assert np.all(cc // npe == e)                 # a cell stays inside its element
        v = cell_volume(pts, cc, int(types[i]))
        assert v > 1e-9 * full                         # no degenerate cell
        vols[e] += v
    assert np.allclose(vols, full, rtol=1e-5), vols

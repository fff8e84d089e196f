// Headless VTK output of a DG solution: one UnstructuredGrid (.vtu) per snapshot, in the XML
// format with raw appended data that the reference's writer uses (backend/Visualization/
// visualization.cpp:194-246, 437-470: Float32 point data and points, Int32 connectivity and
// offsets, UInt8 cell types, each block preceded by its UInt64 byte count), and a .pvd series
// for time-dependent runs (visualization.cpp:299-340).
//
// The points are the DG nodes of every element (npe per element, coordinates from sol.bin's
// xdg), so neighbouring elements keep their own copies; the reference first averages shared
// nodes onto a continuous mesh (VisDG2CG) and writes its model's derived fields, where this
// writer writes the nc components of udg ("udg0", "udg1", ...).  Each element is cut into the
// linear cells of its node lattice: p^d quadrilaterals or hexahedra for tensor elements, p^2
// triangles or p^3 tetrahedra (an octahedron split into four around one diagonal) for
// simplices, p segments in 1D; the lattice index of node a is round(p x_a) from the master
// element's nodes xpe in [0, 1]^d.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <map>
#include <string>
#include <vector>

namespace exa_vtu {

struct Cells {
  std::vector<int> conn;    // node indices within an element, cell after cell
  std::vector<int> size;    // nodes per cell
  std::vector<uint8_t> type;  // VTK cell types
};

// The linear sub-cells of the master element; empty when the nodes do not form the lattice.
inline Cells subcells(int nd, int elemtype, int p, int npe, const double* xpe) {
  Cells c;
  if (p < 1 || nd < 1 || nd > 3) return c;
  std::map<long long, int> at;  // lattice index (i, j, k) -> node
  for (int a = 0; a < npe; ++a) {
    long long key = 0;
    for (int d = nd - 1; d >= 0; --d) {
      const long long v = std::llround(xpe[a + (long long)npe * d] * p);
      if (v < 0 || v > p) return Cells{};
      key = key * (p + 1) + v;
    }
    at[key] = a;
  }
  auto v = [&](int i, int j, int k) -> int {
    const long long key = nd == 1 ? i : (nd == 2 ? (long long)j * (p + 1) + i : ((long long)k * (p + 1) + j) * (p + 1) + i);
    auto it = at.find(key);
    return it == at.end() ? -1 : it->second;
  };
  auto add = [&](std::initializer_list<int> n, uint8_t t) {
    for (int x : n)
      if (x < 0) return false;
    for (int x : n) c.conn.push_back(x);
    c.size.push_back((int)n.size());
    c.type.push_back(t);
    return true;
  };
  bool ok = true;
  if (nd == 1) {
    for (int i = 0; i < p && ok; ++i) ok = add({v(i, 0, 0), v(i + 1, 0, 0)}, 3);
  } else if (nd == 2 && elemtype == 1) {
    for (int j = 0; j < p && ok; ++j)
      for (int i = 0; i < p && ok; ++i) ok = add({v(i, j, 0), v(i + 1, j, 0), v(i + 1, j + 1, 0), v(i, j + 1, 0)}, 9);
  } else if (nd == 2) {
    for (int j = 0; j < p && ok; ++j)
      for (int i = 0; i + j < p && ok; ++i) {
        ok = add({v(i, j, 0), v(i + 1, j, 0), v(i, j + 1, 0)}, 5);
        if (ok && i + j < p - 1) ok = add({v(i + 1, j, 0), v(i + 1, j + 1, 0), v(i, j + 1, 0)}, 5);
      }
  } else if (elemtype == 1) {
    for (int k = 0; k < p && ok; ++k)
      for (int j = 0; j < p && ok; ++j)
        for (int i = 0; i < p && ok; ++i)
          ok = add({v(i, j, k), v(i + 1, j, k), v(i + 1, j + 1, k), v(i, j + 1, k), v(i, j, k + 1), v(i + 1, j, k + 1),
                    v(i + 1, j + 1, k + 1), v(i, j + 1, k + 1)},
                   12);
  } else {
    for (int k = 0; k < p && ok; ++k)
      for (int j = 0; j + k < p && ok; ++j)
        for (int i = 0; i + j + k < p && ok; ++i) {
          const int s = i + j + k;
          ok = add({v(i, j, k), v(i + 1, j, k), v(i, j + 1, k), v(i, j, k + 1)}, 10);
          if (ok && s <= p - 2) {
            // the octahedron between the corner tetrahedra, split around a = (i+1, j, k) - f = (i, j+1, k+1)
            const int a = v(i + 1, j, k), f = v(i, j + 1, k + 1);
            const int b = v(i, j + 1, k), c2 = v(i + 1, j + 1, k), d = v(i + 1, j, k + 1), e = v(i, j, k + 1);
            ok = add({a, f, b, c2}, 10) && add({a, f, c2, d}, 10) && add({a, f, d, e}, 10) && add({a, f, e, b}, 10);
          }
          if (ok && s <= p - 3)
            ok = add({v(i + 1, j + 1, k), v(i + 1, j, k + 1), v(i, j + 1, k + 1), v(i + 1, j + 1, k + 1)}, 10);
        }
  }
  if (!ok) return Cells{};
  return c;
}

inline void block(std::ofstream& f, const void* data, uint64_t bytes) {
  f.write(reinterpret_cast<const char*>(&bytes), sizeof(bytes));
  f.write(reinterpret_cast<const char*>(data), (std::streamsize)bytes);
}

// xdg [npe, ncx, ne] and udg [npe, nc, ne], column-major as Exasim stores them.  Returns false
// (and writes nothing) when the master nodes do not form a lattice or the file cannot be opened.
inline bool write(const std::string& fn, int nd, int elemtype, int p, int npe, const double* xpe, long long ne,
                  int ncx, const double* xdg, int nc, const double* udg) {
  const Cells c = subcells(nd, elemtype, p, npe, xpe);
  if (c.type.empty()) return false;
  std::ofstream f(fn, std::ios::binary);
  if (!f) return false;
  const long long np = (long long)npe * ne, ncell = (long long)c.type.size() * ne;
  const long long nconn = (long long)c.conn.size() * ne;
  // appended offsets: each block is 8 bytes of length plus its data
  std::vector<uint64_t> off;
  uint64_t o = 0;
  for (int q = 0; q < nc; ++q) {
    off.push_back(o);
    o += 8 + 4 * (uint64_t)np;
  }
  const uint64_t o_pts = o;
  o += 8 + 12 * (uint64_t)np;
  const uint64_t o_conn = o;
  o += 8 + 4 * (uint64_t)nconn;
  const uint64_t o_offs = o;
  o += 8 + 4 * (uint64_t)ncell;
  const uint64_t o_types = o;
  f << "<?xml version=\"1.0\"?>\n";
  f << "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
  f << "  <UnstructuredGrid>\n";
  f << "    <Piece NumberOfPoints=\"" << np << "\" NumberOfCells=\"" << ncell << "\">\n";
  f << "      <PointData>\n";
  for (int q = 0; q < nc; ++q)
    f << "        <DataArray type=\"Float32\" Name=\"udg" << q << "\" format=\"appended\" offset=\"" << off[q] << "\"/>\n";
  f << "      </PointData>\n";
  f << "      <Points>\n";
  f << "        <DataArray type=\"Float32\" Name=\"points\" NumberOfComponents=\"3\" format=\"appended\" offset=\"" << o_pts
    << "\"/>\n";
  f << "      </Points>\n";
  f << "      <Cells>\n";
  f << "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"appended\" offset=\"" << o_conn << "\"/>\n";
  f << "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"appended\" offset=\"" << o_offs << "\"/>\n";
  f << "        <DataArray type=\"UInt8\" Name=\"types\" format=\"appended\" offset=\"" << o_types << "\"/>\n";
  f << "      </Cells>\n";
  f << "    </Piece>\n";
  f << "  </UnstructuredGrid>\n";
  f << "  <AppendedData encoding=\"raw\">\n   _";
  std::vector<float> buf((size_t)np);
  for (int q = 0; q < nc; ++q) {
    for (long long e = 0; e < ne; ++e)
      for (int a = 0; a < npe; ++a) buf[(size_t)(a + (long long)npe * e)] = (float)udg[a + (long long)npe * (q + (long long)nc * e)];
    block(f, buf.data(), 4 * (uint64_t)np);
  }
  std::vector<float> pts((size_t)(3 * np), 0.0f);
  for (long long e = 0; e < ne; ++e)
    for (int a = 0; a < npe; ++a)
      for (int d = 0; d < ncx && d < 3; ++d)
        pts[(size_t)(3 * (a + (long long)npe * e) + d)] = (float)xdg[a + (long long)npe * (d + (long long)ncx * e)];
  block(f, pts.data(), 12 * (uint64_t)np);
  std::vector<int32_t> conn((size_t)nconn), offs((size_t)ncell);
  std::vector<uint8_t> types((size_t)ncell);
  long long w = 0, cw = 0, run = 0;
  for (long long e = 0; e < ne; ++e) {
    for (size_t t = 0; t < c.conn.size(); ++t) conn[(size_t)w++] = (int32_t)(c.conn[t] + (long long)npe * e);
    for (size_t t = 0; t < c.size.size(); ++t) {
      run += c.size[t];
      offs[(size_t)cw] = (int32_t)run;
      types[(size_t)cw] = c.type[t];
      ++cw;
    }
  }
  block(f, conn.data(), 4 * (uint64_t)nconn);
  block(f, offs.data(), 4 * (uint64_t)ncell);
  block(f, types.data(), (uint64_t)ncell);
  f << "\n  </AppendedData>\n</VTKFile>\n";
  return (bool)f;
}

// The .pvd series of a time-dependent run: file i at time t[i]
inline bool write_pvd(const std::string& fn, const std::vector<std::string>& files, const std::vector<double>& t) {
  std::ofstream f(fn);
  if (!f) return false;
  f << "<?xml version=\"1.0\"?>\n<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
  f << "  <Collection>\n";
  for (size_t i = 0; i < files.size(); ++i) {
    char tb[64];
    std::snprintf(tb, sizeof(tb), "%.17g", t[i]);
    f << "    <DataSet timestep=\"" << tb << "\" group=\"\" part=\"0\" file=\"" << files[i] << "\"/>\n";
  }
  f << "  </Collection>\n</VTKFile>\n";
  return (bool)f;
}

}  // namespace exa_vtu

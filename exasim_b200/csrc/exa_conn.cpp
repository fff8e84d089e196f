// Face connectivity of a single-rank HDG mesh, built on the host when mesh.bin
// carries raw element-to-vertex lists (Exasim's readmeshstruct -> buildConn,
// backend/Discretization/connectivity.cpp:1212-1385).
//
// The face numbering fixes the layout of every trace vector (uhat, GMRES basis), so
// it reproduces the reference's order:
//  * element faces are visited element by element; a face key (sorted vertex ids)
//    seen for the second time closes an interior face; the first-seen keys left over
//    are the boundary faces, in the iteration order of a std::unordered_map keyed with
//    the 64-bit mixing hash of connectivity.cpp:163-180 and reserved for 1.3*ne*nfe
//    entries (connectivity.cpp:182-231);
//  * interior faces first, then boundary faces stably sorted by boundary code
//    (connectivity.cpp:426-497);
//  * the second element's face nodes are matched through the vertex rotation that maps
//    its face onto the first element's (connectivity.cpp:337-424, 1128-1205).
// The hash-table iteration order is that of this toolchain's libstdc++.
#include "exa_conn.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <utility>
#include <vector>

namespace {

struct FaceId {
  std::array<int, 8> v{};
  uint8_t len{};
  bool operator==(const FaceId& o) const noexcept {
    if (len != o.len) return false;
    for (uint8_t i = 0; i < len; ++i)
      if (v[i] != o.v[i]) return false;
    return true;
  }
};

struct FaceIdHash {
  size_t operator()(const FaceId& k) const noexcept {
    uint64_t h = 0x9E3779B97F4A7C15ull ^ k.len;
    for (uint8_t i = 0; i < k.len; ++i) {
      uint64_t x = static_cast<uint64_t>(k.v[i]) + 0x9E3779B97F4A7C15ull;
      x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
      x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
      x ^= (x >> 31);
      h ^= x + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    }
    return static_cast<size_t>(h);
  }
};

// local vertex lists of the faces of the reference element (connectivity.cpp:1010-1105)
std::vector<int> face_vertices(int dim, int elemtype) {
  std::vector<int> f;
  if (dim == 1) f = {1, 2};
  else if (dim == 2 && elemtype == 0) f = {2, 3, 3, 1, 1, 2};
  else if (dim == 2) f = {1, 2, 2, 3, 3, 4, 4, 1};
  else if (elemtype == 0) f = {2, 3, 4, 1, 4, 3, 1, 2, 4, 1, 3, 2};
  else f = {1, 4, 3, 2, 5, 6, 7, 8, 1, 2, 6, 5, 3, 4, 8, 7, 2, 3, 7, 6, 4, 1, 5, 8};
  for (int& x : f) --x;
  return f;
}

// face-node permutations for each admissible vertex rotation of a neighbour's face
std::vector<int> rotation_perms(const double* xpf, int npf, int dim, int elemtype, int& nrot) {
  std::vector<int> out;
  if (dim == 1) { nrot = 1; return {0}; }
  if (dim == 2) {
    nrot = 1;
    for (int i = 0; i < npf; ++i) out.push_back(npf - 1 - i);
    return out;
  }
  nrot = (elemtype == 0) ? 3 : 4;
  out.assign(npf * nrot, -1);
  for (int r = 0; r < nrot; ++r) {
    for (int i = 0; i < npf; ++i) {
      const double x = xpf[i], y = xpf[i + npf];
      for (int j = 0; j < npf; ++j) {
        const double xj = xpf[j], yj = xpf[j + npf];
        double u, v;
        if (elemtype == 0) {
          if (r == 0) { u = yj; v = xj; }
          else if (r == 1) { u = 1.0 - xj - yj; v = yj; }
          else { u = xj; v = 1.0 - xj - yj; }
        } else {
          if (r == 0) { u = yj; v = xj; }
          else if (r == 1) { u = xj; v = 1.0 - yj; }
          else if (r == 2) { u = 1.0 - yj; v = 1.0 - xj; }
          else { u = 1.0 - xj; v = yj; }
        }
        if (std::fabs(x - u) <= 1e-8 && std::fabs(y - v) <= 1e-8) {
          out[i + npf * r] = j;
          break;
        }
      }
    }
  }
  return out;
}

int match_rotation(const int* a, const int* b, int elemtype) {
  if (elemtype == 0) {
    if (a[0] == b[0] && a[1] == b[2] && a[2] == b[1]) return 0;
    if (a[0] == b[1] && a[1] == b[0] && a[2] == b[2]) return 1;
    if (a[0] == b[2] && a[1] == b[1] && a[2] == b[0]) return 2;
  } else {
    if (a[0] == b[0] && a[1] == b[3] && a[2] == b[2] && a[3] == b[1]) return 0;
    if (a[0] == b[3] && a[1] == b[2] && a[2] == b[1] && a[3] == b[0]) return 1;
    if (a[0] == b[2] && a[1] == b[1] && a[2] == b[0] && a[3] == b[3]) return 2;
    if (a[0] == b[1] && a[1] == b[0] && a[2] == b[3] && a[3] == b[2]) return 3;
  }
  return -1;
}

}  // namespace

int exa_build_connectivity(const int* t, const int* bf, const int* perm, const double* xpf, int dim,
                           int elemtype, int ne, int npe, int npf, ExaConn& out) {
  const int nve = (elemtype == 0) ? dim + 1 : (1 << dim);
  const int nvf = (dim == 3) ? dim + elemtype : dim;
  const int nfe = dim + (dim - 1) * elemtype + 1;
  const std::vector<int> lf = face_vertices(dim, elemtype);

  std::vector<std::array<int, 4>> faces;
  faces.reserve(static_cast<size_t>(ne) * nfe);
  {
    std::unordered_map<FaceId, std::pair<int, int>, FaceIdHash> open;
    open.reserve(static_cast<size_t>(ne) * nfe * 1.3);
    for (int e = 0; e < ne; ++e) {
      for (int l = 0; l < nfe; ++l) {
        FaceId key;
        key.len = static_cast<uint8_t>(nvf);
        for (int i = 0; i < nvf; ++i) key.v[i] = t[e * nve + lf[l * nvf + i]];
        std::sort(key.v.begin(), key.v.begin() + nvf);
        auto it = open.find(key);
        if (it == open.end()) {
          open.emplace(key, std::make_pair(e, l));
        } else {
          faces.push_back({it->second.first, it->second.second, e, l});
          open.erase(it);
        }
      }
    }
    std::vector<std::array<int, 4>> bnd;
    for (const auto& kv : open) bnd.push_back({kv.second.first, kv.second.second, -1, -1});
    std::stable_sort(bnd.begin(), bnd.end(), [&](const std::array<int, 4>& a, const std::array<int, 4>& b) {
      return bf[a[1] + nfe * a[0]] < bf[b[1] + nfe * b[0]];
    });
    out.nf0 = static_cast<int>(faces.size());
    faces.insert(faces.end(), bnd.begin(), bnd.end());
  }
  const int nf = static_cast<int>(faces.size());
  out.nf = nf;
  out.nfe = nfe;
  out.f2e.assign(4 * nf, 0);
  for (int i = 0; i < nf; ++i)
    for (int r = 0; r < 4; ++r) out.f2e[4 * i + r] = faces[i][r];

  int nrot = 1;
  const std::vector<int> rot = rotation_perms(xpf, npf, dim, elemtype, nrot);
  out.elemcon.assign(static_cast<size_t>(npf) * nfe * ne, -1);
  for (int i = 0; i < nf; ++i) {
    const int e1 = faces[i][0], l1 = faces[i][1], e2 = faces[i][2], l2 = faces[i][3];
    for (int j = 0; j < npf; ++j) out.elemcon[j + npf * (l1 + nfe * e1)] = i * npf + j;
    if (e2 < 0) continue;
    int r = 0;
    if (dim == 3) {
      int a[4], b[4];
      for (int v = 0; v < nvf; ++v) {
        a[v] = t[lf[l1 * nvf + v] + nve * e1];
        b[v] = t[lf[l2 * nvf + v] + nve * e2];
      }
      r = match_rotation(a, b, elemtype);
      if (r < 0) return -1;
    }
    for (int j = 0; j < npf; ++j) {
      const int pj = rot[j + npf * r];
      if (pj < 0) return -1;
      out.elemcon[j + npf * (l2 + nfe * e2)] = i * npf + pj;
    }
  }
  (void)perm;
  (void)npe;
  for (int v : out.elemcon)
    if (v < 0) return -1;
  return nf;
}

// Oracle (test infrastructure only): CPU restatement of Exasim's face connectivity
// builder, used to check the HDG solver in exasim_b200/ and never linked into it.
//
// Exasim's backend builds the face numbering itself when mesh.bin carries raw
// element-to-vertex lists (backend/Discretization/connectivity.cpp:1212-1385,
// buildConn -> connectivity() :426-497).  The face order decides the layout of every
// trace vector (uhat, the GMRES vectors), so parity needs the same order:
//   1. faces are keyed by their sorted vertex ids in a std::unordered_map with the
//      64-bit mixing hash of connectivity.cpp:163-180; an element face whose key is
//      already present closes an interior face (f2e = first owner, second owner);
//      faces left in the map are boundary faces, visited in the map's iteration order
//      (connectivity.cpp:182-231, mkf2e_hash);
//   2. interior faces come first in discovery order, then boundary faces stably sorted
//      by their boundary code (connectivity.cpp:453-484);
//   3. facecon/elemcon are filled with the neighbour's face-node permutation found by
//      matching vertex rotations (connectivity.cpp:337-424, permindex :1128-1205).
// The iteration order of std::unordered_map is libstdc++'s; this file is compiled with
// the same toolchain as the solver so both see the same order.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <unordered_map>
#include <utility>
#include <vector>

namespace {

struct Key {
  std::array<int, 8> a{};
  uint8_t len{};
  bool operator==(const Key& o) const noexcept {
    if (len != o.len) return false;
    for (uint8_t i = 0; i < len; ++i)
      if (a[i] != o.a[i]) return false;
    return true;
  }
};

struct KeyHash {
  size_t operator()(const Key& k) const noexcept {
    uint64_t h = 0x9E3779B97F4A7C15ull ^ k.len;
    for (uint8_t i = 0; i < k.len; ++i) {
      uint64_t x = static_cast<uint64_t>(k.a[i]) + 0x9E3779B97F4A7C15ull;
      x ^= (x >> 30);
      x *= 0xBF58476D1CE4E5B9ull;
      x ^= (x >> 27);
      x *= 0x94D049BB133111EBull;
      x ^= (x >> 31);
      h ^= x + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    }
    return static_cast<size_t>(h);
  }
};

void local_faces(std::vector<int>& f, int dim, int elemtype) {
  static const int tri[] = {2, 3, 3, 1, 1, 2};
  static const int quad[] = {1, 2, 2, 3, 3, 4, 4, 1};
  static const int tet[] = {2, 3, 4, 1, 4, 3, 1, 2, 4, 1, 3, 2};
  static const int hex[] = {1, 4, 3, 2, 5, 6, 7, 8, 1, 2, 6, 5, 3, 4, 8, 7, 2, 3, 7, 6, 4, 1, 5, 8};
  static const int line[] = {1, 2};
  const int* src = line;
  int n = 2;
  if (dim == 2 && elemtype == 0) { src = tri; n = 6; }
  else if (dim == 2) { src = quad; n = 8; }
  else if (dim == 3 && elemtype == 0) { src = tet; n = 12; }
  else if (dim == 3) { src = hex; n = 24; }
  f.assign(src, src + n);
  for (auto& v : f) v -= 1;
}

// index of the point of B matching each point of A (both [n, 2] column-major), -1 if none
void match_points(int* out, const double* A, const double* B, int n) {
  for (int i = 0; i < n; ++i) {
    out[i] = -1;
    for (int j = 0; j < n; ++j) {
      if (std::fabs(A[i] - B[j]) <= 1e-8 && std::fabs(A[i + n] - B[j + n]) <= 1e-8) {
        out[i] = j;
        break;
      }
    }
  }
}

// permutations of the face nodes under the vertex rotations a neighbour may see
void face_perms(std::vector<int>& pi, const double* xpf, int npf, int dim, int elemtype) {
  if (dim == 1) { pi.assign(1, 0); return; }
  if (dim == 2) {
    pi.resize(npf);
    for (int i = 0; i < npf; ++i) pi[i] = npf - 1 - i;
    return;
  }
  int ncol = (elemtype == 0) ? 3 : 4;
  pi.assign(npf * ncol, -1);
  std::vector<double> q(2 * npf);
  for (int c = 0; c < ncol; ++c) {
    for (int i = 0; i < npf; ++i) {
      double x = xpf[i], y = xpf[i + npf];
      double u, v;
      if (elemtype == 0) {
        if (c == 0) { u = y; v = x; }
        else if (c == 1) { u = 1.0 - x - y; v = y; }
        else { u = x; v = 1.0 - x - y; }
      } else {
        if (c == 0) { u = y; v = x; }
        else if (c == 1) { u = x; v = 1.0 - y; }
        else if (c == 2) { u = 1.0 - y; v = 1.0 - x; }
        else { u = 1.0 - x; v = y; }
      }
      q[i] = u;
      q[i + npf] = v;
    }
    match_points(&pi[c * npf], xpf, q.data(), npf);
  }
}

}  // namespace

extern "C" {

// Builds f2e [4, nf], elemcon [npf*nfe, ne], facecon [2, npf, nf] (all 0-based) for a
// single-rank mesh.  t: [nve, ne] 0-based vertex ids; bf: [nfe, ne] boundary codes
// (0 interior); perm: [npf, nfe]; xpf: [npf, dim-1].  Output buffers must hold the
// worst case (nf <= nfe*ne).  Returns nf and writes the interior face count to *nf0.
int oracle_build_conn(const int* t, const int* bf, const int* perm, const double* xpf,
                      int dim, int elemtype, int ne, int npe, int npf,
                      int* f2e, int* elemcon, int* facecon, int* nf0) {
  const int nve = (elemtype == 0) ? dim + 1 : (1 << dim);
  const int nvf = (dim == 3) ? dim + elemtype : dim;
  const int nfe = dim + (dim - 1) * elemtype + 1;
  std::vector<int> lf;
  local_faces(lf, dim, elemtype);

  // 1. face discovery
  std::vector<int> f2t(4 * nfe * ne);
  int nf = 0;
  {
    std::unordered_map<Key, std::pair<int, int>, KeyHash> map;
    map.reserve(static_cast<size_t>(ne) * nfe * 1.3);
    for (int e = 0; e < ne; ++e) {
      for (int l = 0; l < nfe; ++l) {
        Key k;
        k.len = static_cast<uint8_t>(nvf);
        for (int i = 0; i < nvf; ++i) k.a[i] = t[e * nve + lf[l * nvf + i]];
        std::sort(k.a.begin(), k.a.begin() + nvf);
        auto it = map.find(k);
        if (it == map.end()) {
          map.emplace(k, std::make_pair(e, l));
        } else {
          f2t[4 * nf + 0] = it->second.first;
          f2t[4 * nf + 1] = it->second.second;
          f2t[4 * nf + 2] = e;
          f2t[4 * nf + 3] = l;
          map.erase(it);
          ++nf;
        }
      }
    }
    for (const auto& kv : map) {
      f2t[4 * nf + 0] = kv.second.first;
      f2t[4 * nf + 1] = kv.second.second;
      f2t[4 * nf + 2] = -1;
      f2t[4 * nf + 3] = -1;
      ++nf;
    }
  }

  // 2. interior faces first, then boundary faces stably sorted by code
  std::vector<int> inner, bnd;
  for (int i = 0; i < nf; ++i) (f2t[4 * i + 2] >= 0 ? inner : bnd).push_back(i);
  std::stable_sort(bnd.begin(), bnd.end(), [&](int a, int b) {
    return bf[f2t[4 * a + 1] + nfe * f2t[4 * a]] < bf[f2t[4 * b + 1] + nfe * f2t[4 * b]];
  });
  std::vector<int> order(inner);
  order.insert(order.end(), bnd.begin(), bnd.end());
  for (int i = 0; i < nf; ++i)
    for (int r = 0; r < 4; ++r) f2e[4 * i + r] = f2t[4 * order[i] + r];
  *nf0 = static_cast<int>(inner.size());

  // 3. node connectivity of each face
  std::vector<int> pi;
  face_perms(pi, xpf, npf, dim, elemtype);
  for (int i = 0; i < npf * nfe * ne; ++i) elemcon[i] = -1;
  for (int i = 0; i < 2 * npf * nf; ++i) facecon[i] = -1;
  for (int i = 0; i < nf; ++i) {
    int e1 = f2e[4 * i], l1 = f2e[4 * i + 1], e2 = f2e[4 * i + 2], l2 = f2e[4 * i + 3];
    for (int j = 0; j < npf; ++j) {
      facecon[2 * j + 2 * npf * i] = e1 * npe + perm[j + npf * l1];
      elemcon[j + npf * (l1 + nfe * e1)] = i * npf + j;
    }
    if (e2 < 0) {
      for (int j = 0; j < npf; ++j) facecon[1 + 2 * j + 2 * npf * i] = facecon[2 * j + 2 * npf * i];
      continue;
    }
    int k = 0;
    if (dim == 3) {
      int a[4], b[4];
      for (int v = 0; v < nvf; ++v) {
        a[v] = t[lf[l1 * nvf + v] + nve * e1];
        b[v] = t[lf[l2 * nvf + v] + nve * e2];
      }
      k = -1;
      if (elemtype == 0) {
        if (a[0] == b[0] && a[1] == b[2] && a[2] == b[1]) k = 0;
        else if (a[0] == b[1] && a[1] == b[0] && a[2] == b[2]) k = 1;
        else if (a[0] == b[2] && a[1] == b[1] && a[2] == b[0]) k = 2;
      } else {
        if (a[0] == b[0] && a[1] == b[3] && a[2] == b[2] && a[3] == b[1]) k = 0;
        else if (a[0] == b[3] && a[1] == b[2] && a[2] == b[1] && a[3] == b[0]) k = 1;
        else if (a[0] == b[2] && a[1] == b[1] && a[2] == b[0] && a[3] == b[3]) k = 2;
        else if (a[0] == b[1] && a[1] == b[0] && a[2] == b[3] && a[3] == b[2]) k = 3;
      }
      if (k < 0) return -1;
    }
    for (int j = 0; j < npf; ++j) {
      int pj = pi[j + npf * k];
      facecon[1 + 2 * j + 2 * npf * i] = e2 * npe + perm[pj + npf * l2];
      elemcon[j + npf * (l2 + nfe * e2)] = i * npf + pj;
    }
  }
  return nf;
}

}  // extern "C"

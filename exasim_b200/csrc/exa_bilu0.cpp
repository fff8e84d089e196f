// Host set-up of the block ILU(0) preconditioner (Exasim preconditioner = 2).
//
// The steps follow the reference's preprocessing so that the sub-domain matrices, and so
// the preconditioner, are the reference's:
//   partition        backend/Common/cpuimpl.h:1332-1496 (gridpartition2d / 3d)
//   face ordering    cpuimpl.h:1266-1330 (crs_faceordering): the faces of the first
//                    sub-domain's elements in first-seen order, remapped to local element
//                    numbers (a face whose first element lies outside takes the second's
//                    place, and the outside element becomes -1); the sub-domain's boundary
//                    faces first, ordered by how often their element recurs (then by element,
//                    then by position), then the interior faces peeled repeatedly by their
//                    number of not-yet-ordered neighbours (stable); CRS rows with the
//                    diagonal first and the neighbours sorted; the face map of every
//                    sub-domain through its corresponding element
//   ILU(0) schedule  cpuimpl.h:1498-1625 (crs_indexingilu0) and matvec.cpp:119-166
#include "exa_bilu0.h"

#include <algorithm>
#include <cstdio>
#include <map>
#include <numeric>

namespace {

using Vec = std::vector<int>;

// element -> faces (nfe x ne, -1 where absent)
Vec elem_faces(const Vec& f2e, int nf, int nfe, int ne) {
  Vec e2f((size_t)nfe * ne, -1);
  for (int i = 0; i < nf; ++i) {
    e2f[f2e[4 * i + 1] + nfe * f2e[4 * i]] = i;
    if (f2e[4 * i + 2] >= 0) e2f[f2e[4 * i + 3] + nfe * f2e[4 * i + 2]] = i;
  }
  return e2f;
}

// neighbour faces (2 (nfe - 1) x nf, -1 where absent): the other faces of e1, then of e2
Vec face_neighbours(const Vec& f2e, const Vec& e2f, int nf, int nfe) {
  const int nbf = 2 * (nfe - 1);
  Vec f2f((size_t)nbf * nf, -1);
  for (int i = 0; i < nf; ++i) {
    int k = 0;
    for (int s = 0; s < 2; ++s) {
      const int e = f2e[4 * i + 2 * s], l0 = f2e[4 * i + 2 * s + 1];
      if (e < 0) continue;
      for (int l = 0; l < nfe; ++l)
        if (l != l0) f2f[k++ + (size_t)nbf * i] = e2f[l + nfe * e];
    }
  }
  return f2f;
}

Vec stable_order(const Vec& key) {
  Vec idx(key.size());
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return key[a] < key[b]; });
  return idx;
}

void permute_columns(Vec& f2e, const Vec& cols, int first) {
  Vec tmp(4 * cols.size());
  for (size_t i = 0; i < cols.size(); ++i)
    for (int r = 0; r < 4; ++r) tmp[4 * i + r] = f2e[4 * cols[i] + r];
  for (size_t i = 0; i < cols.size(); ++i)
    for (int r = 0; r < 4; ++r) f2e[4 * (first + i) + r] = tmp[4 * i + r];
}

// boundary faces of the sub-domain first (by recurrence of their element), then interior faces
void reorder_faces(Vec& f2e, int nf) {
  Vec b;
  for (int i = 0; i < nf; ++i)
    if (f2e[4 * i + 3] == -1) b.push_back(i);
  Vec el(b.size());
  for (size_t i = 0; i < b.size(); ++i) el[i] = f2e[4 * b[i]];
  Vec rec(b.size(), 0);
  int maxrec = 0;
  for (size_t i = 0; i < b.size(); ++i) {
    for (size_t j = 0; j < b.size(); ++j) rec[i] += el[i] == el[j];
    maxrec = std::max(maxrec, rec[i]);
  }
  Vec order;
  for (int k = 1; k <= maxrec; ++k) {
    Vec sel, key;
    for (size_t i = 0; i < b.size(); ++i)
      if (rec[i] == k) sel.push_back((int)i), key.push_back(el[i]);
    for (int s : stable_order(key)) order.push_back(b[sel[s]]);
  }
  Vec isb(nf, 0);
  for (int v : b) isb[v] = 1;
  for (int i = 0; i < nf; ++i)
    if (!isb[i]) order.push_back(i);
  permute_columns(f2e, order, 0);

  int ne = 0, nfe = 0;
  for (int i = 0; i < nf; ++i) {
    ne = std::max(ne, std::max(f2e[4 * i], f2e[4 * i + 2]) + 1);
    nfe = std::max(nfe, std::max(f2e[4 * i + 1], f2e[4 * i + 3]) + 1);
  }
  const int nbf = 2 * (nfe - 1);
  int done = (int)b.size();
  while (done < nf) {
    const Vec f2f = face_neighbours(f2e, elem_faces(f2e, nf, nfe, ne), nf, nfe);
    Vec cnt(nf - done, 0), rest(nf - done);
    for (int i = done; i < nf; ++i) {
      rest[i - done] = i;
      for (int j = 0; j < nbf; ++j) cnt[i - done] += f2f[j + (size_t)nbf * i] >= done;
    }
    const Vec a = stable_order(cnt);
    Vec cols(a.size());
    int inc = 0;
    for (size_t i = 0; i < a.size(); ++i) {
      cols[i] = rest[a[i]];
      inc += cnt[a[i]] < nbf;
    }
    permute_columns(f2e, cols, done);
    if (inc == 0) break;  // no face can be ordered further (not a Cartesian sub-domain)
    done += inc;
  }
}

}  // namespace

int exa_bilu_setup(const int* cgp, int ncgp, const int* f2e_in, int nf, int nfe, int ne, ExaBilu& b, char* err,
                   int errlen) {
  // ---- partition
  const int dim = ncgp > 0 ? cgp[0] : 0;
  if (!((dim == 2 && ncgp >= 6) || (dim == 3 && ncgp >= 8))) {
    snprintf(err, errlen, "cartgridpart must be [2, Nx, Ny, Mx, My, opt] or [3, Nx, Ny, Nz, Mx, My, Mz, opt]");
    return -1;
  }
  int N[3] = {1, 1, 1}, M[3] = {1, 1, 1};
  for (int k = 0; k < dim; ++k) N[k] = cgp[1 + k], M[k] = cgp[1 + dim + k];
  const int opt = cgp[1 + 2 * dim];
  long long cells = 1;
  for (int k = 0; k < dim; ++k) {
    if (M[k] <= 0 || N[k] % M[k] != 0) {
      snprintf(err, errlen, "cartgridpart: grid size %d is not a multiple of block size %d", N[k], M[k]);
      return -1;
    }
    cells *= N[k];
  }
  if (cells != ne) {
    snprintf(err, errlen, "cartgridpart describes %lld elements, the mesh has %d", cells, ne);
    return -1;
  }
  int nb[3] = {N[0] / M[0], N[1] / M[1], N[2] / M[2]};
  b.nse = nb[0] * nb[1] * nb[2];
  b.nese = M[0] * M[1] * M[2];
  auto cell_id = [&](const int* g) {
    long long r = 0, s = 1;
    if (opt == 0)
      for (int k = 0; k < dim; ++k) r += g[k] * s, s *= N[k];
    else
      for (int k = dim - 1; k >= 0; --k) r += g[k] * s, s *= N[k];
    return (int)r;
  };
  b.elem.assign((size_t)b.nse * b.nese, 0);
  int r = 0;
  auto emit = [&](int bx, int by, int bz) {  // block r: its cells, x fastest
    int c = 0;
    for (int z = 0; z < M[2]; ++z)
      for (int y = 0; y < M[1]; ++y)
        for (int x = 0; x < M[0]; ++x, ++c) {
          const int g[3] = {bx * M[0] + x, by * M[1] + y, bz * M[2] + z};
          b.elem[r + (size_t)b.nse * c] = cell_id(g);
        }
    ++r;
  };
  // blocks x fastest (opt 0) or the last coordinate fastest (opt 1)
  if (opt == 0) {
    for (int bz = 0; bz < nb[2]; ++bz)
      for (int by = 0; by < nb[1]; ++by)
        for (int bx = 0; bx < nb[0]; ++bx) emit(bx, by, bz);
  } else {
    for (int bx = 0; bx < nb[0]; ++bx)
      for (int by = 0; by < nb[1]; ++by)
        for (int bz = 0; bz < nb[2]; ++bz) emit(bx, by, bz);
  }

  // ---- faces of the first sub-domain, in local element numbers
  const Vec f2e(f2e_in, f2e_in + 4 * (size_t)nf);
  const Vec e2f = elem_faces(f2e, nf, nfe, ne);
  std::map<int, int> loc;
  for (int c = 0; c < b.nese; ++c) loc[b.elem[(size_t)b.nse * c]] = c;
  Vec felem, seen(nf, 0);
  for (int c = 0; c < b.nese; ++c)
    for (int l = 0; l < nfe; ++l) {
      const int f = e2f[l + nfe * b.elem[(size_t)b.nse * c]];
      if (f >= 0 && !seen[f]) seen[f] = 1, felem.push_back(f);
    }
  const int nfs = (int)felem.size();
  Vec f2el(4 * (size_t)nfs);
  for (int i = 0; i < nfs; ++i) {
    const int* q = &f2e[4 * (size_t)felem[i]];
    const auto i1 = loc.find(q[0]);
    const auto i2 = q[2] >= 0 ? loc.find(q[2]) : loc.end();
    const bool in1 = i1 != loc.end(), in2 = i2 != loc.end();
    int v[4] = {q[0], q[1], q[2], q[3]};
    if (in1) v[0] = i1->second;
    if (in2) v[2] = i2->second;
    if (!in1 && in2) v[0] = i2->second, v[1] = q[3], v[2] = -1, v[3] = -1;
    if (!in2) v[2] = -1, v[3] = -1;
    for (int k = 0; k < 4; ++k) f2el[4 * (size_t)i + k] = v[k];
  }
  reorder_faces(f2el, nfs);
  b.nfse = nfs;

  // ---- CRS of the sub-domain face graph and the face map of every sub-domain
  const Vec f2f = face_neighbours(f2el, elem_faces(f2el, nfs, nfe, b.nese), nfs, nfe);
  const int nbf = 2 * (nfe - 1);
  b.row_ptr.assign(1, 0);
  b.col_ind.clear();
  for (int i = 0; i < nfs; ++i) {
    Vec nbr;
    for (int j = 0; j < nbf; ++j)
      if (f2f[j + (size_t)nbf * i] >= 0) nbr.push_back(f2f[j + (size_t)nbf * i]);
    std::sort(nbr.begin(), nbr.end());
    b.col_ind.push_back(i);
    b.col_ind.insert(b.col_ind.end(), nbr.begin(), nbr.end());
    b.row_ptr.push_back((int)b.col_ind.size());
  }
  b.nnz = (int)b.col_ind.size();
  b.face.assign((size_t)b.nse * nfs, 0);
  for (int s = 0; s < b.nse; ++s)
    for (int i = 0; i < nfs; ++i)
      b.face[s + (size_t)b.nse * i] = e2f[f2el[4 * (size_t)i + 1] + nfe * b.elem[s + (size_t)b.nse * f2el[4 * (size_t)i]]];

  // ---- ILU(0) schedule
  std::map<std::pair<int, int>, int> pos;
  b.row_of.assign(b.nnz, 0);
  for (int i = 0; i < nfs; ++i)
    for (int t = b.row_ptr[i]; t < b.row_ptr[i + 1]; ++t) pos[{i, b.col_ind[t]}] = t, b.row_of[t] = i;
  b.fac_ptr.assign(1, 0);
  b.fac_ji.clear();
  b.upd_ptr.assign(1, 0);
  b.upd_jl.clear();
  b.upd_il.clear();
  for (int i = 0; i < nfs; ++i) {
    for (int t = b.row_ptr[i]; t < b.row_ptr[i + 1]; ++t) {
      const int j = b.col_ind[t];
      const auto ji = pos.find({j, i});
      if (j <= i || ji == pos.end()) continue;
      b.fac_ji.push_back(ji->second);
      for (int t2 = b.row_ptr[i]; t2 < b.row_ptr[i + 1]; ++t2) {
        const int l = b.col_ind[t2];
        const auto jl = pos.find({j, l});
        if (l <= i || jl == pos.end()) continue;
        b.upd_jl.push_back(jl->second);
        b.upd_il.push_back(t2);
      }
      b.upd_ptr.push_back((int)b.upd_jl.size());
    }
    b.fac_ptr.push_back((int)b.fac_ji.size());
  }
  // ---- summing back: copies of each global face in fixed (sub-domain, local face) order
  std::vector<Vec> copies(nf);
  for (int i = 0; i < nfs; ++i)
    for (int s = 0; s < b.nse; ++s) copies[b.face[s + (size_t)b.nse * i]].push_back(s + b.nse * i);
  b.gf_ptr.assign(1, 0);
  b.gf_pos.clear();
  for (int f = 0; f < nf; ++f) {
    b.gf_pos.insert(b.gf_pos.end(), copies[f].begin(), copies[f].end());
    b.gf_ptr.push_back((int)b.gf_pos.size());
  }
  return 0;
}

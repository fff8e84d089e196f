// Host set-up of the super-element additive Schwarz preconditioner with block ILU(0)
// (Exasim preconditioner = 2): the Cartesian sub-domain partition, the face ordering of a
// sub-domain (the same CRS pattern for every sub-domain) and the schedule of the block
// factorization, as flat index arrays for the device kernels.
#pragma once
#include <vector>

struct ExaBilu {
  int nse = 0, nese = 0, nfse = 0, nnz = 0;
  std::vector<int> elem;                 // [nse, nese], column-major (r + nse * c)
  std::vector<int> row_ptr, col_ind;     // CRS of the sub-domain face graph, diagonal first
  std::vector<int> face;                 // [nse, nfse]: global face of local face i of domain r
  std::vector<int> row_of;               // [nnz]: row of each stored block
  // factorization: for row i, the blocks (j, i) with j > i (fac_ji[fac_ptr[i] .. fac_ptr[i+1]]),
  // and for each of them the updates (j, l) -= (j, i)(i, l), l > i (upd_ptr / upd_jl / upd_il)
  std::vector<int> fac_ptr, fac_ji, upd_ptr, upd_jl, upd_il;
  // summing back: the sub-domain copies (r + nse * i) of each global face
  std::vector<int> gf_ptr, gf_pos;
};

// Builds the partition and the ordering from cartgridpart ([2, Nx, Ny, Mx, My, opt] or
// [3, Nx, Ny, Nz, Mx, My, Mz, opt]) and the face connectivity f2e [4, nf] (0-based).
// Returns 0, or -1 with a message in err.
int exa_bilu_setup(const int* cgp, int ncgp, const int* f2e, int nf, int nfe, int ne, ExaBilu& b, char* err,
                   int errlen);

// Host-side face connectivity (see exa_conn.cpp).
#pragma once
#include <vector>

struct ExaConn {
  int nf = 0;                 // number of faces
  int nf0 = 0;                // interior faces (they come first)
  int nfe = 0;                // faces per element
  std::vector<int> f2e;       // [4, nf]: (e1, l1, e2, l2); e2 = l2 = -1 on boundary faces
  std::vector<int> elemcon;   // [npf*nfe, ne]: global face-node index of each element face node
};

// t [nve, ne] 0-based vertices; bf [nfe, ne] boundary codes (0 interior); perm [npf, nfe];
// xpf [npf, dim-1].  Returns nf, or -1 when two faces cannot be matched.
int exa_build_connectivity(const int* t, const int* bf, const int* perm, const double* xpf, int dim,
                           int elemtype, int ne, int npe, int npf, ExaConn& out);

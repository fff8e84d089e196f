// Test infrastructure: exposes the reference's own Cartesian sub-domain partition, face
// ordering and ILU(0) index routines (backend/Common/cpuimpl.h:1266-1625) through a C ABI,
// so the oracle's restatement of them can be checked against the reference itself.  Built
// by oracle/build_ref.sh from the reference tree into oracle/_ref/; never part of the product.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <numeric>
#include <string>
#include <vector>
using namespace std;
typedef double dstype;
typedef int Int;
static void error(const std::string& s) {
  fprintf(stderr, "%s\n", s.c_str());
  exit(1);
}
#include REF_CPUIMPL

extern "C" int ref_partition(int dim, const int* cgp, int** elem_out, int* nse_out, int* nese_out) {
  int* elem = nullptr;
  int nse = 0, nese = 0;
  if (dim == 2) {
    nse = gridpartition2d(&elem, cgp[1], cgp[2], cgp[3], cgp[4], cgp[5]);
    nese = cgp[3] * cgp[4];
  } else {
    nse = gridpartition3d(&elem, cgp[1], cgp[2], cgp[3], cgp[4], cgp[5], cgp[6], cgp[7]);
    nese = cgp[4] * cgp[5] * cgp[6];
  }
  *elem_out = elem;
  *nse_out = nse;
  *nese_out = nese;
  return 0;
}

// row_ptr [nfse + 1], col_ind [nnz], face [nse * nfse] written to caller buffers of the given
// capacities; returns nfse (or -1 when a buffer is too small)
extern "C" int ref_faceordering(const int* elem, const int* f2e, int nse, int nese, int nfe, int nf, int* row_ptr,
                                int cap_rp, int* col_ind, int cap_ci, int* face, int cap_face) {
  int *rp = nullptr, *ci = nullptr, *fc = nullptr, *fe = nullptr;
  int n = crs_faceordering(&rp, &ci, &fc, &fe, elem, f2e, nse, nese, nfe, nf);
  if (n + 1 > cap_rp || rp[n] > cap_ci || nse * n > cap_face) return -1;
  memcpy(row_ptr, rp, sizeof(int) * (n + 1));
  memcpy(col_ind, ci, sizeof(int) * rp[n]);
  memcpy(face, fc, sizeof(int) * nse * n);
  free(rp);
  free(ci);
  free(fc);
  free(fe);
  return n;
}

extern "C" void ref_free(void* p) { free(p); }

// Sizes shared by the HDG kernels and their host-side launchers.
#pragma once
#include "exa_common.cuh"

struct ExaDims {
  int nd, ncu, nc, ncq, ncx, nco, ncw;   // dimension and field components
  int npe, npf, nge, ngf, nfe, ndf;       // nodes / quadrature points per element and face
  int n, m;                               // n = npe*ncu (element block), m = ncu*npf*nfe (trace block)
  int ne, nf, nf0;                        // elements, faces, interior faces
  __host__ __device__ int elemg_stride() const { return nge * (ncx + nd * nd + 1); }
  __host__ __device__ int faceg_stride() const { return ngf * (ncx + nd + 1); }
};

int exa_k_geometry(const ExaDims& P, const double* shapegt, const double* shapfgt, const int* perm,
                   const double* xdg, double* elemg, double* faceg, cudaStream_t st);
int exa_k_qmats(const ExaDims& P, const double* shapegt, const double* shapegw, const double* shapfgt,
                const double* shapfgw, const int* perm, const double* elemg, const double* faceg, double* mass,
                double* cw, double* ew, cudaStream_t st);
int exa_k_scatter(const ExaDims& P, const int* f2e, const int* elemcon, const double* we, double* w, cudaStream_t st);
// block kernels, T = double (plain form) or float (mixed-precision form); vectors stay FP64
// flag (may be null): FP32 blocks given a device flag stream through shared memory by bulk
// copies with bounded waits; a wait that runs out sets *flag to EXA_UMMA_TIMEOUT
template <typename T>
int exa_k_elem_matvec(const ExaDims& P, const int* elemcon, const T* A, const double* v, double* we,
                      cudaStream_t st, int* flag = nullptr);
template <typename T>
int exa_k_bj_build(const ExaDims& P, const int* f2e, const int* elemcon, const T* H, T* BE, cudaStream_t st);
template <typename T>
int exa_k_eas_build(const ExaDims& P, const int* f2e, const int* elemcon, const T* H, T* BE, cudaStream_t st);
template <typename T>
int exa_k_bj_apply(const ExaDims& P, const T* BE, const double* x, double* y, cudaStream_t st);
template <typename T>
int exa_k_dudg(const ExaDims& P, const int* elemcon, const T* DinvF, const double* Ru, const double* x,
               double* du, cudaStream_t st, int* flag = nullptr);
// y_e = alpha A_e x_e + beta y_e per element e: A_e FP32 [M, K] column-major sA apart,
// x_e, y_e FP64 sx, sy apart (FP64 accumulation)
int exa_k_gemv32(int M, int K, int batch, double alpha, const float* A, long long sA, const double* x, long long sx,
                 double beta, double* y, long long sy, cudaStream_t st, int* flag = nullptr);
// D and B volume blocks on the tcgen05 tensor cores (3xTF32) for the mixed-precision form,
// with S = shapegt[:, :, 0] packed as a B operand (rows npe, K nge) and shapegw32 = shapegw in
// FP32; npe, nge <= 128.
struct UPacked;
bool exa_vol_mat_tc_fits(const ExaDims& P);
// With Bp.hi set, B goes into Bp (the packed FP32 A operand of the q elimination, one part per
// trace component: row i + npe k, k = j + qk_group(npe) d) instead of B.
int exa_k_vol_mat_tc(const ExaDims& P, const float* shapegw32, const UPacked& Sp, const double* rgJ, double* D,
                     double* B, const UPacked& Bp, int nb, int* flag, cudaStream_t st);
// Block ILU(0) preconditioner on Cartesian sub-domains (Exasim preconditioner = 2): the
// schedule built on the host (exa_bilu0.h) in device memory, and the sub-domain results.
struct ExaBiluDev {
  int nse = 0, nfse = 0, nnz = 0;
  int *row_ptr = nullptr, *col_ind = nullptr, *face = nullptr, *row_of = nullptr;
  int *fac_ptr = nullptr, *fac_ji = nullptr, *upd_ptr = nullptr, *upd_jl = nullptr, *upd_il = nullptr;
  int *gf_ptr = nullptr, *gf_pos = nullptr;
  double* out = nullptr;  // [nse * nfse, ncf]
};
size_t exa_bilu_apply_smem(int ncf, int nfse);
// blocks from the condensed element matrices H, then the block ILU(0) in place
template <typename T>
int exa_k_bilu_build(const ExaDims& P, const ExaBiluDev& b, const int* f2e, const int* elemcon, const T* H, T* BE,
                     int* flag, cudaStream_t st);
// w = P x (x and w trace vectors, x != w)
template <typename T>
int exa_k_bilu_apply(const ExaDims& P, const ExaBiluDev& b, const T* BE, const double* x, double* w,
                     cudaStream_t st);
// y = (float) x
int exa_k_to_f32(const double* x, float* y, long long n, cudaStream_t st);
int exa_k_udg_update(const ExaDims& P, double* udg, const double* du, double alpha, cudaStream_t st);
// q = Minv (C u - E uhat) by quadrature (no MinvC / MinvE reads).  With wpre, C u is taken
// from there (exa_k_getq_gemm) instead of computed per element.
size_t exa_getq_mf_smem(const ExaDims& P, bool wpre);  // shared memory of exa_k_getq_mf (wpre given or not)
int exa_k_getq_mf(const ExaDims& P, const double* shapegt, const double* shapegw, const double* shapfgt,
                  const double* shapfgw, const int* perm, const int* elemcon, const double* elemg,
                  const double* faceg, const double* Minv, const double* uh, double* udg, cudaStream_t st,
                  const double* wpre = nullptr);
// C_d u of every element as two FP64 tensor-core GEMMs whose left operands (shapegt, shapegw)
// all elements share: UG = shapegt u (nge x ncu ne), V = Xx (.) UG (nge nd x ncu nd ne), W =
// shapegw[:, :, 1..nd] V (npe x ncu nd ne, element e's block at W + e npe ncu nd, laid out as
// the per-element w of exa_k_getq_mf).  UG, V and W are caller workspace of those sizes.
int exa_k_getq_gemm(const ExaDims& P, const double* shapegt, const double* shapegw, const double* elemg,
                    const double* udg, double* UG, double* V, double* W, cudaStream_t st);
int exa_k_getq(const ExaDims& P, const int* elemcon, const double* MC, const double* ME, const double* uh,
               double* udg, cudaStream_t st);
int exa_k_face_nodes(const ExaDims& P, const int* f2e, const int* perm, const double* udg, double* uh, cudaStream_t st);

// LDG (exa_ldg.cu): the face-node table of both sides [2, npf, nf]; the element residual from
// the volume residual Rue and the face residuals Rh [npf, ncu, nf]; out = a x + b y
int exa_k_ldg_fcon(const ExaDims& P, const int* f2e, const int* perm, const int* elemcon, int* fcon, cudaStream_t st);
int exa_k_ldg_gather(const ExaDims& P, const int* f2e, const int* perm, const int* elemcon, const double* Rue,
                     const double* Rh, double* Ru, int tdep, double dtfactor, cudaStream_t st);
int exa_lincomb(double* out, double a, const double* x, double b, const double* y, long long n, cudaStream_t st);
// the element mass matrices [npe, npe, ne] (the LDG preconditioner inverts them)
int exa_k_ldg_mass(const ExaDims& P, const double* shapegt, const double* shapegw, const double* elemg, double* mass,
                   cudaStream_t st);

// Shared definitions of the B200 HDG solver: error codes, checked CUDA calls,
// launch helpers and the device-side linear-algebra entry points.
//
// Data layouts (column-major, first index fastest) follow Exasim's HDG backend
// after its Schur reordering (backend/Common/kokkosimpl.h:1797-2020), with the
// element index outermost so one element's block is contiguous in HBM:
//   udg  [npe, nc, ne]            uh  [ncu, npf, nf]
//   D    [n, n]     per element   n = npe*ncu, row (i,k) = i + npe*k
//   F    [n, m]     per element   m = ncu*npf*nfe, col (c,jf) = c + ncu*jf
//   K    [m, n]     per element   row (k,jf) = k + ncu*jf
//   H    [m, m]     per element
//   B    [n, npe*nd*ncu], G [m, npe*nd*ncu]: column (j, d, n) = j + npe*d + npe*nd*n
//   MinvC [npe, nd, npe], MinvE [npe, nd, ndf] per element (dimension next to the row)
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

// Status codes returned by every exa_* entry point (include/exasim_b200.h).
enum ExaStatus {
  EXA_OK = 0,
  EXA_ERR_ARG = 1,          // bad argument or inconsistent input sizes
  EXA_ERR_UNSUPPORTED = 2,  // input asks for a feature outside the HDG hot path
  EXA_ERR_CUDA = 3,         // a CUDA call failed (message via exa_last_error)
  EXA_ERR_SINGULAR = 4,     // a dense block had a zero pivot
  EXA_ERR_MESH = 5,         // mesh connectivity could not be built
  EXA_ERR_NOTCONV = 6,      // solver stopped without reaching its tolerance
  EXA_ERR_NAN = 7,          // residual norm is NaN
  EXA_ERR_NOMEM = 8,        // device allocation refused
  EXA_ERR_TIMEOUT = 9,      // a wait ran out before its request finished
};

void exa_set_error(const char* fmt, ...);
// Lets `fn` launch with `bytes` of dynamic shared memory.  The attribute is set to the
// device maximum (227 KB), the same value for every caller, so host threads launching the
// same kernel with different sizes cannot undo each other's setting.
int exa_allow_smem(const void* fn, size_t bytes);
const char* exa_get_error();

#define EXA_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      exa_set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
      return EXA_ERR_CUDA;                                                          \
    }                                                                               \
  } while (0)

#define EXA_TRY(call)               \
  do {                              \
    int s_ = (call);                \
    if (s_ != EXA_OK) return s_;    \
  } while (0)

// Every kernel launch site ends with EXA_LAUNCH_CHECK(), which also counts the launch
// (exa_launch_count() in the C ABI).
void exa_count_launch();
// Launches made by the calling host thread, and an adjustment of both counts: a captured CUDA
// graph's kernels are counted when the graph is replayed, not when it is captured.
long long exa_thread_launches();
void exa_add_launches(long long n);

#define EXA_LAUNCH_CHECK()                                                          \
  do {                                                                              \
    exa_count_launch();                                                             \
    cudaError_t e_ = cudaGetLastError();                                            \
    if (e_ != cudaSuccess) {                                                        \
      exa_set_error("%s:%d launch: %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
      return EXA_ERR_CUDA;                                                          \
    }                                                                               \
  } while (0)

// Strided batched GEMM in FP64:  C = alpha * A * B + beta * C  for every batch entry
// (b1, b2) in [0, batch) x [0, batch2), with
//   A(r, k) = A[r + lda*k + sA*b1 + sA2*b2], B(k, c) = B[k + ldb*c + ...], C(r, c) = C[r + ldc*c + ...].
// beta == 0 does not read C.
struct GemmBatch {
  int M, N, K;
  double alpha, beta;
  const double* A; long long lda, sA, sA2;
  const double* B; long long ldb, sB, sB2;
  double* C; long long ldc, sC, sC2;
  int batch, batch2;
};
int exa_gemm(const GemmBatch& g, cudaStream_t st);
// Times the FP64 GEMM's candidate CTA tiles for one shape on scratch blocks and keeps the
// fastest for this device (an autotuner; exa_gemm uses a padding heuristic for shapes not
// tuned).  The tile does not change the result.  Not for use inside stream capture.
int exa_gemm_tune(int M, int N, int K, int batch, cudaStream_t st);
// The same for the dense element inverse of order 32 < n <= 128: times the column-by-warp
// shapes on up to 4096 scratch blocks (the default shape stays if they do not fit) and keeps
// the fastest for this device, order and type (all shapes give the same bits).  Synchronizes
// st; call it outside stream capture.
int exa_inverse_tune(int n, int batch, int fp64, cudaStream_t st);
int exa_inverse_variant_of(int n, int fp64);  // the shape exa_inverse uses for order n (-1: not tuned here)
int exa_gemm_tile_of(int M, int N, int K);  // index of the tile exa_gemm uses for the shape

// In-place explicit inverse of `batch` n x n column-major matrices spaced `stride`
// doubles apart (Gauss-Jordan with partial pivoting in shared memory).  Sets
// *d_flag (device int) non-zero when a pivot is exactly zero.
int exa_inverse(double* A, int n, long long stride, int batch, int* d_flag, cudaStream_t st);
int exa_inverse(float* A, int n, long long stride, int batch, int* d_flag, cudaStream_t st);
// The same for n up to exa_inverse_max_n(): orders above the register kernel's limit
// (exa_inverse_needs_ws) are inverted blockwise and need ws, n^2 entries per matrix,
// spaced n^2 apart.
int exa_inverse_max_n();
int exa_inverse_needs_ws(int n);
int exa_inverse_ws(double* A, int n, long long stride, int batch, double* ws, int* d_flag, cudaStream_t st);
int exa_inverse_ws(float* A, int n, long long stride, int batch, float* ws, int* d_flag, cudaStream_t st);
// FP32 blocks of order up to exa_inverse_max_n(): above the register kernel's limit by the
// blocked form applied recursively, its products on the tcgen05 3xTF32 GEMM.  ws holds
// exa_inverse_tc32_ws(n) floats and pk exa_inverse_tc32_pk(n) floats per matrix (both 0 for
// orders the register kernel takes whole); *uflag reports a tensor-core wait that ran out.
long long exa_inverse_tc32_ws(int n);
long long exa_inverse_tc32_pk(int n);
int exa_inverse_tc32(float* A, int n, long long stride, int batch, float* ws, float* pk, int* d_flag, int* uflag,
                     cudaStream_t st);

// Vector kernels for the Krylov solver.  Reductions are deterministic: each block
// writes a partial sum and consumers reduce the partial array in a fixed order.
int exa_vec_blocks();
int exa_dot_partials(const double* x, const double* y, long long n, double* part, cudaStream_t st);
int exa_reduce_partials(const double* part, long long n, double* out, int take_sqrt, cudaStream_t st);
int exa_axpby(double* y, const double* x, double a, double b, long long n, cudaStream_t st);
int exa_scale(double* y, const double* x, double a, long long n, cudaStream_t st);
int exa_fill(double* y, double a, long long n, cudaStream_t st);
// One modified Gram-Schmidt step: h = sum(part_in); w -= h * vprev; part_out = partial(w . vnext).
int exa_mgs_step(double* w, const double* vprev, const double* vnext, const double* part_in,
                 double* part_out, double* h_out, long long n, cudaStream_t st);
// h = sqrt(sum(part_in)); v = w / h.
int exa_mgs_finish(double* v, const double* w, const double* part_in, double* h_out, long long n,
                   cudaStream_t st);
// Givens rotations on Hessenberg column i (cpuApplyGivensRotation semantics); writes
// |s[i+1]| / nrmb to *relerr.
int exa_givens(double* hcol, double* s, double* cs, double* sn, int i, const double* nrmb,
               double* relerr, cudaStream_t st);
// x += V(:, 0:k) y   (V column-major N x k, y on device)
int exa_gemv_add(double* x, const double* V, const double* y, long long n, int k, cudaStream_t st);
// hcol(0:k) = V(:, 0:k)^T w, then w -= V(:,0:k) hcol(0:k)   (classical Gram-Schmidt)
int exa_cgs(double* w, const double* V, double* hcol, double* part, long long n, int k, cudaStream_t st);

inline int exa_ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Dense FP64 building blocks of the HDG solver: strided batched GEMM, batched
// Gauss-Jordan inverse, and the deterministic vector reductions used by GMRES.
//
// Exasim runs these steps through cuBLAS (DgemmStridedBatched, DgetrfBatched +
// DgetriBatched, Ddot/Daxpy/Dscal: backend/Common/pblas.h:163-734).  Here they are
// plain SIMT kernels: the element blocks (n, m <= a few hundred) are too small for
// tensor-core tiles in FP64, and the reductions stay on the device so the Krylov loop
// only synchronises once per iteration.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cmath>

#include "exa_common.cuh"

#include <atomic>

static char g_err[1024] = "";
static std::atomic<long long> g_launches{0};

void exa_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
extern "C" long long exa_launch_count(void) { return g_launches.load(); }

void exa_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
const char* exa_get_error() { return g_err; }

// ----------------------------------------------------------------------------------
// batched GEMM: 64x64 output tile per block, 256 threads, 4x4 accumulators per thread
// (rows ty + 16*a, cols tx + 16*b so shared-memory reads are conflict free), K staged
// through shared memory in chunks of 16.
// ----------------------------------------------------------------------------------
namespace {
constexpr int TM = 64, TN = 64, TK = 16;

__global__ void __launch_bounds__(256) gemm_kernel(GemmBatch g) {
  __shared__ double As[TK][TM + 1];
  __shared__ double Bs[TK][TN + 1];
  const int tilesM = (g.M + TM - 1) / TM;
  const int tm = blockIdx.x % tilesM, tn = blockIdx.x / tilesM;
  const long long b1 = blockIdx.y, b2 = blockIdx.z;
  const double* A = g.A + b1 * g.sA + b2 * g.sA2;
  const double* B = g.B + b1 * g.sB + b2 * g.sB2;
  double* C = g.C + b1 * g.sC + b2 * g.sC2;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int r0 = tm * TM, c0 = tn * TN;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;

  for (int k0 = 0; k0 < g.K; k0 += TK) {
    // A tile: 64 rows x 16 k, element t -> (row t%64, k t/64), coalesced along rows
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int t = threadIdx.x + 256 * q;
      int r = t & 63, k = t >> 6;
      int gr = r0 + r, gk = k0 + k;
      As[k][r] = (gr < g.M && gk < g.K) ? A[gr + g.lda * gk] : 0.0;
    }
    // B tile: 16 k x 64 cols, element t -> (k t%16, col t/16), coalesced along k
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int t = threadIdx.x + 256 * q;
      int k = t & 15, c = t >> 4;
      int gk = k0 + k, gc = c0 + c;
      Bs[k][c] = (gk < g.K && gc < g.N) ? B[gk + g.ldb * gc] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < TK; ++k) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = As[k][ty + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = Bs[k][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    int gr = r0 + ty + 16 * a;
    if (gr >= g.M) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      int gc = c0 + tx + 16 * b;
      if (gc >= g.N) continue;
      double* p = C + gr + g.ldc * gc;
      double v = g.alpha * acc[a][b];
      *p = (g.beta == 0.0) ? v : v + g.beta * (*p);
    }
  }
}
}  // namespace

int exa_gemm(const GemmBatch& g, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0 || g.batch2 <= 0) return EXA_OK;
  if (g.batch > 65535 * 1024 || g.batch2 > 65535) {
    exa_set_error("gemm batch too large (%d, %d)", g.batch, g.batch2);
    return EXA_ERR_ARG;
  }
  dim3 grid((unsigned)(exa_ceil_div(g.M, TM) * exa_ceil_div(g.N, TN)), (unsigned)g.batch, (unsigned)g.batch2);
  if (grid.y > 65535) {
    // split the first batch dimension into chunks the grid can hold
    for (int b0 = 0; b0 < g.batch; b0 += 65535) {
      GemmBatch h = g;
      h.A += (long long)b0 * g.sA;
      h.B += (long long)b0 * g.sB;
      h.C += (long long)b0 * g.sC;
      h.batch = (g.batch - b0 < 65535) ? g.batch - b0 : 65535;
      EXA_TRY(exa_gemm(h, st));
    }
    return EXA_OK;
  }
  gemm_kernel<<<grid, 256, 0, st>>>(g);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

// ----------------------------------------------------------------------------------
// batched explicit inverse (Gauss-Jordan, partial pivoting, column swaps undone at the
// end).  Exasim forms the same explicit inverse with getrf + getri
// (backend/Common/pblas.h:163-260); the pivot choice (largest magnitude, first on ties)
// matches LAPACK's partial pivoting.
// ----------------------------------------------------------------------------------
namespace {
constexpr int INV_MAX_N = 160;

__global__ void __launch_bounds__(512) inverse_kernel(double* Aall, int n, long long stride, int* flag) {
  extern __shared__ double sm[];
  double* A = sm;                                  // n x n, column-major
  __shared__ int ipiv[INV_MAX_N];
  __shared__ double s_d;
  __shared__ int s_p;
  double* G = Aall + (long long)blockIdx.x * stride;
  const int nn = n * n;
  for (int t = threadIdx.x; t < nn; t += blockDim.x) A[t] = G[t];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < n; ++k) {
    if (warp == 0) {
      double best = -1.0;
      int bi = n;
      for (int i = k + lane; i < n; i += 32) {
        double v = fabs(A[i + n * k]);
        if (v > best) { best = v; bi = i; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        double ob = __shfl_down_sync(0xffffffffu, best, off);
        int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (lane == 0) {
        if (!(best > 0.0)) { atomicExch(flag, 1); bi = k; }
        s_p = bi;
        ipiv[k] = bi;
      }
    }
    __syncthreads();
    const int p = s_p;
    if (p != k) {
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double t = A[k + n * j];
        A[k + n * j] = A[p + n * j];
        A[p + n * j] = t;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) s_d = 1.0 / A[k + n * k];
    __syncthreads();
    const double d = s_d;
    for (int j = threadIdx.x; j < n; j += blockDim.x) A[k + n * j] = (j == k) ? d : A[k + n * j] * d;
    __syncthreads();
    // rank-1 update of every entry off row k and column k
    for (int t = threadIdx.x; t < nn; t += blockDim.x) {
      int i = t % n, j = t / n;
      if (i != k && j != k) A[t] -= A[i + n * k] * A[k + n * j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      if (i != k) A[i + n * k] = -A[i + n * k] * d;
    __syncthreads();
  }
  for (int k = n - 1; k >= 0; --k) {
    const int p = ipiv[k];
    if (p != k) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double t = A[i + n * k];
        A[i + n * k] = A[i + n * p];
        A[i + n * p] = t;
      }
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < nn; t += blockDim.x) G[t] = A[t];
}
}  // namespace

int exa_inverse(double* A, int n, long long stride, int batch, int* d_flag, cudaStream_t st) {
  if (batch <= 0) return EXA_OK;
  if (n > INV_MAX_N || n <= 0) {
    exa_set_error("dense inverse of order %d exceeds the shared-memory kernel limit %d", n, INV_MAX_N);
    return EXA_ERR_UNSUPPORTED;
  }
  size_t smem = (size_t)n * n * sizeof(double);
  static bool attr_set = false;
  if (!attr_set) {
    EXA_CUDA(cudaFuncSetAttribute(inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  INV_MAX_N * INV_MAX_N * (int)sizeof(double)));
    attr_set = true;
  }
  int threads = n * n >= 4096 ? 512 : (n * n >= 1024 ? 256 : 128);
  for (int b0 = 0; b0 < batch; b0 += 1 << 30) {
    int nb = batch - b0;
    inverse_kernel<<<nb, threads, smem, st>>>(A + (long long)b0 * stride, n, stride, d_flag);
    EXA_LAUNCH_CHECK();
  }
  return EXA_OK;
}

// ----------------------------------------------------------------------------------
// vector kernels.  A fixed grid of VB blocks (two per SM) covers every vector with a
// grid-stride loop; each reduction leaves VB partial sums that the consumer kernel
// adds up in index order, so results do not depend on scheduling.
// ----------------------------------------------------------------------------------
namespace {
constexpr int VB = 296, VT = 256;

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[VT / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < VT / 32; ++w) s += red[w];
  }
  return s;  // valid in thread 0
}

// every block reduces the VB partials in the same order (thread-parallel, then fixed tree)
__device__ __forceinline__ double sum_partials(const double* part) {
  __shared__ double tot;
  double v = 0.0;
  for (int i = threadIdx.x; i < VB; i += VT) v += part[i];
  double s = block_sum(v);
  if (threadIdx.x == 0) tot = s;
  __syncthreads();
  return tot;
}

__global__ void __launch_bounds__(VT) dot_kernel(const double* x, const double* y, long long n, double* part) {
  double v = 0.0;
  for (long long i = blockIdx.x * (long long)VT + threadIdx.x; i < n; i += (long long)VB * VT) v = fma(x[i], y[i], v);
  double s = block_sum(v);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(VT) reduce_kernel(const double* part, double* out, int take_sqrt) {
  double s = sum_partials(part);
  if (threadIdx.x == 0) *out = take_sqrt ? sqrt(s) : s;
}

__global__ void axpby_kernel(double* y, const double* x, double a, double b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

__global__ void scale_kernel(double* y, const double* x, double a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = a * x[i];
}

__global__ void fill_kernel(double* y, double a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = a;
}

__global__ void __launch_bounds__(VT) mgs_step_kernel(double* w, const double* vprev, const double* vnext,
                                                      const double* part_in, double* part_out, double* h_out,
                                                      long long n) {
  const double h = sum_partials(part_in);
  if (blockIdx.x == 0 && threadIdx.x == 0) *h_out = h;
  double v = 0.0;
  for (long long i = blockIdx.x * (long long)VT + threadIdx.x; i < n; i += (long long)VB * VT) {
    double wi = w[i] - h * vprev[i];
    w[i] = wi;
    v = fma(wi, vnext ? vnext[i] : wi, v);
  }
  double s = block_sum(v);
  if (threadIdx.x == 0) part_out[blockIdx.x] = s;
}

__global__ void __launch_bounds__(VT) mgs_finish_kernel(double* vout, const double* w, const double* part_in,
                                                        double* h_out, long long n) {
  const double h = sqrt(sum_partials(part_in));
  if (blockIdx.x == 0 && threadIdx.x == 0) *h_out = h;
  const double r = 1.0 / h;
  for (long long i = blockIdx.x * (long long)VT + threadIdx.x; i < n; i += (long long)VB * VT) vout[i] = w[i] * r;
}

// cpuApplyGivensRotation (backend/Common/cpuimpl.h:167-196) on the device
__global__ void givens_kernel(double* H, double* s, double* cs, double* sn, int i, const double* nrmb, double* relerr) {
  double temp;
  for (int k = 0; k < i; k++) {
    temp = cs[k] * H[k] + sn[k] * H[k + 1];
    H[k + 1] = -sn[k] * H[k] + cs[k] * H[k + 1];
    H[k] = temp;
  }
  if (H[i + 1] == 0.0) {
    cs[i] = 1.0;
    sn[i] = 0.0;
  } else if (fabs(H[i + 1]) > fabs(H[i])) {
    temp = H[i] / H[i + 1];
    sn[i] = 1.0 / sqrt(1.0 + temp * temp);
    cs[i] = temp * sn[i];
  } else {
    temp = H[i + 1] / H[i];
    cs[i] = 1.0 / sqrt(1.0 + temp * temp);
    sn[i] = temp * cs[i];
  }
  temp = cs[i] * s[i];
  s[i + 1] = -sn[i] * s[i];
  s[i] = temp;
  H[i] = cs[i] * H[i] + sn[i] * H[i + 1];
  H[i + 1] = 0.0;
  *relerr = fabs(s[i + 1]) / *nrmb;
}

__global__ void gemv_add_kernel(double* x, const double* V, const double* y, long long n, int k) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int j = 0; j < k; ++j) acc = fma(V[i + n * j], y[j], acc);
    x[i] += acc;
  }
}

// partial dots of w against the k columns of V: part[j*VB + block]
__global__ void __launch_bounds__(VT) multi_dot_kernel(const double* w, const double* V, long long n, int k, double* part) {
  for (int j = 0; j < k; ++j) {
    double v = 0.0;
    for (long long i = blockIdx.x * (long long)VT + threadIdx.x; i < n; i += (long long)VB * VT)
      v = fma(V[i + n * j], w[i], v);
    double s = block_sum(v);
    if (threadIdx.x == 0) part[j * VB + blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(VT) multi_reduce_kernel(const double* part, double* h, int k) {
  for (int j = 0; j < k; ++j) {
    double s = sum_partials(part + j * VB);
    if (threadIdx.x == 0) h[j] = s;
    __syncthreads();
  }
}

__global__ void gemv_sub_kernel(double* w, const double* V, const double* h, long long n, int k) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int j = 0; j < k; ++j) acc = fma(V[i + n * j], h[j], acc);
    w[i] -= acc;
  }
}
}  // namespace

int exa_vec_blocks() { return VB; }

int exa_dot_partials(const double* x, const double* y, long long n, double* part, cudaStream_t st) {
  dot_kernel<<<VB, VT, 0, st>>>(x, y, n, part);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_reduce_partials(const double* part, double* out, int take_sqrt, cudaStream_t st) {
  reduce_kernel<<<1, VT, 0, st>>>(part, out, take_sqrt);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_axpby(double* y, const double* x, double a, double b, long long n, cudaStream_t st) {
  if (n <= 0) return EXA_OK;
  axpby_kernel<<<VB, VT, 0, st>>>(y, x, a, b, n);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_scale(double* y, const double* x, double a, long long n, cudaStream_t st) {
  if (n <= 0) return EXA_OK;
  scale_kernel<<<VB, VT, 0, st>>>(y, x, a, n);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_fill(double* y, double a, long long n, cudaStream_t st) {
  if (n <= 0) return EXA_OK;
  fill_kernel<<<VB, VT, 0, st>>>(y, a, n);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_mgs_step(double* w, const double* vprev, const double* vnext, const double* part_in,
                 double* part_out, double* h_out, long long n, cudaStream_t st) {
  mgs_step_kernel<<<VB, VT, 0, st>>>(w, vprev, vnext, part_in, part_out, h_out, n);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_mgs_finish(double* v, const double* w, const double* part_in, double* h_out, long long n, cudaStream_t st) {
  mgs_finish_kernel<<<VB, VT, 0, st>>>(v, w, part_in, h_out, n);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_givens(double* hcol, double* s, double* cs, double* sn, int i, const double* nrmb, double* relerr,
               cudaStream_t st) {
  givens_kernel<<<1, 1, 0, st>>>(hcol, s, cs, sn, i, nrmb, relerr);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_gemv_add(double* x, const double* V, const double* y, long long n, int k, cudaStream_t st) {
  if (k <= 0) return EXA_OK;
  gemv_add_kernel<<<VB, VT, 0, st>>>(x, V, y, n, k);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_cgs(double* w, const double* V, double* hcol, double* part, long long n, int k, cudaStream_t st) {
  multi_dot_kernel<<<VB, VT, 0, st>>>(w, V, n, k, part);
  EXA_LAUNCH_CHECK();
  multi_reduce_kernel<<<1, VT, 0, st>>>(part, hcol, k);
  EXA_LAUNCH_CHECK();
  gemv_sub_kernel<<<VB, VT, 0, st>>>(w, V, hcol, n, k);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

// Dense FP64 building blocks of the HDG solver: strided batched GEMM, batched
// Gauss-Jordan inverse, and the deterministic vector reductions used by GMRES.
//
// Exasim runs these steps through cuBLAS (DgemmStridedBatched, DgetrfBatched +
// DgetriBatched, Ddot/Daxpy/Dscal: backend/Common/pblas.h:163-734).  Here the GEMM runs
// on the FP64 tensor cores (DMMA) with CTA tiles sized to the element blocks (n, m of a
// few hundred), the inverse keeps each block in registers across a 512-thread CTA, and
// the reductions stay on the device so the Krylov loop only synchronises once per
// iteration.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cmath>

#include "exa_common.cuh"
#include "exa_umma.cuh"

#include <algorithm>
#include <array>
#include <atomic>
#include <map>
#include <mutex>
#include <set>
#include <utility>

static thread_local char g_err[1024] = "";  // per host thread: each context is driven by one thread
static std::atomic<long long> g_launches{0};

int exa_allow_smem(const void* fn, size_t bytes) {
  constexpr size_t kMax = 227 * 1024;
  if (bytes > kMax) {
    exa_set_error("kernel needs %zu bytes of shared memory, more than %zu", bytes, kMax);
    return EXA_ERR_UNSUPPORTED;
  }
  if (bytes <= 48 * 1024) return EXA_OK;
  // once per device and kernel: later launches (graph captures among them) make no call
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  if (done.count({dev, fn})) return EXA_OK;
  // the kernel's static shared memory counts against the same per-block limit
  cudaFuncAttributes fa{};
  EXA_CUDA(cudaFuncGetAttributes(&fa, fn));
  const size_t cap = kMax > fa.sharedSizeBytes ? kMax - fa.sharedSizeBytes : 0;
  if (bytes > cap) {
    exa_set_error("kernel needs %zu bytes of dynamic shared memory, more than %zu", bytes, cap);
    return EXA_ERR_UNSUPPORTED;
  }
  EXA_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap));
  done.insert({dev, fn});
  return EXA_OK;
}

static thread_local long long t_launches = 0;  // this host thread's launches (graph captures count them)

void exa_count_launch() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  ++t_launches;
}
long long exa_thread_launches() { return t_launches; }
void exa_add_launches(long long n) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  t_launches += n;
}
extern "C" long long exa_launch_count(void) { return g_launches.load(); }

void exa_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
const char* exa_get_error() { return g_err; }

namespace {
// C = alpha A x + beta C for N = 1: one thread per output row
__global__ void gemv_batch_kernel(GemmBatch g) {
  const long long b1 = blockIdx.y, b2 = blockIdx.z;
  const double* A = g.A + b1 * g.sA + b2 * g.sA2;
  const double* x = g.B + b1 * g.sB + b2 * g.sB2;
  double* C = g.C + b1 * g.sC + b2 * g.sC2;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < g.M; r += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < g.K; ++k) s = fma(A[r + g.lda * k], x[k], s);
    const double v = g.alpha * s;
    C[r] = (g.beta == 0.0) ? v : v + g.beta * C[r];
  }
}

// ----------------------------------------------------------------------------------
// FP64 tensor-core (DMMA, mma.sync m8n8k4 f64) batched GEMM.  A warp owns a
// (8 TI) x (8 TJ) block of C held as TI*TJ 8x8 accumulator fragments; the CTA is a
// WM x WN grid of warps, one CTA tile of one batch entry per block.  A and B stream
// through a GST-stage ring of shared-memory buffers, GK deep along K, filled with
// cp.async (8-byte copies, zero-filled outside the matrix) so no registers stage the
// loads and up to GST-1 chunks are in flight while one is multiplied.  Tiles are stored
// k-major with a row stride of 4 (mod 16) doubles: the fragment loads of each half-warp
// and the cp.async writes of four consecutive k by four columns hit distinct banks.
// Fragment layout (PTX ISA, m8n8k4 .f64): a0 = A[lane/4][lane%4], b0 = B[lane%4][lane/4],
// c0/c1 = C[lane/4][2 (lane%4) + 0/1].
// ----------------------------------------------------------------------------------
constexpr int GK = 16, GST = 3;

__host__ __device__ constexpr int dmma_stride(int w) { return (w + 15) / 16 * 16 + 4; }

template <int TI, int TJ, int WM, int WN>
constexpr size_t dmma_smem() {
  return sizeof(double) * (size_t)GST * GK * (dmma_stride(8 * TI * WM) + dmma_stride(8 * TJ * WN));
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// 8-byte asynchronous copy global -> shared; src_bytes = 0 writes zeros and reads nothing
__device__ __forceinline__ void cp_async8(double* dst, const double* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int TI, int TJ, int WM, int WN>
__global__ void __launch_bounds__(32 * WM * WN, 2) dmma_gemm_kernel(GemmBatch g) {
  constexpr int BM = 8 * TI * WM, BN = 8 * TJ * WN, NT = 32 * WM * WN;
  constexpr int SA = dmma_stride(BM), SB = dmma_stride(BN);
  constexpr int LA = (BM * GK + NT - 1) / NT, LB = (BN * GK + NT - 1) / NT;
  extern __shared__ __align__(16) double dsm[];
  double* As = dsm;                    // [GST][GK][SA]
  double* Bs = dsm + GST * GK * SA;    // [GST][GK][SB]
  const int tilesM = (g.M + BM - 1) / BM;
  const int tm = blockIdx.x % tilesM, tn = blockIdx.x / tilesM;
  const long long b1 = blockIdx.y, b2 = blockIdx.z;
  const double* A = g.A + b1 * g.sA + b2 * g.sA2;
  const double* B = g.B + b1 * g.sB + b2 * g.sB2;
  double* C = g.C + b1 * g.sC + b2 * g.sC2;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % WM, wn = warp / WM;
  const int r0 = tm * BM, c0 = tn * BN;
  const int gq = lane >> 2, tq = lane & 3;
  double acc[TI][TJ][2];
#pragma unroll
  for (int i = 0; i < TI; ++i)
#pragma unroll
    for (int j = 0; j < TJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int nk = (g.K + GK - 1) / GK;
  // stage s <- K chunk kc.  A: consecutive threads take consecutive rows (contiguous in
  // global and in shared memory).  B: groups of four threads take four consecutive k of
  // one column (one 32-byte sector), the next group the next column.
  auto load = [&](int s, int kc) {
    const int k0 = kc * GK;
    double* as = As + s * GK * SA;
    double* bs = Bs + s * GK * SB;
#pragma unroll
    for (int q = 0; q < LA; ++q) {
      const int t = tid + NT * q;
      const int r = t % BM, k = t / BM;
      if (k < GK) {
        const int gr = r0 + r, gk = k0 + k;
        const bool in = gr < g.M && gk < g.K;
        cp_async8(as + k * SA + r, in ? A + gr + g.lda * gk : A, in ? 8 : 0);
      }
    }
#pragma unroll
    for (int q = 0; q < LB; ++q) {
      const int t = tid + NT * q;
      const int rest = t >> 2, c = rest % BN, k = (t & 3) + 4 * (rest / BN);
      if (k < GK) {
        const int gk = k0 + k, gc = c0 + c;
        const bool in = gk < g.K && gc < g.N;
        cp_async8(bs + k * SB + c, in ? B + gk + g.ldb * gc : B, in ? 8 : 0);
      }
    }
  };
#pragma unroll
  for (int s = 0; s < GST - 1; ++s) {
    if (s < nk) load(s, s);
    cp_async_commit();
  }
  const int wr = wm * 8 * TI, wc = wn * 8 * TJ;
  for (int kc = 0; kc < nk; ++kc) {
    cp_async_wait<GST - 2>();
    __syncthreads();  // chunk kc visible to all; the buffer of chunk kc-1 is free
    if (kc + GST - 1 < nk) load((kc + GST - 1) % GST, kc + GST - 1);
    cp_async_commit();
    const double* as = As + (kc % GST) * GK * SA;
    const double* bs = Bs + (kc % GST) * GK * SB;
#pragma unroll
    for (int k4 = 0; k4 < GK; k4 += 4) {
      double af[TI], bf[TJ];
#pragma unroll
      for (int i = 0; i < TI; ++i) af[i] = as[(k4 + tq) * SA + wr + 8 * i + gq];
#pragma unroll
      for (int j = 0; j < TJ; ++j) bf[j] = bs[(k4 + tq) * SB + wc + 8 * j + gq];
#pragma unroll
      for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int j = 0; j < TJ; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int i = 0; i < TI; ++i) {
    const int gr = r0 + wr + 8 * i + gq;
    if (gr >= g.M) continue;
#pragma unroll
    for (int j = 0; j < TJ; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gc = c0 + wc + 8 * j + 2 * tq + h;
        if (gc >= g.N) continue;
        double* p = C + gr + g.ldc * gc;
        const double v = g.alpha * acc[i][j][h];
        *p = (g.beta == 0.0) ? v : v + g.beta * (*p);
      }
  }
}

template <int TI, int TJ, int WM, int WN>
int launch_dmma(const GemmBatch& g, cudaStream_t st) {
  constexpr int BM = 8 * TI * WM, BN = 8 * TJ * WN;
  constexpr size_t smem = dmma_smem<TI, TJ, WM, WN>();
  static_assert(smem <= 227 * 1024, "GEMM tile exceeds shared memory");
  auto kern = dmma_gemm_kernel<TI, TJ, WM, WN>;
  EXA_TRY(exa_allow_smem((const void*)kern, smem));
  dim3 grid((unsigned)(exa_ceil_div(g.M, BM) * exa_ceil_div(g.N, BN)), (unsigned)g.batch, (unsigned)g.batch2);
  kern<<<grid, 32 * WM * WN, smem, st>>>(g);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

long long tiles_cost(int M, int N, int bm, int bn) {
  return (long long)((M + bm - 1) / bm) * bm * ((N + bn - 1) / bn) * bn;
}

// CTA tiles sized to the element blocks: 128 x 64, 128 x 80, 160 x 32 and 160 x 64 cover
// 125 -> 128 and 150 -> 160 with little padding; 64 x 128 and 64 x 64 fit the chunk-wide
// products with 64 rows (Gauss points or nodes of a p = 3 hexahedron) and long rows of columns
constexpr int kTiles = 6;
constexpr int kTile[kTiles][2] = {{128, 64}, {128, 80}, {160, 32}, {160, 64}, {64, 128}, {64, 64}};

int launch_tile(int t, const GemmBatch& g, cudaStream_t st) {
  switch (t) {
    case 0: return launch_dmma<4, 4, 4, 2>(g, st);
    case 1: return launch_dmma<4, 5, 4, 2>(g, st);
    case 2: return launch_dmma<5, 2, 4, 2>(g, st);
    case 3: return launch_dmma<5, 4, 4, 2>(g, st);
    case 4: return launch_dmma<2, 8, 4, 2>(g, st);
    default: return launch_dmma<2, 4, 4, 2>(g, st);
  }
}

std::mutex g_tune_mu;
std::map<std::array<int, 4>, int> g_tune;  // (device, M, N, K) -> measured fastest tile

// the measured tile of this shape, else the least padded of 128 x 64, 128 x 80 and 160 x 32
int gemm_tile(int M, int N, int K) {
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find({dev, M, N, K});
    if (it != g_tune.end()) return it->second;
  }
  int best = 0;
  long long bc = -1;
  for (int i = 0; i < 3; ++i) {
    const long long c = tiles_cost(M, N, kTile[i][0], kTile[i][1]);
    if (bc < 0 || c < bc) { bc = c; best = i; }
  }
  return best;
}
}  // namespace

int exa_gemm(const GemmBatch& g, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0 || g.batch2 <= 0) return EXA_OK;
  if (g.batch2 > 65535) {
    exa_set_error("gemm second batch dimension too large (%d)", g.batch2);
    return EXA_ERR_ARG;
  }
  if (g.batch > 65535) {
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
  if (g.N == 1) {
    dim3 grid((unsigned)exa_ceil_div(g.M, 128), (unsigned)g.batch, (unsigned)g.batch2);
    gemv_batch_kernel<<<grid, 128, 0, st>>>(g);
    EXA_LAUNCH_CHECK();
    return EXA_OK;
  }
  if (g.M <= 40 && g.N <= 40) return launch_dmma<2, 2, 2, 2>(g, st);
  return launch_tile(gemm_tile(g.M, g.N, g.K), g, st);
}

// Measures the candidate tiles of an M x N x K product on `batch` scratch blocks (at most
// 512) and keeps the fastest for this device and shape; later products of that shape use
// it.  Every tile accumulates each entry over k in the same order, so the choice changes
// the time, not the result.  Allocates its scratch stream-ordered on `st` and synchronizes
// `st`; call it outside stream capture.
int exa_gemm_tune(int M, int N, int K, int batch, cudaStream_t st) {
  if (M <= 0 || N <= 1 || K <= 0 || (M <= 40 && N <= 40)) return EXA_OK;
  int dev = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_tune.count({dev, M, N, K})) return EXA_OK;
  }
  const int nb = std::max(1, std::min(batch, 512));
  const size_t sa = (size_t)M * K, sb = (size_t)K * N, sc = (size_t)M * N;
  double* buf = nullptr;
  EXA_CUDA(cudaMallocAsync((void**)&buf, sizeof(double) * (sa + sb + sc) * nb, st));
  // bytes 0x3f: every double is 4.8e-4, so no product overflows
  cudaError_t e = cudaMemsetAsync(buf, 0x3f, sizeof(double) * (sa + sb) * nb, st);
  GemmBatch g{M, N, K, 1.0, 0.0, buf, M, (long long)sa, 0, buf + sa * nb, K, (long long)sb, 0,
              buf + (sa + sb) * nb, M, (long long)sc, 0, nb, 1};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  int best = gemm_tile(M, N, K);
  float best_ms = -1.0f;
  for (int t = 0; t < kTiles && e == cudaSuccess; ++t) {
    if (launch_tile(t, g, st) != EXA_OK) break;  // warm
    e = cudaEventRecord(e0, st);
    for (int r = 0; r < 3 && e == cudaSuccess; ++r)
      if (launch_tile(t, g, st) != EXA_OK) e = cudaErrorUnknown;
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && (best_ms < 0 || ms < best_ms)) {
      best_ms = ms;
      best = t;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFreeAsync(buf, st);
  if (e != cudaSuccess) {
    exa_set_error("gemm tuning of %d x %d x %d: %s", M, N, K, cudaGetErrorString(e));
    return EXA_ERR_CUDA;
  }
  EXA_CUDA(cudaStreamSynchronize(st));
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[{dev, M, N, K}] = best;
  return EXA_OK;
}

int exa_gemm_tile_of(int M, int N, int K) { return gemm_tile(M, N, K); }

// ----------------------------------------------------------------------------------
// batched explicit inverse.  Exasim forms the explicit inverse of each element block
// with getrf + getri (backend/Common/pblas.h:163-260).  Here: Gauss-Jordan exchange
// steps with partial pivoting (pivot = largest magnitude among the rows not yet used,
// first on ties), the matrix held in registers.  Rows are never swapped physically; the
// pivot order is recorded and undone when the result is written, which gives the same
// pivots and arithmetic as swapping.  Each exchange at pivot (p, k), with d = 1/a_pk:
//   a_pk <- d,  a_pj <- a_pj d,  a_ik <- -a_ik d,  a_ij <- a_ij - a_ik (a_pj d).
// Both kernels below perform exactly these operations in this order, so they give the
// same bits for the same matrix.
// ----------------------------------------------------------------------------------
namespace {
constexpr int INV_MAX_N = 160;

template <typename T>
__device__ __forceinline__ T absval(T x) { return x < T(0) ? -x : x; }

// n <= 32: one warp per matrix, lane r holding row r.  The pivot search is a warp argmax,
// the pivot row reaches every lane by shuffles.  8 matrices per 256-thread CTA.
template <typename T>
__global__ void __launch_bounds__(256) inverse_warp_kernel(T* Aall, int n, long long stride, int batch, int* flag) {
  const int lane = threadIdx.x & 31;
  const long long mat = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
  if (mat >= batch) return;
  T* G = Aall + mat * stride;
  T a[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) a[j] = (lane < n && j < n) ? G[lane + (long long)n * j] : T(0);
  bool used = lane >= n;
  bool singular = false;
  int mystep = 0, myperm = 0;
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    if (k >= n) break;
    T best = used ? T(-1) : absval(a[k]);
    int bi = used ? n : lane;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const T ob = __shfl_xor_sync(0xffffffffu, best, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (!(best > T(0)) || bi >= n) {
      singular = true;
      const unsigned free_rows = __ballot_sync(0xffffffffu, !used);
      bi = free_rows ? __ffs(free_rows) - 1 : 0;
    }
    const int p = bi;
    const T d = T(1) / __shfl_sync(0xffffffffu, a[k], p);
    if (lane == p) { used = true; mystep = k; }
    if (lane == k) myperm = p;
    const T f = a[k];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const T rpd = __shfl_sync(0xffffffffu, a[j], p) * d;   // a_pj d
      if (lane == p) a[j] = (j == k) ? d : rpd;
      else a[j] = (j == k) ? -f * d : a[j] - f * rpd;
    }
  }
  if (singular && lane == 0) atomicExch(flag, 1);
  // entry (r, c) of the tableau is inverse(pos[r], perm[c]); pos[r] = the step of row r
#pragma unroll
  for (int c = 0; c < 32; ++c) {
    const int pc = __shfl_sync(0xffffffffu, myperm, c);
    if (c < n && lane < n) G[mystep + (long long)n * pc] = a[c];
  }
}

// 32 < n <= 16 RC: a CTA of 16 x TY threads; thread (tx, ty) owns rows ty + TY i (i < RR)
// and columns tx + 16 j (j < RC).  The pivot loop runs over column blocks kb (unrolled) and
// columns kt within them, so the register column of the pivot column is known at compile
// time.  Each step: the owners of column k publish it, every warp finds the pivot, the
// owners of the pivot row publish it scaled by d, every thread updates its entries.  The
// column and row buffers alternate between steps, so one barrier after each publication
// suffices.
template <typename T, int TY, int RR, int RC>
__global__ void __launch_bounds__(16 * TY, (sizeof(T) == 4 && TY == 16) ? 2 : 1)
    inverse_kernel(T* Aall, int n, long long stride, int* flag) {
  __shared__ T colk[2][INV_MAX_N];
  __shared__ T rowp[2][INV_MAX_N];
  __shared__ int perm[INV_MAX_N];   // perm[k] = pivot row of step k
  __shared__ int pos[INV_MAX_N];
  T* G = Aall + (long long)blockIdx.x * stride;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int lane = threadIdx.x & 31;
  T a[RR][RC];
#pragma unroll
  for (int i = 0; i < RR; ++i)
#pragma unroll
    for (int j = 0; j < RC; ++j) {
      const int r = ty + TY * i, c = tx + 16 * j;
      a[i][j] = (r < n && c < n) ? G[r + (long long)n * c] : T(0);
    }
  unsigned used = 0u;  // bit q: row lane + 32 q already pivoted (identical in every warp)
  bool singular = false;
  int step = 0;
#pragma unroll
  for (int kb = 0; kb < RC; ++kb) {
    for (int kt = 0; kt < 16; ++kt) {
      const int k = 16 * kb + kt;
      if (k >= n) break;
      const int buf = step & 1;
      ++step;
      if (tx == kt) {
#pragma unroll
        for (int i = 0; i < RR; ++i) {
          const int r = ty + TY * i;
          if (r < n) colk[buf][r] = a[i][kb];
        }
      }
      __syncthreads();
      T best = T(-1);
      int bi = n;
#pragma unroll
      for (int q = 0; q < (TY * RR + 31) / 32; ++q) {
        const int r = lane + 32 * q;
        if (r < n && !((used >> q) & 1u)) {
          const T v = absval(colk[buf][r]);
          if (v > best) { best = v; bi = r; }
        }
      }
      // a non-negative value orders as its bit pattern: the warp's largest |v| by 32-bit
      // reductions (for FP64 the high word, then the low word among lanes that tie on it),
      // and the lowest row holding it by one more: the choice of a shuffle tree that keeps
      // the larger value and, on ties, the lower row
      if constexpr (sizeof(T) == 4) {
        const unsigned key = bi < n ? __float_as_uint(best) : 0u;
        const unsigned mx = __reduce_max_sync(0xffffffffu, key);
        const unsigned mn = __reduce_min_sync(0xffffffffu, (bi < n && key == mx) ? (unsigned)bi : 0xffffffffu);
        best = __uint_as_float(mx);
        bi = mn == 0xffffffffu ? n : (int)mn;
      } else {
        const unsigned long long key = bi < n ? (unsigned long long)__double_as_longlong(best) : 0ull;
        const unsigned khi = (unsigned)(key >> 32), klo = (unsigned)key;
        const unsigned mhi = __reduce_max_sync(0xffffffffu, khi);
        const unsigned mlo = __reduce_max_sync(0xffffffffu, khi == mhi ? klo : 0u);
        const bool top = bi < n && khi == mhi && klo == mlo;
        const unsigned mn = __reduce_min_sync(0xffffffffu, top ? (unsigned)bi : 0xffffffffu);
        best = __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
        bi = mn == 0xffffffffu ? n : (int)mn;
      }
      if (!(best > T(0)) || bi >= n) {
        singular = true;
        // continue on the first unused row so the block still terminates
        bi = n;
        for (int r = 0; r < n; ++r) {
          const unsigned u = __shfl_sync(0xffffffffu, used, r & 31);
          if (!((u >> (r >> 5)) & 1u)) { bi = r; break; }
        }
        if (bi >= n) bi = 0;
      }
      const int p = bi;
      if (lane == (p & 31)) used |= 1u << (p >> 5);
      const T d = T(1) / colk[buf][p];
      if (threadIdx.x == 0) perm[k] = p;
      const int pa = p / TY, pt = p % TY;
      if (ty == pt) {
#pragma unroll
        for (int i = 0; i < RR; ++i)
          if (i == pa) {
#pragma unroll
            for (int j = 0; j < RC; ++j) {
              const int c = tx + 16 * j;
              const T v = (j == kb && tx == kt) ? d : a[i][j] * d;
              a[i][j] = v;
              if (c < n) rowp[buf][c] = v;
            }
          }
      }
      __syncthreads();
      T fv[RR], rv[RC];
      bool isp[RR];
#pragma unroll
      for (int i = 0; i < RR; ++i) {
        const int r = ty + TY * i;
        isp[i] = (r == p);
        fv[i] = (r < n && r != p) ? colk[buf][r] : T(0);
      }
#pragma unroll
      for (int j = 0; j < RC; ++j) {
        const int c = tx + 16 * j;
        rv[j] = (c < n) ? rowp[buf][c] : T(0);
      }
#pragma unroll
      for (int i = 0; i < RR; ++i)
#pragma unroll
        for (int j = 0; j < RC; ++j) {
          if (j == kb) {
            // column k: -a_ik d off the pivot row (the pivot row holds d already)
            if (tx == kt) { if (!isp[i]) a[i][j] = -fv[i] * d; }
            else a[i][j] = a[i][j] - fv[i] * rv[j];
          } else {
            a[i][j] = a[i][j] - fv[i] * rv[j];
          }
        }
    }
  }
  if (singular && threadIdx.x == 0) atomicExch(flag, 1);
  __syncthreads();
  for (int t = threadIdx.x; t < n; t += blockDim.x) pos[perm[t]] = t;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < RR; ++i)
#pragma unroll
    for (int j = 0; j < RC; ++j) {
      const int r = ty + TY * i, c = tx + 16 * j;
      if (r < n && c < n) G[pos[r] + (long long)n * perm[c]] = a[i][j];
    }
}

// 32 < n <= 128: columns by warp.  Warp w owns columns w + NW j (j < CW) of every row, lane l
// rows l + 32 i (i < RL), so column k = NW jk + w lies in one warp: the pivot search is a warp
// argmax on registers, and the pivot row reaches each warp's lanes by shuffles from the lane
// that holds it.  Per step the column's warp publishes the column, the pivot row index and its
// reciprocal in shared memory (two buffers, alternating), and one barrier separates that from
// the update.  The arithmetic per entry is the same as in inverse_kernel (a_pj d for the pivot
// row, d and -a_ik d in column k, a_ij - a_ik (a_pj d) elsewhere) with the same pivot choice, so
// every shape (NW, CW, RL) and inverse_kernel give the same bits.
template <typename T>
__device__ __forceinline__ void warp_argmax(T best, int bi, int n, T& mbest, int& mbi) {
  // a non-negative value orders as its bit pattern: the warp's largest |v|, and the lowest
  // row holding it (for FP64 the high word, then the low word among lanes that tie on it)
  if constexpr (sizeof(T) == 4) {
    const unsigned key = bi < n ? __float_as_uint(best) : 0u;
    const unsigned mx = __reduce_max_sync(0xffffffffu, key);
    const unsigned mn = __reduce_min_sync(0xffffffffu, (bi < n && key == mx) ? (unsigned)bi : 0xffffffffu);
    mbest = __uint_as_float(mx);
    mbi = mn == 0xffffffffu ? n : (int)mn;
  } else {
    const unsigned long long key = bi < n ? (unsigned long long)__double_as_longlong(best) : 0ull;
    const unsigned khi = (unsigned)(key >> 32), klo = (unsigned)key;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, khi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, khi == mhi ? klo : 0u);
    const bool top = bi < n && khi == mhi && klo == mlo;
    const unsigned mn = __reduce_min_sync(0xffffffffu, top ? (unsigned)bi : 0xffffffffu);
    mbest = __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
    mbi = mn == 0xffffffffu ? n : (int)mn;
  }
}

template <typename T, int NW, int CW, int RL>
__global__ void __launch_bounds__(32 * NW, sizeof(T) == 4 ? 2 : 1)
    inverse_wcol_kernel(T* Aall, int n, long long stride, int* flag) {
  __shared__ T colb[2][32 * RL];
  __shared__ int sp[2];
  __shared__ T sd[2];
  __shared__ int perm[32 * RL];
  __shared__ int pos[32 * RL];
  __shared__ __align__(16) T rowb[NW][CW];  // each warp's part of the pivot row
  static_assert((CW * sizeof(T)) % 16 == 0, "pivot-row copies in 16-byte vectors");
  T* G = Aall + (long long)blockIdx.x * stride;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T a[RL][CW];
#pragma unroll
  for (int i = 0; i < RL; ++i)
#pragma unroll
    for (int j = 0; j < CW; ++j) {
      const int r = lane + 32 * i, c = warp + NW * j;
      a[i][j] = (r < n && c < n) ? G[r + (long long)n * c] : T(0);
    }
  unsigned used = 0u;  // bit i: row lane + 32 i already pivoted (the same in every warp)
  bool singular = false;
  int step = 0;
#pragma unroll
  for (int jk = 0; jk < CW; ++jk) {
    for (int wk = 0; wk < NW; ++wk) {
      const int k = NW * jk + wk;
      if (k >= n) break;
      const int buf = step & 1;
      ++step;
      if (warp == wk) {
        // the pivot: largest |a_rk| over the rows not yet pivoted, lowest row on ties
        T best = T(-1);
        int bi = n;
#pragma unroll
        for (int i = 0; i < RL; ++i) {
          const int r = lane + 32 * i;
          if (r < n && !((used >> i) & 1u)) {
            const T v = fabs(a[i][jk]);  // fabsf for float: the compare takes |x| as an operand
            if (v > best) { best = v; bi = r; }
          }
        }
        {
          T mb;
          int mi;
          warp_argmax(best, bi, n, mb, mi);
          best = mb;
          bi = mi;
        }
        if (!(best > T(0)) || bi >= n) {
          singular = true;
          // continue on the first unused row so the block still terminates
          bi = n;
          for (int r = 0; r < n; ++r) {
            const unsigned u = __shfl_sync(0xffffffffu, used, r & 31);
            if (!((u >> (r >> 5)) & 1u)) { bi = r; break; }
          }
          if (bi >= n) bi = 0;
        }
        const int pi = bi >> 5;
        T own = a[0][jk];
#pragma unroll
        for (int i = 1; i < RL; ++i)
          if (i == pi) own = a[i][jk];
        const T apk = __shfl_sync(0xffffffffu, own, bi & 31);
#pragma unroll
        for (int i = 0; i < RL; ++i) colb[buf][lane + 32 * i] = a[i][jk];
        if (lane == 0) {
          sp[buf] = bi;
          sd[buf] = T(1) / apk;
          perm[k] = bi;
        }
      }
      __syncthreads();
      const int p = sp[buf];
      const T d = sd[buf];
      const int pl = p & 31, pi = p >> 5;
      if (lane == pl) used |= 1u << pi;
      T f[RL];
#pragma unroll
      for (int i = 0; i < RL; ++i) f[i] = (lane + 32 * i == p) ? T(0) : colb[buf][lane + 32 * i];
      // this warp's part of the pivot row, scaled: r_j = a_pj d.  The lane that holds row p
      // stores it (one branch of RL, taken by one lane), the warp reads it back as broadcasts
      if (lane == pl) {
#pragma unroll
        for (int i = 0; i < RL; ++i)
          if (i == pi) {
#pragma unroll
            for (int j = 0; j < CW; j += 16 / (int)sizeof(T)) {
              if constexpr (sizeof(T) == 4)
                *reinterpret_cast<float4*>(&rowb[warp][j]) = make_float4(a[i][j], a[i][j + 1], a[i][j + 2], a[i][j + 3]);
              else
                *reinterpret_cast<double2*>(&rowb[warp][j]) = make_double2(a[i][j], a[i][j + 1]);
            }
          }
      }
      __syncwarp();
      T r[CW];
#pragma unroll
      for (int j = 0; j < CW; j += 16 / (int)sizeof(T)) {
        if constexpr (sizeof(T) == 4) {
          const float4 v = *reinterpret_cast<const float4*>(&rowb[warp][j]);
          r[j] = v.x * d;
          r[j + 1] = v.y * d;
          r[j + 2] = v.z * d;
          r[j + 3] = v.w * d;
        } else {
          const double2 v = *reinterpret_cast<const double2*>(&rowb[warp][j]);
          r[j] = v.x * d;
          r[j + 1] = v.y * d;
        }
      }
      // rows other than p (f_p = 0 leaves row p as it is), then row p and column k
#pragma unroll
      for (int i = 0; i < RL; ++i)
#pragma unroll
        for (int j = 0; j < CW; ++j) a[i][j] = a[i][j] - f[i] * r[j];
      if (warp == wk) {
#pragma unroll
        for (int i = 0; i < RL; ++i) a[i][jk] = -f[i] * d;
      }
      if (lane == pl) {
#pragma unroll
        for (int i = 0; i < RL; ++i)
          if (i == pi) {
#pragma unroll
            for (int j = 0; j < CW; ++j) a[i][j] = r[j];
            if (warp == wk) a[i][jk] = d;
          }
      }
    }
  }
  if (singular && lane == 0) atomicExch(flag, 1);
  __syncthreads();
  for (int t = threadIdx.x; t < n; t += blockDim.x) pos[perm[t]] = t;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < RL; ++i)
#pragma unroll
    for (int j = 0; j < CW; ++j) {
      const int r = lane + 32 * i, c = warp + NW * j;
      if (r < n && c < n) G[pos[r] + (long long)n * perm[c]] = a[i][j];
    }
}

// The column-by-warp shapes: warps x columns per warp x rows per lane.  Variants 0-1 hold up
// to 128 rows and columns, 2-3 up to 64.  exa_inverse_tune times them per order and type.
constexpr int kInvVariants = 4;
__host__ __device__ constexpr int inv_variant_nmax(int v) { return v < 2 ? 128 : 64; }

template <typename T>
int launch_wcol(int v, T* A, int n, long long stride, int batch, int* d_flag, cudaStream_t st) {
  switch (v) {
    case 0: inverse_wcol_kernel<T, 8, 16, 4><<<batch, 256, 0, st>>>(A, n, stride, d_flag); break;
    case 1: inverse_wcol_kernel<T, 16, 8, 4><<<batch, 512, 0, st>>>(A, n, stride, d_flag); break;
    case 2: inverse_wcol_kernel<T, 4, 16, 2><<<batch, 128, 0, st>>>(A, n, stride, d_flag); break;
    default: inverse_wcol_kernel<T, 8, 8, 2><<<batch, 256, 0, st>>>(A, n, stride, d_flag); break;
  }
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

std::mutex g_inv_mu;
std::map<std::array<int, 3>, int> g_inv_tune;  // (device, n, fp64) -> measured fastest variant

// the measured variant for this order and type, else the default: FP32 8 warps x 16 columns
// (4 warps up to 64), FP64 16 warps x 8 columns (8 x 8 up to 64)
int inv_variant(int n, bool fp64) {
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) {
    std::lock_guard<std::mutex> lk(g_inv_mu);
    auto it = g_inv_tune.find({dev, n, fp64 ? 1 : 0});
    if (it != g_inv_tune.end()) return it->second;
  }
  if (fp64) return n <= 64 ? 3 : 1;
  return n <= 64 ? 2 : 0;
}

template <typename T, int TY, int RR, int RC>
int launch_inverse(T* A, int n, long long stride, int batch, int* d_flag, cudaStream_t st) {
  static_assert(TY * RR <= INV_MAX_N + 31 && 16 * RC <= INV_MAX_N, "inverse tile exceeds the buffers");
  inverse_kernel<T, TY, RR, RC><<<batch, 16 * TY, 0, st>>>(A, n, stride, d_flag);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

template <typename T>
int inverse_dispatch(T* A, int n, long long stride, int batch, int* d_flag, cudaStream_t st) {
  if (batch <= 0) return EXA_OK;
  if (n > INV_MAX_N || n <= 0) {
    exa_set_error("dense inverse of order %d exceeds the register kernel limit %d", n, INV_MAX_N);
    return EXA_ERR_UNSUPPORTED;
  }
  if (n <= 32) {
    for (int b0 = 0; b0 < batch; b0 += 8 * 65535) {
      const int nb = (batch - b0 < 8 * 65535) ? batch - b0 : 8 * 65535;
      inverse_warp_kernel<T><<<exa_ceil_div(nb, 8), 256, 0, st>>>(A + (long long)b0 * stride, n, stride, nb, d_flag);
      EXA_LAUNCH_CHECK();
    }
    return EXA_OK;
  }
  const int rc = (n + 15) / 16;
  // FP32 blocks up to 128: 256 threads with 8 x 8 entries each, two CTAs per SM
  if (n <= 128) return launch_wcol<T>(inv_variant(n, sizeof(T) == 8), A, n, stride, batch, d_flag, st);
  const int rr = (n + 31) / 32;
  if (rr <= 2 && rc <= 4) return launch_inverse<T, 32, 2, 4>(A, n, stride, batch, d_flag, st);
  if (rr <= 2 && rc <= 6) return launch_inverse<T, 32, 2, 6>(A, n, stride, batch, d_flag, st);
  if (rr <= 3 && rc <= 6) return launch_inverse<T, 32, 3, 6>(A, n, stride, batch, d_flag, st);
  if (rr <= 4 && rc <= 8) return launch_inverse<T, 32, 4, 8>(A, n, stride, batch, d_flag, st);
  return launch_inverse<T, 32, 5, 10>(A, n, stride, batch, d_flag, st);
}
}  // namespace

int exa_inverse(double* A, int n, long long stride, int batch, int* d_flag, cudaStream_t st) {
  return inverse_dispatch(A, n, stride, batch, d_flag, st);
}

int exa_inverse(float* A, int n, long long stride, int batch, int* d_flag, cudaStream_t st) {
  return inverse_dispatch(A, n, stride, batch, d_flag, st);
}

namespace {
// scratch blocks for timing: hashed values uniform in [-1, 1), so partial pivoting permutes
// the rows as it does on element blocks (and the final store is scattered as there)
template <typename T>
__global__ void inv_tune_fill_kernel(T* A, int n, long long total) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    unsigned long long z = (unsigned long long)t * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    A[t] = T((double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0);
  }
}

template <typename T>
int inverse_tune(int n, int batch, cudaStream_t st) {
  int dev = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  const std::array<int, 3> key{dev, n, sizeof(T) == 8 ? 1 : 0};
  {
    std::lock_guard<std::mutex> lk(g_inv_mu);
    if (g_inv_tune.count(key)) return EXA_OK;
  }
  // as many blocks as the caller inverts (up to 4096): fewer fit in L2 and would time the
  // shapes on cached data
  const int nb = std::max(1, std::min(batch, 4096));
  const long long total = (long long)n * n * nb;
  T* buf = nullptr;
  if (cudaMallocAsync((void**)&buf, sizeof(T) * total + 16, st) != cudaSuccess) {
    cudaGetLastError();  // no room for scratch: keep the default shape
    return EXA_OK;
  }
  int* flag = reinterpret_cast<int*>(buf + total);  // the timing runs' own singular flag
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  int best = inv_variant(n, sizeof(T) == 8);
  float best_ms = -1.0f;
  for (int v = 0; v < kInvVariants && e == cudaSuccess; ++v) {
    if (n > inv_variant_nmax(v)) continue;
    inv_tune_fill_kernel<T><<<1024, 256, 0, st>>>(buf, n, total);
    if (launch_wcol<T>(v, buf, n, (long long)n * n, nb, flag, st) != EXA_OK) break;  // warm
    e = cudaEventRecord(e0, st);
    for (int r = 0; r < 3 && e == cudaSuccess; ++r)
      if (launch_wcol<T>(v, buf, n, (long long)n * n, nb, flag, st) != EXA_OK) e = cudaErrorUnknown;
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && (best_ms < 0 || ms < best_ms)) {
      best_ms = ms;
      best = v;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFreeAsync(buf, st);
  if (e != cudaSuccess) {
    exa_set_error("inverse tuning of order %d: %s", n, cudaGetErrorString(e));
    return EXA_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(g_inv_mu);
  g_inv_tune[key] = best;
  return EXA_OK;
}
}  // namespace

int exa_inverse_variant_of(int n, int fp64) { return n > 32 && n <= 128 ? inv_variant(n, fp64 != 0) : -1; }

int exa_inverse_tune(int n, int batch, int fp64, cudaStream_t st) {
  if (n <= 32 || n > 128 || batch <= 0) return EXA_OK;
  return fp64 ? inverse_tune<double>(n, batch, st) : inverse_tune<float>(n, batch, st);
}

// ----------------------------------------------------------------------------------
// blocked inverse for INV_MAX_N < n <= 2 INV_MAX_N (e.g. 320 x 320 blocks of 3D Euler at
// p = 3), by the 2 x 2 block formula with n1 = n/2 rounded up and n2 = n - n1:
//   X = A11^-1 (Gauss-Jordan, pivoting within the block), W1 = X A12, S = A22 - A21 W1,
//   Y = S^-1, W3 = A21 X;  inverse = [X + W1 Y W3, -W1 Y; -Y W3, Y].
// The products run on the FP64 DMMA GEMM (or an FP32 SIMT GEMM for the FP32 blocks).
// Workspace: n^2 entries per matrix.
// ----------------------------------------------------------------------------------
namespace {
// C(r, c) = alpha sum_k A(r, k) B(k, c) + beta C(r, c), one batch entry per blockIdx.y;
// 64 x 64 tiles, 256 threads with 4 x 4 outputs each, K in steps of 16 through shared memory
template <typename T>
__global__ void __launch_bounds__(256) simt_gemm_kernel(int M, int N, int K, T alpha, T beta, const T* A,
                                                        long long lda, long long sA, const T* B, long long ldb,
                                                        long long sB, T* C, long long ldc, long long sC) {
  __shared__ T as[16][65], bs[16][65];
  const long long b = blockIdx.y;
  A += b * sA;
  B += b * sB;
  C += b * sC;
  const int tilesM = (M + 63) / 64;
  const int r0 = (blockIdx.x % tilesM) * 64, c0 = (blockIdx.x / tilesM) * 64;
  const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
  T acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int t = threadIdx.x; t < 16 * 64; t += 256) {
      const int kk = t >> 6, rr = t & 63;
      as[kk][rr] = (r0 + rr < M && k0 + kk < K) ? A[(r0 + rr) + lda * (k0 + kk)] : T(0);
      bs[kk][rr] = (c0 + rr < N && k0 + kk < K) ? B[(k0 + kk) + ldb * (c0 + rr)] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      T av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = as[kk][tr + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = bs[kk][tc + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += av[i] * bv[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = r0 + tr + 16 * i, c = c0 + tc + 16 * j;
      if (r < M && c < N) {
        T* p = C + r + ldc * c;
        *p = (beta == T(0)) ? alpha * acc[i][j] : alpha * acc[i][j] + beta * (*p);
      }
    }
}

// batched sub-matrix copy: dst(r, c) = src(r, c) for r < R, c < Cn
template <typename T>
__global__ void submat_copy_kernel(T* dst, long long ldd, long long sd, const T* src, long long lds, long long ss,
                                   int R, int Cn) {
  const long long b = blockIdx.y;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < R * Cn; t += gridDim.x * blockDim.x) {
    const int r = t % R, c = t / R;
    dst[b * sd + r + ldd * c] = src[b * ss + r + lds * c];
  }
}

template <typename T>
int bgemm(int M, int N, int K, T alpha, T beta, const T* A, long long lda, long long sA, const T* B, long long ldb,
          long long sB, T* C, long long ldc, long long sC, int batch, cudaStream_t st) {
  if constexpr (sizeof(T) == 8) {
    GemmBatch g{M, N, K, alpha, beta, A, lda, sA, 0, B, ldb, sB, 0, C, ldc, sC, 0, batch, 1};
    return exa_gemm(g, st);
  } else {
    for (int b0 = 0; b0 < batch; b0 += 65535) {
      const int nb = (batch - b0 < 65535) ? batch - b0 : 65535;
      dim3 grid((unsigned)(exa_ceil_div(M, 64) * exa_ceil_div(N, 64)), (unsigned)nb);
      simt_gemm_kernel<T><<<grid, 256, 0, st>>>(M, N, K, alpha, beta, A + b0 * sA, lda, sA, B + b0 * sB, ldb, sB,
                                                C + b0 * sC, ldc, sC);
      EXA_LAUNCH_CHECK();
    }
    return EXA_OK;
  }
}

template <typename T>
int subcopy(T* dst, long long ldd, long long sd, const T* src, long long lds, long long ss, int R, int Cn, int batch,
            cudaStream_t st) {
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    const int nb = (batch - b0 < 65535) ? batch - b0 : 65535;
    dim3 grid((unsigned)exa_ceil_div(R * Cn, 256 * 4), (unsigned)nb);
    submat_copy_kernel<T><<<grid, 256, 0, st>>>(dst + b0 * sd, ldd, sd, src + b0 * ss, lds, ss, R, Cn);
    EXA_LAUNCH_CHECK();
  }
  return EXA_OK;
}

template <typename T>
int inverse_blocked(T* A, int n, long long stride, int batch, T* ws, int* d_flag, cudaStream_t st) {
  const int n1 = (n + 1) / 2, n2 = n - n1;
  const long long sw = (long long)n * n;
  T* W0 = ws;                                  // n1 x n1: A11, then X
  T* W1 = W0 + (long long)n1 * n1;             // n1 x n2: X A12
  T* W2 = W1 + (long long)n1 * n2;             // n2 x n2: S, then Y
  T* W3 = W2 + (long long)n2 * n2;             // n2 x n1: A21 X
  T* A11 = A;
  T* A21 = A + n1;
  T* A12 = A + (long long)n * n1;
  T* A22 = A + n1 + (long long)n * n1;
  EXA_TRY(subcopy<T>(W0, n1, sw, A11, n, stride, n1, n1, batch, st));
  EXA_TRY(inverse_dispatch<T>(W0, n1, sw, batch, d_flag, st));
  EXA_TRY(bgemm<T>(n1, n2, n1, T(1), T(0), W0, n1, sw, A12, n, stride, W1, n1, sw, batch, st));
  EXA_TRY(bgemm<T>(n2, n2, n1, T(-1), T(1), A21, n, stride, W1, n1, sw, A22, n, stride, batch, st));
  EXA_TRY(subcopy<T>(W2, n2, sw, A22, n, stride, n2, n2, batch, st));
  EXA_TRY(inverse_dispatch<T>(W2, n2, sw, batch, d_flag, st));
  EXA_TRY(bgemm<T>(n2, n1, n1, T(1), T(0), A21, n, stride, W0, n1, sw, W3, n2, sw, batch, st));
  EXA_TRY(bgemm<T>(n1, n2, n2, T(-1), T(0), W1, n1, sw, W2, n2, sw, A12, n, stride, batch, st));
  EXA_TRY(subcopy<T>(A11, n, stride, W0, n1, sw, n1, n1, batch, st));
  EXA_TRY(bgemm<T>(n1, n1, n2, T(-1), T(1), A12, n, stride, W3, n2, sw, A11, n, stride, batch, st));
  EXA_TRY(bgemm<T>(n2, n1, n2, T(-1), T(0), W2, n2, sw, W3, n2, sw, A21, n, stride, batch, st));
  EXA_TRY(subcopy<T>(A22, n, stride, W2, n2, sw, n2, n2, batch, st));
  return EXA_OK;
}

template <typename T>
int inverse_ws(T* A, int n, long long stride, int batch, T* ws, int* d_flag, cudaStream_t st) {
  if (n <= INV_MAX_N || batch <= 0) return inverse_dispatch<T>(A, n, stride, batch, d_flag, st);
  if (n > 2 * INV_MAX_N) {
    exa_set_error("dense inverse of order %d exceeds the blocked kernel limit %d", n, 2 * INV_MAX_N);
    return EXA_ERR_UNSUPPORTED;
  }
  if (!ws) {
    exa_set_error("dense inverse of order %d needs a workspace of n^2 entries per matrix", n);
    return EXA_ERR_ARG;
  }
  return inverse_blocked<T>(A, n, stride, batch, ws, d_flag, st);
}
}  // namespace

// ----------------------------------------------------------------------------------
// The same 2 x 2 block inverse for FP32 blocks with the five products on the tcgen05
// 3xTF32 GEMM (the mixed-precision form), for orders above the register kernel's limit,
// applied recursively: the two diagonal inverses are themselves blocked until their order
// is at most INV_TC_LEAF, where the register kernel takes over.  At order 320 (3D Euler,
// p = 3) leaves of 80 (two levels) took 134 ms per solve of 32^3 elements against 161 ms
// for leaves of 160 and 168 ms for leaves of 40; at 125 the register kernel alone beat one
// level with leaves of 63 (2.6 against 2.8 ms for 4096 blocks).  With
// X = A11^-1 and Y = S^-1:
//   W1 = X A12, S = A22 - A21 W1, W3 = A21 X,
//   A12 <- -W1 Y, A11 <- X - A12 W3, A21 <- -Y W3, A22 <- Y.
// W1 and W3 exist only packed: the products that make them write their packed copies
// (A and B operand layouts) from the epilogue.  Per level the packed operands take seven
// slots of hi and lo parts per matrix; X as A and A12 as B are dead once W1 exists, and
// W1 as B once S does, so Y (A and B) and the new A12 (A) take their slots.  Per matrix,
// level L keeps X and Y (n1^2 + n2^2 floats) and its slots in ws and pk after those of the
// levels above it; the two inner inversions of a level run one after the other and share
// the next level's space.
// ----------------------------------------------------------------------------------
namespace {
constexpr int INV_TC_LEAF = 96;

long long inv_tc_slot(int n) {
  const int n1 = (n + 1) / 2;
  return exa_pack_size(n1, n1);  // every operand of a level has at most n1 rows and n1 k
}

long long inv_tc_ws(int n) {
  if (n <= INV_TC_LEAF) return 0;
  const long long n1 = (n + 1) / 2, n2 = n - n1;
  return n1 * n1 + n2 * n2 + inv_tc_ws((int)n1);
}

long long inv_tc_pk(int n) { return n <= INV_TC_LEAF ? 0 : 14 * inv_tc_slot(n) + inv_tc_pk((n + 1) / 2); }

// A: batch n x n blocks (leading dimension n) `stride` floats apart; ws and pk: this level's
// part of the workspaces, wstride and pstride floats per matrix
int inverse_tc32_level(float* A, int n, long long stride, int batch, float* ws, long long wstride, float* pk,
                       long long pstride, int* d_flag, int* uflag, cudaStream_t st) {
  if (n <= INV_TC_LEAF) return inverse_dispatch<float>(A, n, stride, batch, d_flag, st);
  const int n1 = (n + 1) / 2, n2 = n - n1;
  const long long S = inv_tc_slot(n);
  float* W0 = ws;                       // n1 x n1: A11, then X
  float* W2 = W0 + (long long)n1 * n1;  // n2 x n2: S, then Y
  float* wsi = W2 + (long long)n2 * n2;  // the inner levels
  float* pki = pk + 14 * S;
  float* A11 = A;
  float* A21 = A + n1;
  float* A12 = A + (long long)n * n1;
  float* A22 = A + n1 + (long long)n * n1;
  // slot k: hi at pk + 2kS, lo at pk + (2k+1)S
  auto op = [&](int k, int R, int K, bool as_b) {
    UPacked u{};
    u.hi = pk + 2LL * k * S;
    u.lo = u.hi + S;
    u.sb = pstride;
    u.sb2 = 0;
    u.R = R;
    u.K = K;
    u.TR = as_b ? (R + 15) / 16 * 16 : 128;  // a B operand is one tile of all its rows
    return u;
  };
  const UPacked Xa = op(0, n1, n1, false), A12b = op(1, n2, n1, true), W1b = op(2, n2, n1, true);
  const UPacked Xb = op(3, n1, n1, true), A21a = op(4, n2, n1, false), W1a = op(5, n1, n2, false);
  const UPacked W3b = op(6, n1, n2, true);
  const UPacked Ya = op(0, n2, n2, false), Yb = op(1, n2, n2, true), A12a = op(2, n1, n2, false);
  auto gemm = [&](int M, int N, int K, double alpha, const UPacked& Aop, const UPacked& Bop, double beta,
                  const float* Cin, long long ldci, long long sci, float* C, long long ldc, long long sc,
                  std::initializer_list<UPackOut> outs) {
    UGemmP g{};
    g.M = M; g.N = N; g.K = K; g.alpha = alpha; g.beta = beta;
    g.A = Aop; g.B = Bop;
    g.Cin = Cin; g.tci = EXA_T_F32; g.ldci = ldci; g.sCi = sci;
    g.C = C; g.tco = EXA_T_F32; g.ldc = ldc; g.sC = sc;
    g.nout = 0;
    for (const UPackOut& o : outs) g.out[g.nout++] = o;
    g.batch = batch; g.batch2 = 1;
    return exa_gemm_3xtf32(g, uflag, st);
  };
  // the packs write every entry of an operand, padding included; the products' packed
  // outputs write only the rows and k of the product, so where halves are not multiples of
  // 16 the slots they write are cleared first (a slot may hold another shape's entries)
  const bool padded = (n1 % 16) != 0 || (n2 % 16) != 0;
  auto clear = [&](int k) -> cudaError_t {
    if (!padded) return cudaSuccess;
    return cudaMemset2DAsync(pk + 2LL * k * S, sizeof(float) * (size_t)pstride, 0, sizeof(float) * 2 * (size_t)S,
                             (size_t)batch, st);
  };
  EXA_TRY(subcopy<float>(W0, n1, wstride, A11, n, stride, n1, n1, batch, st));
  EXA_TRY(inverse_tc32_level(W0, n1, wstride, batch, wsi, wstride, pki, pstride, d_flag, uflag, st));
  EXA_TRY(exa_pack(W0, 0, 1, n1, wstride, 0, batch, 1, Xa, st));
  EXA_TRY(exa_pack(W0, 0, n1, 1, wstride, 0, batch, 1, Xb, st));
  EXA_TRY(exa_pack(A12, 0, n, 1, stride, 0, batch, 1, A12b, st));
  EXA_TRY(exa_pack(A21, 0, 1, n, stride, 0, batch, 1, A21a, st));
  // W1 = X A12 (packed as A and as B only)
  EXA_CUDA(clear(2));
  EXA_CUDA(clear(5));
  EXA_TRY(gemm(n1, n2, n1, 1.0, Xa, A12b, 0.0, nullptr, 0, 0, nullptr, 0, 0,
               {UPackOut{W1a, 0, 1, 0}, UPackOut{W1b, 1, 1, 0}}));
  // S = A22 - A21 W1, in place
  EXA_TRY(gemm(n2, n2, n1, -1.0, A21a, W1b, 1.0, A22, n, stride, A22, n, stride, {}));
  EXA_TRY(subcopy<float>(W2, n2, wstride, A22, n, stride, n2, n2, batch, st));
  EXA_TRY(inverse_tc32_level(W2, n2, wstride, batch, wsi, wstride, pki, pstride, d_flag, uflag, st));
  EXA_TRY(exa_pack(W2, 0, 1, n2, wstride, 0, batch, 1, Ya, st));
  EXA_TRY(exa_pack(W2, 0, n2, 1, wstride, 0, batch, 1, Yb, st));
  // W3 = A21 X (packed as B only)
  EXA_CUDA(clear(6));
  EXA_TRY(gemm(n2, n1, n1, 1.0, A21a, Xb, 0.0, nullptr, 0, 0, nullptr, 0, 0, {UPackOut{W3b, 1, 1, 0}}));
  // A12 = -W1 Y (and packed as A)
  EXA_CUDA(clear(2));
  EXA_TRY(gemm(n1, n2, n2, -1.0, W1a, Yb, 0.0, nullptr, 0, 0, A12, n, stride, {UPackOut{A12a, 0, 1, 0}}));
  // A11 = X - A12 W3
  EXA_TRY(gemm(n1, n1, n2, -1.0, A12a, W3b, 1.0, W0, n1, wstride, A11, n, stride, {}));
  // A21 = -Y W3
  EXA_TRY(gemm(n2, n1, n2, -1.0, Ya, W3b, 0.0, nullptr, 0, 0, A21, n, stride, {}));
  EXA_TRY(subcopy<float>(A22, n, stride, W2, n2, wstride, n2, n2, batch, st));
  return EXA_OK;
}
}  // namespace

long long exa_inverse_tc32_ws(int n) { return n <= INV_MAX_N ? 0 : inv_tc_ws(n); }
long long exa_inverse_tc32_pk(int n) { return n <= INV_MAX_N ? 0 : inv_tc_pk(n); }

int exa_inverse_tc32(float* A, int n, long long stride, int batch, float* ws, float* pk, int* d_flag, int* uflag,
                     cudaStream_t st) {
  if (n <= INV_MAX_N || batch <= 0) return inverse_dispatch<float>(A, n, stride, batch, d_flag, st);
  if (n > 2 * INV_MAX_N) {
    exa_set_error("dense inverse of order %d exceeds the blocked kernel limit %d", n, 2 * INV_MAX_N);
    return EXA_ERR_UNSUPPORTED;
  }
  if (!ws || !pk) {
    exa_set_error("tensor-core inverse of order %d needs workspaces", n);
    return EXA_ERR_ARG;
  }
  return inverse_tc32_level(A, n, stride, batch, ws, inv_tc_ws(n), pk, inv_tc_pk(n), d_flag, uflag, st);
}

int exa_inverse_max_n() { return 2 * INV_MAX_N; }
int exa_inverse_needs_ws(int n) { return n > INV_MAX_N; }

int exa_inverse_ws(double* A, int n, long long stride, int batch, double* ws, int* d_flag, cudaStream_t st) {
  return inverse_ws<double>(A, n, stride, batch, ws, d_flag, st);
}

int exa_inverse_ws(float* A, int n, long long stride, int batch, float* ws, int* d_flag, cudaStream_t st) {
  return inverse_ws<float>(A, n, stride, batch, ws, d_flag, st);
}

// ----------------------------------------------------------------------------------
// vector kernels.  A vector of n entries runs on vec_grid(n) blocks (one entry per thread,
// at most VB = two blocks per SM) with a grid-stride loop; each reduction leaves one partial
// sum per block, which the consumer kernel adds up in index order, so results do not depend
// on scheduling.
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

// Vectors of n entries run on vec_grid(n) blocks, one entry per thread up to VB blocks:
// short vectors (a small mesh's trace space) occupy a few SMs instead of the whole GPU,
// which leaves room for other contexts' kernels (on the served stream this was faster both
// for one solve at a time and for 16 overlapping solves than a fixed VB blocks, and than
// four entries per thread).  The count depends on n alone, so every reduction over the
// same n takes the same partition and order.
inline int vec_grid(long long n) {
  const long long b = (n + VT - 1) / VT;
  return (int)(b < 1 ? 1 : (b > VB ? VB : b));
}

// every block reduces the first nb partials in the same order (thread-parallel, then fixed tree)
__device__ __forceinline__ double sum_partials_n(const double* part, int nb) {
  __shared__ double tot_n;
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += VT) v += part[i];
  double s = block_sum(v);
  if (threadIdx.x == 0) tot_n = s;
  __syncthreads();
  return tot_n;
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
  // four strides' loads in flight, summed in the order of one stride at a time
  const long long stride = (long long)gridDim.x * VT;
  long long i = blockIdx.x * (long long)VT + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {
    double a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[u] = x[i + u * stride];
      b[u] = y[i + u * stride];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) v = fma(a[u], b[u], v);
  }
  for (; i < n; i += stride) v = fma(x[i], y[i], v);
  double s = block_sum(v);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(VT) reduce_kernel(const double* part, int nb, double* out, int take_sqrt) {
  double s = sum_partials_n(part, nb);
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
  const double h = sum_partials_n(part_in, gridDim.x);
  if (blockIdx.x == 0 && threadIdx.x == 0) *h_out = h;
  double v = 0.0;
  // the basis vectors stream through (evict-first loads), so a vector being orthogonalised
  // that fits in L2 stays there across the steps of its Gram-Schmidt sweep.  Four strides'
  // loads are issued before their updates (long vectors need the loads in flight); the
  // products are summed in the same order as one stride at a time.
  const long long stride = (long long)gridDim.x * VT;
  long long i = blockIdx.x * (long long)VT + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {
    double ww[4], p[4], q[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      ww[u] = w[i + u * stride];
      p[u] = __ldcs(vprev + i + u * stride);
      q[u] = vnext ? __ldcs(vnext + i + u * stride) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double wi = ww[u] - h * p[u];
      w[i + u * stride] = wi;
      v = fma(wi, vnext ? q[u] : wi, v);
    }
  }
  for (; i < n; i += stride) {
    double wi = w[i] - h * __ldcs(vprev + i);
    w[i] = wi;
    v = fma(wi, vnext ? __ldcs(vnext + i) : wi, v);
  }
  double s = block_sum(v);
  if (threadIdx.x == 0) part_out[blockIdx.x] = s;
}

__global__ void __launch_bounds__(VT) mgs_finish_kernel(double* vout, const double* w, const double* part_in,
                                                        double* h_out, long long n) {
  const double h = sqrt(sum_partials_n(part_in, gridDim.x));
  if (blockIdx.x == 0 && threadIdx.x == 0) *h_out = h;
  const double r = 1.0 / h;
  const long long stride = (long long)gridDim.x * VT;
  long long i = blockIdx.x * (long long)VT + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {
    double a[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) a[u] = w[i + u * stride];
#pragma unroll
    for (int u = 0; u < 4; ++u) vout[i + u * stride] = a[u] * r;
  }
  for (; i < n; i += stride) vout[i] = w[i] * r;
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
    for (long long i = blockIdx.x * (long long)VT + threadIdx.x; i < n; i += (long long)gridDim.x * VT)
      v = fma(V[i + n * j], w[i], v);
    double s = block_sum(v);
    if (threadIdx.x == 0) part[j * VB + blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(VT) multi_reduce_kernel(const double* part, double* h, int k, int nb) {
  for (int j = 0; j < k; ++j) {
    double s = sum_partials_n(part + j * VB, nb);
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
  dot_kernel<<<vec_grid(n), VT, 0, st>>>(x, y, n, part);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_reduce_partials(const double* part, long long n, double* out, int take_sqrt, cudaStream_t st) {
  reduce_kernel<<<1, VT, 0, st>>>(part, vec_grid(n), out, take_sqrt);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_axpby(double* y, const double* x, double a, double b, long long n, cudaStream_t st) {
  if (n <= 0) return EXA_OK;
  axpby_kernel<<<vec_grid(n), VT, 0, st>>>(y, x, a, b, n);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_scale(double* y, const double* x, double a, long long n, cudaStream_t st) {
  if (n <= 0) return EXA_OK;
  scale_kernel<<<vec_grid(n), VT, 0, st>>>(y, x, a, n);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_fill(double* y, double a, long long n, cudaStream_t st) {
  if (n <= 0) return EXA_OK;
  fill_kernel<<<vec_grid(n), VT, 0, st>>>(y, a, n);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_mgs_step(double* w, const double* vprev, const double* vnext, const double* part_in,
                 double* part_out, double* h_out, long long n, cudaStream_t st) {
  mgs_step_kernel<<<vec_grid(n), VT, 0, st>>>(w, vprev, vnext, part_in, part_out, h_out, n);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_mgs_finish(double* v, const double* w, const double* part_in, double* h_out, long long n, cudaStream_t st) {
  mgs_finish_kernel<<<vec_grid(n), VT, 0, st>>>(v, w, part_in, h_out, n);
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
  gemv_add_kernel<<<vec_grid(n), VT, 0, st>>>(x, V, y, n, k);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_cgs(double* w, const double* V, double* hcol, double* part, long long n, int k, cudaStream_t st) {
  const int nb = vec_grid(n);
  multi_dot_kernel<<<nb, VT, 0, st>>>(w, V, n, k, part);
  EXA_LAUNCH_CHECK();
  multi_reduce_kernel<<<1, VT, 0, st>>>(part, hcol, k, nb);
  EXA_LAUNCH_CHECK();
  gemv_sub_kernel<<<nb, VT, 0, st>>>(w, V, hcol, n, k);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

// ----------------------------------------------------------------------------------
// Column 2-norms with fixed scratch (exa_dnrm2_cols_fixed in the C ABI).
//
// The Krylov norms above take their per-block partial sums from memory that a solver
// context allocates when it is created.  This variant serves callers that hold no
// context and may not allocate device memory where they call it: code running inside
// another framework's memory pool, which has already reserved the free device memory so
// a cudaMalloc there can fail, and step loops that cannot afford the device-wide
// synchronisation that cudaFree performs.  Its partial sums live in the file-scope
// device array below, a fixed 151,552 bytes (COLNRM_MAXCOLS x VB doubles), so it handles
// at most COLNRM_MAXCOLS columns per call and rejects more with EXA_ERR_ARG.
//
// Nothing in the scratch has to start at zero: the first kernel overwrites every
// partial of the columns it handles before the second kernel reads them.  The array is
// one per device and per loaded library, so two calls whose kernels can overlap (on
// different streams without an ordering event, or from several host threads) race on
// it; calls on the same device must be ordered, e.g. issued on one stream.
//
// The arithmetic (grid-stride sums of squares per block, then the partials added in
// block order) is that of the context's norm, so both give the same bits.
// ----------------------------------------------------------------------------------
#include <mutex>

namespace {
constexpr int COLNRM_MAXCOLS = 64;
constexpr int COLNRM_MAXDEV = 64;
}  // namespace

static __device__ __align__(256) double g_colnrm_scratch[COLNRM_MAXCOLS * VB];

namespace {
std::mutex g_colnrm_mu;
double* g_colnrm_ptr[COLNRM_MAXDEV] = {};

// part[j * VB + block] = sum over this block's share of column j of x(i)^2
__global__ void __launch_bounds__(VT) colnrm_partial_kernel(const double* X, long long n, long long ldx,
                                                             double* part) {
  const int j = blockIdx.y;
  const double* x = X + ldx * j;
  double v = 0.0;
  for (long long i = blockIdx.x * (long long)VT + threadIdx.x; i < n; i += (long long)VB * VT) v = fma(x[i], x[i], v);
  double s = block_sum(v);
  if (threadIdx.x == 0) part[j * VB + blockIdx.x] = s;
}

// out[j] = sqrt(sum of column j's VB partials), one block per column.  The partial kernel runs
// VB blocks where the context's norm runs vec_grid(n): entry i lands in block (i / VT) mod VB
// in both, and the blocks past vec_grid(n) hold exact zeros, so both sums give the same bits.
__global__ void __launch_bounds__(VT) colnrm_finish_kernel(const double* part, double* out) {
  double s = sum_partials(part + blockIdx.x * VB);
  if (threadIdx.x == 0) out[blockIdx.x] = sqrt(s);
}

// Device address of this device's scratch, looked up on the first call made with that
// device current and cached afterwards.
int colnrm_scratch(double** out) {
  int dev = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= COLNRM_MAXDEV) {
    exa_set_error("exa_dnrm2_cols_fixed: device ordinal %d outside the %d devices it keeps scratch for", dev,
                  COLNRM_MAXDEV);
    return EXA_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_colnrm_mu);
  if (!g_colnrm_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_colnrm_scratch);
    if (e != cudaSuccess || p == nullptr) {
      exa_set_error("exa_dnrm2_cols_fixed: scratch address lookup failed: %s", cudaGetErrorString(e));
      return EXA_ERR_CUDA;
    }
    g_colnrm_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_colnrm_ptr[dev];
  return EXA_OK;
}
}  // namespace

extern "C" int exa_dnrm2_cols_fixed(const double* X, long long n, long long ldx, int ncols, double* out_dev,
                                    void* stream) {
  if (ncols < 1 || ncols > COLNRM_MAXCOLS) {
    exa_set_error("exa_dnrm2_cols_fixed: ncols = %d, but its fixed scratch holds 1 to %d columns per call", ncols,
                  COLNRM_MAXCOLS);
    return EXA_ERR_ARG;
  }
  if (n < 0 || (ncols > 1 && ldx < n)) {
    exa_set_error("exa_dnrm2_cols_fixed: bad sizes n = %lld, ldx = %lld", n, ldx);
    return EXA_ERR_ARG;
  }
  if (out_dev == nullptr || (n > 0 && X == nullptr)) {
    exa_set_error("exa_dnrm2_cols_fixed: null pointer");
    return EXA_ERR_ARG;
  }
  double* part = nullptr;
  EXA_TRY(colnrm_scratch(&part));
  cudaStream_t st = (cudaStream_t)stream;
  colnrm_partial_kernel<<<dim3(VB, ncols), VT, 0, st>>>(X, n, ldx, part);
  EXA_LAUNCH_CHECK();
  colnrm_finish_kernel<<<ncols, VT, 0, st>>>(part, out_dev);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

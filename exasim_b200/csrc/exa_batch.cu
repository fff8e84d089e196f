// Batched GMRES across contexts: the Arnoldi steps of many independent solves of one model
// (meshes of different sizes and polynomial orders) advance together, one set of launches per
// step for all of them.  No counterpart in the reference, which runs one problem per process.
//
// A context with a batcher attached hands each GMRES call (exa_drv_gmres) to the batcher and
// blocks until it is done; its own stream waits for the batcher's.  The batcher thread admits
// calls as they arrive, into free slots of a device table of job descriptors (continuous
// batching at the granularity of Arnoldi steps), and runs each step for all jobs at once:
//   matvec   w = H gather(v_i)              one launch over every job's elements
//   scatter  element -> face vectors        one launch over every job's faces
//   precond  v_{i+1} = P w (block Jacobi)   one launch over every job's faces
//   MGS      h_k, v_{i+1} -= h_k v_k        launch k serves every job whose step index is >= k
//   Givens   Hessenberg column, residual    one thread per job
// Each job has its own step index inside its restart cycle, so jobs join and leave at any
// step.  A step is one CUDA graph per highest step index, captured on its second use, with
// the jobs read from the device table.  The host reads every job's residual estimate one
// step late, as the single-context GMRES does.  Every reduction is per job with a partition
// that depends on the job's own sizes alone (the vector kernels' vec_grid), so a job's
// arithmetic, and its result, do not depend on what else is in the batch.  The elements per
// warp of the matvec are chosen by timing the candidates on the first batch (an autotuner).
#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "exa_batch.cuh"
#include "exa_solver.cuh"

namespace {

constexpr int BT = 256;        // threads of the grid-stride kernels
constexpr int VT = 256;        // threads of the reduction kernels (as the single-context ones)
constexpr int BMV_WARPS = 4;   // warps per block of the batched matvec

// device descriptor of one job (plain data)
struct BJob {
  const double* H;       // FP64 condensed blocks [m, m, ne] (plain form), or
  const float* H32;      // FP32 blocks (mixed form)
  const double* P;       // FP64 block-Jacobi blocks [ncf, ncf, nf], or
  const float* P32;      // FP32 blocks
  const int* elemcon;    // [ndf, ne]
  const int* f2e;        // [4, nf]
  double* V;             // Krylov basis [N, n1]
  double* w;             // [N]
  double* we;            // [m, ne]
  double* hess;          // [n1, restart]
  double* gs;
  double* gcs;
  double* gsn;
  double* part0;         // partial sums of the reductions (ping-pong)
  double* part1;
  const double* nrmb;    // device scalar: |P b|
  double* relerr;        // device scalar: the step's residual estimate
  long long N;
  int ne, nf, nf0, m, ncu, npf, ndf, n1;
  int step;              // Arnoldi step index of this batched step, -1: no step
  int vblocks;           // vec_grid(N): blocks of this job's reductions
};

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[VT / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < VT / 32; ++w) s += red[w];
  return s;  // valid in thread 0
}

__device__ __forceinline__ double sum_partials(const double* part, int nb) {
  __shared__ double tot;
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += VT) v += part[i];
  const double s = block_sum(v);
  if (threadIdx.x == 0) tot = s;
  __syncthreads();
  return tot;
}

// w_e = H_e gather(v_i) for every element of every stepping job: one warp per element, lane l
// keeps rows l and l + 32 (m <= 64), columns summed in index order
template <int EPW>
__global__ void __launch_bounds__(BMV_WARPS * 32) bmv_kernel(const BJob* jobs) {
  const BJob& J = jobs[blockIdx.y];
  if (J.step < 0) return;
  __shared__ double vs[BMV_WARPS][64];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int m = J.m, ncu = J.ncu, ndf = J.ndf;
  const double* v = J.V + (long long)J.step * J.N;
  const long long e0 = ((long long)blockIdx.x * BMV_WARPS + warp) * EPW;
  for (int t = 0; t < EPW; ++t) {
    const long long e = e0 + t;
    if (e >= J.ne) break;  // warp-uniform
    for (int k = lane; k < m; k += 32) vs[warp][k] = v[k % ncu + (long long)ncu * J.elemcon[k / ncu + (long long)ndf * e]];
    __syncwarp();
    double s0 = 0.0, s1 = 0.0;
    const int r0 = lane, r1 = lane + 32;
    if (J.H32) {
      const float* A = J.H32 + e * m * m;
      for (int c = 0; c < m; ++c) {
        const double x = vs[warp][c];
        if (r0 < m) s0 = fma((double)A[r0 + (long long)m * c], x, s0);
        if (r1 < m) s1 = fma((double)A[r1 + (long long)m * c], x, s1);
      }
    } else {
      const double* A = J.H + e * m * m;
      for (int c = 0; c < m; ++c) {
        const double x = vs[warp][c];
        if (r0 < m) s0 = fma(A[r0 + (long long)m * c], x, s0);
        if (r1 < m) s1 = fma(A[r1 + (long long)m * c], x, s1);
      }
    }
    if (r0 < m) J.we[e * m + r0] = s0;
    if (r1 < m) J.we[e * m + r1] = s1;
    __syncwarp();
  }
}

// element vectors to the face vector (the single-context scatter_kernel's sum order)
__global__ void bscatter_kernel(const BJob* jobs) {
  const BJob& J = jobs[blockIdx.y];
  if (J.step < 0) return;
  const int ncu = J.ncu, npf = J.npf, m = J.m;
  for (long long idx = blockIdx.x * (long long)BT + threadIdx.x; idx < J.N; idx += (long long)gridDim.x * BT) {
    const int k = idx % ncu;
    const long long q = idx / ncu;
    const int a = q % npf;
    const int f = (int)(q / npf);
    const int e1 = J.f2e[4 * f], l1 = J.f2e[4 * f + 1], e2 = J.f2e[4 * f + 2], l2 = J.f2e[4 * f + 3];
    double val = J.we[(long long)e1 * m + k + ncu * (a + npf * l1)];
    if (f < J.nf0 && e2 >= 0) {
      const int ii = J.elemcon[a + npf * l2 + J.ndf * e2] - npf * f;
      val += J.we[(long long)e2 * m + k + ncu * (ii + npf * l2)];
    }
    J.w[idx] = val;
  }
}

// v_{i+1} = P w, block Jacobi (the single-context bj_apply_kernel's sum order)
__global__ void bbj_kernel(const BJob* jobs) {
  const BJob& J = jobs[blockIdx.y];
  if (J.step < 0) return;
  const int ncf = J.ncu * J.npf;
  double* y = J.V + (long long)(J.step + 1) * J.N;
  for (long long idx = blockIdx.x * (long long)BT + threadIdx.x; idx < J.N; idx += (long long)gridDim.x * BT) {
    const int r = idx % ncf;
    const long long f = idx / ncf;
    const double* xf = J.w + f * ncf;
    double s = 0.0;
    if (J.P32) {
      const float* A = J.P32 + f * ncf * ncf;
      for (int c = 0; c < ncf; ++c) s = fma((double)A[r + ncf * c], xf[c], s);
    } else {
      const double* A = J.P + f * ncf * ncf;
      for (int c = 0; c < ncf; ++c) s = fma(A[r + ncf * c], xf[c], s);
    }
    y[idx] = s;
  }
}

// Modified Gram-Schmidt, launch k of a step (the single-context sequence of exa_dot_partials,
// mgs_step and mgs_finish, per job): k = 0 dots v_{i+1} with v_0; 1 <= k <= i subtracts h_{k-1}
// v_{k-1} and dots with v_k; k = i + 1 subtracts h_i v_i and takes |v_{i+1}|^2; k = i + 2 scales
// v_{i+1} by 1 / h_{i+1}.  Jobs with i + 2 < k have nothing to do.
__global__ void __launch_bounds__(VT) bmgs_kernel(const BJob* jobs, int k) {
  const BJob& J = jobs[blockIdx.y];
  const int i = J.step;
  if (i < 0 || k > i + 2 || (int)blockIdx.x >= J.vblocks) return;
  const long long N = J.N;
  const int nb = J.vblocks;
  double* vn = J.V + (long long)(i + 1) * N;
  double* hcol = J.hess + (long long)J.n1 * i;
  const double* pin = ((k + 1) & 1) ? J.part1 : J.part0;
  double* pout = (k & 1) ? J.part1 : J.part0;
  const long long i0 = blockIdx.x * (long long)VT + threadIdx.x, stride = (long long)nb * VT;
  if (k == 0) {
    double v = 0.0;
    for (long long t = i0; t < N; t += stride) v = fma(vn[t], J.V[t], v);
    const double s = block_sum(v);
    if (threadIdx.x == 0) pout[blockIdx.x] = s;
    return;
  }
  if (k <= i + 1) {
    const double h = sum_partials(pin, nb);
    if (blockIdx.x == 0 && threadIdx.x == 0) hcol[k - 1] = h;
    const double* vprev = J.V + (long long)(k - 1) * N;
    const double* vnext = k <= i ? J.V + (long long)k * N : nullptr;
    double v = 0.0;
    for (long long t = i0; t < N; t += stride) {
      const double wi = vn[t] - h * vprev[t];
      vn[t] = wi;
      v = fma(wi, vnext ? vnext[t] : wi, v);
    }
    const double s = block_sum(v);
    if (threadIdx.x == 0) pout[blockIdx.x] = s;
    return;
  }
  const double h = sqrt(sum_partials(pin, nb));
  if (blockIdx.x == 0 && threadIdx.x == 0) hcol[i + 1] = h;
  const double r = 1.0 / h;
  for (long long t = i0; t < N; t += stride) vn[t] = vn[t] * r;
}

// cpuApplyGivensRotation (backend/Common/cpuimpl.h:167-196) per job, and the residual estimate
// |s_{i+1}| / |P b|, also gathered into rel[slot] for one copy to the host
__global__ void bgivens_kernel(const BJob* jobs, int cap, double* rel) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cap) return;
  const BJob& J = jobs[j];
  const int i = J.step;
  if (i < 0) return;
  double* H = J.hess + (long long)J.n1 * i;
  double *s = J.gs, *cs = J.gcs, *sn = J.gsn;
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
  const double re = fabs(s[i + 1]) / *J.nrmb;
  *J.relerr = re;
  rel[j] = re;
}

int vec_blocks(long long n) {
  const long long b = (n + VT - 1) / VT;
  return (int)(b < 1 ? 1 : (b > 296 ? 296 : b));
}

enum { JOB_STEPPING = 0, JOB_CYCLE_END = 1, JOB_DONE = 2 };

struct Job {
  ExaCtx* c = nullptr;
  cudaStream_t orig = nullptr;
  cudaEvent_t ready = nullptr;
  int slot = -1;
  int state = JOB_STEPPING;
  int next_i = 0;           // step index to enqueue next in this cycle
  int enq[2] = {-1, -1};    // step index enqueued in batched step s (by s % 2), -1: none
  int last_i = -1;          // last step index whose result was read
  int taken = 0;            // Arnoldi steps whose results were read
  int enqueued = 0;         // Arnoldi steps enqueued in all
  double nrmb = 0.0, tol = 0.0, relerr = 1.0;
  bool finished = false;
  int status = EXA_OK;
};

}  // namespace

struct ExaBatcher {
  int device = 0, cap = 0;
  cudaStream_t st = nullptr;
  BJob* d_jobs = nullptr;
  BJob* h_jobs[2] = {nullptr, nullptr};   // pinned staging (alternating steps)
  double* d_rel = nullptr;
  double* h_rel[2] = {nullptr, nullptr};  // pinned
  cudaEvent_t ev[2] = {nullptr, nullptr};
  std::vector<Job*> slots;
  std::deque<Job*> pending;
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::thread th;
  bool stop = false;
  // launch extents, grown with the largest job admitted (captured graphs are dropped then)
  long long max_N = 0;
  int max_ne = 0, max_vb = 1;
  int epw = 0;                             // tuned elements per warp of the matvec (0: untuned)
  std::vector<cudaGraphExec_t> graphs;     // per highest step index
  std::vector<unsigned char> seen;
  long long launches = 0, steps = 0, jobs_done = 0;
};

namespace {

int launch_bmv(ExaBatcher& b, int epw) {
  const long long per = (long long)BMV_WARPS * epw;
  dim3 grid((unsigned)std::max<long long>(1, (b.max_ne + per - 1) / per), (unsigned)b.cap);
  switch (epw) {
    case 1: bmv_kernel<1><<<grid, BMV_WARPS * 32, 0, b.st>>>(b.d_jobs); break;
    case 2: bmv_kernel<2><<<grid, BMV_WARPS * 32, 0, b.st>>>(b.d_jobs); break;
    case 4: bmv_kernel<4><<<grid, BMV_WARPS * 32, 0, b.st>>>(b.d_jobs); break;
    default: bmv_kernel<8><<<grid, BMV_WARPS * 32, 0, b.st>>>(b.d_jobs); break;
  }
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

// the launches of one batched Arnoldi step whose highest step index is maxi
int step_ops(ExaBatcher& b, int maxi) {
  EXA_TRY(launch_bmv(b, b.epw));
  const unsigned gf = (unsigned)std::max<long long>(1, std::min<long long>((b.max_N + BT - 1) / BT, 1184));
  bscatter_kernel<<<dim3(gf, b.cap), BT, 0, b.st>>>(b.d_jobs);
  EXA_LAUNCH_CHECK();
  bbj_kernel<<<dim3(gf, b.cap), BT, 0, b.st>>>(b.d_jobs);
  EXA_LAUNCH_CHECK();
  for (int k = 0; k <= maxi + 2; ++k) {
    bmgs_kernel<<<dim3((unsigned)b.max_vb, b.cap), VT, 0, b.st>>>(b.d_jobs, k);
    EXA_LAUNCH_CHECK();
  }
  bgivens_kernel<<<(b.cap + 127) / 128, 128, 0, b.st>>>(b.d_jobs, b.cap, b.d_rel);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

// the elements per warp of the matvec: each candidate timed on the current batch (it only
// rewrites the jobs' element vectors, which the step recomputes), the fastest kept
int tune_matvec(ExaBatcher& b) {
  const int cand[] = {1, 2, 4, 8};
  cudaEvent_t e0, e1;
  EXA_CUDA(cudaEventCreate(&e0));
  EXA_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int pick = 2;
  for (int epw : cand) {
    EXA_TRY(launch_bmv(b, epw));  // warm
    EXA_CUDA(cudaEventRecord(e0, b.st));
    for (int r = 0; r < 5; ++r) EXA_TRY(launch_bmv(b, epw));
    EXA_CUDA(cudaEventRecord(e1, b.st));
    EXA_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    EXA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best) {
      best = ms;
      pick = epw;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b.epw = pick;
  return EXA_OK;
}

void drop_graphs(ExaBatcher& b) {
  for (auto& g : b.graphs)
    if (g) cudaGraphExecDestroy(g);
  b.graphs.assign(b.graphs.size(), nullptr);
  std::fill(b.seen.begin(), b.seen.end(), 0);
}

// one batched step: from its second use at a given highest step index it is a captured graph
int run_step(ExaBatcher& b, int maxi) {
  const long long l0 = exa_thread_launches();
  if (maxi >= (int)b.graphs.size()) {
    b.graphs.resize(maxi + 1, nullptr);
    b.seen.resize(maxi + 1, 0);
  }
  cudaGraphExec_t& ex = b.graphs[maxi];
  if (ex) {
    EXA_CUDA(cudaGraphLaunch(ex, b.st));
    exa_add_launches(maxi + 7);
    b.launches += maxi + 7;
    return EXA_OK;
  }
  if (!b.seen[maxi]) {
    b.seen[maxi] = 1;
    EXA_TRY(step_ops(b, maxi));
    b.launches += exa_thread_launches() - l0;
    return EXA_OK;
  }
  EXA_CUDA(cudaStreamBeginCapture(b.st, cudaStreamCaptureModeThreadLocal));
  const int s = step_ops(b, maxi);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b.st, &g);
  exa_add_launches(-(exa_thread_launches() - l0));  // counted at the replay below
  if (s == EXA_OK && e == cudaSuccess && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess) {
    cudaGraphDestroy(g);
    EXA_CUDA(cudaGraphLaunch(ex, b.st));
    exa_add_launches(maxi + 7);
    b.launches += maxi + 7;
    return EXA_OK;
  }
  if (g) cudaGraphDestroy(g);
  ex = nullptr;
  cudaGetLastError();
  EXA_TRY(step_ops(b, maxi));
  b.launches += exa_thread_launches() - l0;
  return EXA_OK;
}

// a new restart cycle from r (its norm nrmr): v_0 = r / nrmr, s = (nrmr, 0, ...)
int start_cycle(ExaCtx& c, Job& j, double nrmr) {
  const int n1 = c.restart + 1;
  EXA_TRY(exa_scale(c.V, c.r, 1.0 / nrmr, c.ndofuhat(), c.st));
  std::vector<double> s0(n1, 0.0);
  s0[0] = nrmr;
  EXA_CUDA(cudaStreamSynchronize(c.st));  // c.pinned is free again
  std::copy(s0.begin(), s0.end(), c.pinned);
  EXA_CUDA(cudaMemcpyAsync(c.gs, c.pinned, sizeof(double) * n1, cudaMemcpyHostToDevice, c.st));
  EXA_CUDA(cudaStreamSynchronize(c.st));
  j.state = JOB_STEPPING;
  j.next_i = 0;
  return EXA_OK;
}

// admission: x = 0, the tolerance, r = P b and the first cycle (gmres.cpp:396-455 without a
// reduced-basis guess); done at once when |b| is below the Newton tolerance
int admit(ExaBatcher& b, Job& j) {
  ExaCtx& c = *j.c;
  const long long N = c.ndofuhat();
  EXA_CUDA(cudaStreamWaitEvent(b.st, j.ready, 0));
  j.orig = c.st;
  c.st = b.st;
  EXA_CUDA(cudaMemsetAsync(c.x, 0, sizeof(double) * N, c.st));
  double nrmb = 0.0;
  EXA_TRY(exa_drv_norm(c, c.b, N, &nrmb));
  if (nrmb < c.newton_tol) {
    j.finished = true;
    j.relerr = 0.0;
    return EXA_OK;
  }
  j.tol = std::min(0.1, c.gmres_tol);
  EXA_TRY(exa_drv_precond(c, c.b, c.r));
  EXA_TRY(exa_drv_norm(c, c.r, N, &nrmb));
  j.nrmb = nrmb;
  c.pinned[0] = nrmb;
  EXA_CUDA(cudaMemcpyAsync(c.scal + 14, c.pinned, sizeof(double), cudaMemcpyHostToDevice, c.st));
  return start_cycle(c, j, nrmb);
}

// the end of a cycle (or of the iteration budget) after step i: x += V y, r = P (b - A x)
int cycle_end(ExaBatcher& b, Job& j, int i) {
  ExaCtx& c = *j.c;
  const long long N = c.ndofuhat();
  EXA_TRY(exa_drv_gmres_update(c, i));
  EXA_TRY(exa_drv_matvec(c, c.x, c.w));
  EXA_TRY(exa_axpby(c.w, c.b, 1.0, -1.0, N, c.st));
  EXA_TRY(exa_drv_precond(c, c.w, c.r));
  double nrmr = 0.0;
  EXA_TRY(exa_drv_norm(c, c.r, N, &nrmr));
  j.relerr = nrmr / j.nrmb;
  if (j.relerr < j.tol || j.taken >= c.gmres_maxit) {
    j.finished = true;
    return EXA_OK;
  }
  return start_cycle(c, j, nrmr);
}

void finish(ExaBatcher& b, Job& j) {
  ExaCtx& c = *j.c;
  if (j.status == EXA_OK) {
    c.last_gmres_converged = j.relerr < j.tol || j.nrmb == 0.0;
    cudaEvent_t done = nullptr;
    if (cudaEventCreateWithFlags(&done, cudaEventDisableTiming) == cudaSuccess) {
      cudaEventRecord(done, b.st);
      cudaStreamWaitEvent(j.orig, done, 0);
      cudaEventDestroy(done);
    } else {
      cudaStreamSynchronize(b.st);
    }
  } else {
    cudaStreamSynchronize(b.st);
  }
  c.st = j.orig;
  if (j.slot >= 0) b.slots[j.slot] = nullptr;
  ++b.jobs_done;
  {
    std::lock_guard<std::mutex> lk(b.mu);
    j.finished = true;
    j.state = JOB_DONE;
  }
  b.done_cv.notify_all();
}

void fail(ExaBatcher& b, Job& j, int st) {
  j.status = st;
  finish(b, j);
}

void loop(ExaBatcher* bp) {
  ExaBatcher& b = *bp;
  cudaSetDevice(b.device);
  long long s = 0;  // batched steps enqueued
  bool prev = false;
  for (;;) {
    // admit new calls into free slots
    std::vector<Job*> fresh;
    {
      std::unique_lock<std::mutex> lk(b.mu);
      bool any = prev;
      for (Job* j : b.slots) any = any || j;
      if (!any) b.cv.wait(lk, [&] { return b.stop || !b.pending.empty(); });
      if (b.stop && b.pending.empty() && !any) return;
      for (int k = 0; k < b.cap && !b.pending.empty(); ++k)
        if (!b.slots[k]) {
          Job* j = b.pending.front();
          b.pending.pop_front();
          j->slot = k;
          b.slots[k] = j;
          fresh.push_back(j);
        }
    }
    for (Job* j : fresh) {
      ExaCtx& c = *j->c;
      const int st = admit(b, *j);
      if (st != EXA_OK) { fail(b, *j, st); continue; }
      if (j->finished) { finish(b, *j); continue; }
      if (c.ndofuhat() > b.max_N || c.P.ne > b.max_ne || vec_blocks(c.ndofuhat()) > b.max_vb) {
        b.max_N = std::max(b.max_N, c.ndofuhat());
        b.max_ne = std::max(b.max_ne, c.P.ne);
        b.max_vb = std::max(b.max_vb, vec_blocks(c.ndofuhat()));
        drop_graphs(b);
      }
    }
    // descriptors of step s
    const int cur = (int)(s & 1);
    BJob* hj = b.h_jobs[cur];
    int maxi = -1;
    for (int k = 0; k < b.cap; ++k) {
      BJob d{};
      d.step = -1;
      Job* j = b.slots[k];
      if (j) j->enq[cur] = -1;
      if (j && !j->finished && j->state == JOB_STEPPING) {
        ExaCtx& c = *j->c;
        const ExaDims& P = c.P;
        d.H = c.precision == 1 ? nullptr : c.H;
        d.H32 = c.precision == 1 ? c.H32 : nullptr;
        d.P = c.precision == 1 ? nullptr : c.Pc;
        d.P32 = c.precision == 1 ? c.Pc32 : nullptr;
        d.elemcon = c.elemcon;
        d.f2e = c.f2e;
        d.V = c.V;
        d.w = c.w;
        d.we = c.we;
        d.hess = c.hess;
        d.gs = c.gs;
        d.gcs = c.gcs;
        d.gsn = c.gsn;
        d.part0 = c.part_a;
        d.part1 = c.part_b;
        d.nrmb = c.scal + 14;
        d.relerr = c.scal + 13;
        d.N = c.ndofuhat();
        d.ne = P.ne; d.nf = P.nf; d.nf0 = P.nf0; d.m = P.m; d.ncu = P.ncu; d.npf = P.npf; d.ndf = P.ndf;
        d.n1 = c.restart + 1;
        d.vblocks = vec_blocks(d.N);
        d.step = j->next_i;
        j->enq[cur] = j->next_i;
        maxi = std::max(maxi, j->next_i);
        ++j->enqueued;
        ++j->next_i;
        if (j->next_i >= c.restart || j->enqueued >= c.gmres_maxit) j->state = JOB_CYCLE_END;
      }
      hj[k] = d;
    }
    const bool this_step = maxi >= 0;
    if (this_step) {
      int st = EXA_OK;
      if (cudaMemcpyAsync(b.d_jobs, hj, sizeof(BJob) * b.cap, cudaMemcpyHostToDevice, b.st) != cudaSuccess)
        st = EXA_ERR_CUDA;
      if (st == EXA_OK && b.epw == 0) st = tune_matvec(b);
      if (st == EXA_OK) st = run_step(b, maxi);
      if (st == EXA_OK &&
          cudaMemcpyAsync(b.h_rel[cur], b.d_rel, sizeof(double) * b.cap, cudaMemcpyDeviceToHost, b.st) != cudaSuccess)
        st = EXA_ERR_CUDA;
      if (st == EXA_OK && cudaEventRecord(b.ev[cur], b.st) != cudaSuccess) st = EXA_ERR_CUDA;
      if (st != EXA_OK) {
        for (Job* j : b.slots)
          if (j) fail(b, *j, st);
        s = 0;
        prev = false;
        continue;
      }
      ++b.steps;
    }
    // results of step s - 1 (one step late), then those of step s when nothing follows it
    auto read_results = [&](int half) {
      cudaEventSynchronize(b.ev[half]);
      for (Job* j : b.slots) {
        if (!j || j->finished || j->enq[half] < 0) continue;
        const int i = j->enq[half];
        j->enq[half] = -1;
        j->relerr = b.h_rel[half][j->slot];
        ++j->taken;
        j->last_i = i;
        ExaCtx& c = *j->c;
        int st = EXA_OK;
        if (j->relerr < j->tol) {
          // converged at step i; a step i + 1 enqueued meanwhile writes nothing the update reads
          st = exa_drv_gmres_update(c, i);
          if (st == EXA_OK) {
            j->finished = true;
            finish(b, *j);
          }
        } else if (j->state == JOB_CYCLE_END && j->enq[half ^ 1] < 0) {
          st = cycle_end(b, *j, i);
          if (st == EXA_OK && j->finished) finish(b, *j);
        }
        if (st != EXA_OK) fail(b, *j, st);
      }
    };
    if (prev) read_results((int)((s - 1) & 1));
    prev = this_step;
    if (this_step) ++s;
    bool more = false;
    for (Job* j : b.slots) more = more || (j && !j->finished && j->state == JOB_STEPPING);
    if (!more && prev) {
      read_results((int)((s - 1) & 1));
      prev = false;
    }
  }
}

}  // namespace

bool exa_batchable(const ExaCtx& c) {
  return c.preconditioner == 0 && c.RBdim == 0 && c.ortho == 0 && c.ppdegree <= 1 && c.P.m <= 64 &&
         c.P.ncu * c.P.npf <= 64 && c.restart >= 1 && !c.prof.on;
}

int exa_batcher_create(int device, int capacity, ExaBatcher** out) {
  if (capacity < 1 || capacity > 1024) {
    exa_set_error("batcher capacity %d outside 1..1024", capacity);
    return EXA_ERR_ARG;
  }
  auto* b = new ExaBatcher();
  b->device = device;
  b->cap = capacity;
  b->slots.assign(capacity, nullptr);
  int st = EXA_OK;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&b->d_jobs, sizeof(BJob) * capacity) != cudaSuccess ||
      cudaMalloc(&b->d_rel, sizeof(double) * capacity) != cudaSuccess ||
      cudaMallocHost(&b->h_jobs[0], sizeof(BJob) * capacity) != cudaSuccess ||
      cudaMallocHost(&b->h_jobs[1], sizeof(BJob) * capacity) != cudaSuccess ||
      cudaMallocHost(&b->h_rel[0], sizeof(double) * capacity) != cudaSuccess ||
      cudaMallocHost(&b->h_rel[1], sizeof(double) * capacity) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev[1], cudaEventDisableTiming) != cudaSuccess) {
    exa_set_error("batcher set-up: %s", cudaGetErrorString(cudaGetLastError()));
    st = EXA_ERR_CUDA;
  }
  if (st != EXA_OK) {
    exa_batcher_destroy(b);
    return st;
  }
  b->th = std::thread(loop, b);
  *out = b;
  return EXA_OK;
}

void exa_batcher_destroy(ExaBatcher* b) {
  if (!b) return;
  if (b->th.joinable()) {
    {
      std::lock_guard<std::mutex> lk(b->mu);
      b->stop = true;
    }
    b->cv.notify_all();
    b->th.join();
  }
  cudaSetDevice(b->device);
  if (b->st) cudaStreamSynchronize(b->st);
  drop_graphs(*b);
  for (cudaEvent_t e : b->ev)
    if (e) cudaEventDestroy(e);
  if (b->d_jobs) cudaFree(b->d_jobs);
  if (b->d_rel) cudaFree(b->d_rel);
  for (int k = 0; k < 2; ++k) {
    if (b->h_jobs[k]) cudaFreeHost(b->h_jobs[k]);
    if (b->h_rel[k]) cudaFreeHost(b->h_rel[k]);
  }
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
}

int exa_batcher_gmres(ExaBatcher* b, ExaCtx& c, int* iters_out, double* relerr_out) {
  Job j;
  j.c = &c;
  EXA_CUDA(cudaEventCreateWithFlags(&j.ready, cudaEventDisableTiming));
  EXA_CUDA(cudaEventRecord(j.ready, c.st));
  {
    std::lock_guard<std::mutex> lk(b->mu);
    b->pending.push_back(&j);
  }
  b->cv.notify_all();
  {
    std::unique_lock<std::mutex> lk(b->mu);
    b->done_cv.wait(lk, [&] { return j.state == JOB_DONE; });
  }
  cudaEventDestroy(j.ready);
  *iters_out = j.taken;
  *relerr_out = j.relerr;
  if (j.status != EXA_OK) {
    exa_set_error("batched GMRES failed (status %d)", j.status);
    return j.status;
  }
  return EXA_OK;
}

void exa_batcher_stats(ExaBatcher* b, long long* out) {
  out[0] = b->steps;
  out[1] = b->launches;
  out[2] = b->jobs_done;
  out[3] = b->epw;
}

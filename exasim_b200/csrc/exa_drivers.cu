// Linear-system, Krylov, Newton and DIRK drivers on top of the device kernels.
// The control flow is Exasim's (references at each function); all vectors stay on
// the device, and the host reads one scalar per GMRES iteration (the Givens residual)
// as the reference does with its host-side Givens rotations.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "exa_batch.cuh"
#include "exa_solver.cuh"

// ---- phase profile: a pool of event pairs, summed into per-phase totals when read or full
namespace {
constexpr int PROF_SLOTS = 2048;
}

int exa_prof_flush(ExaCtx& c) {
  ExaProf& p = c.prof;
  if (p.used == 0) return EXA_OK;
  EXA_CUDA(cudaStreamSynchronize(c.st));
  for (int i = 0; i < p.used; ++i) {
    float ms = 0.0f;
    EXA_CUDA(cudaEventElapsedTime(&ms, p.ev[2 * i], p.ev[2 * i + 1]));
    p.ms[p.phase[i]] += ms;
    p.count[p.phase[i]] += 1;
  }
  p.used = 0;
  return EXA_OK;
}

int exa_prof_enable(ExaCtx& c, int on) {
  ExaProf& p = c.prof;
  if (on) {
    if (p.ev.empty()) {
      p.ev.resize(2 * PROF_SLOTS);
      p.phase.resize(PROF_SLOTS);
      for (auto& e : p.ev) EXA_CUDA(cudaEventCreate(&e));
    }
    EXA_TRY(exa_prof_flush(c));
    for (int i = 0; i < EXA_NPHASE; ++i) p.ms[i] = 0.0, p.count[i] = 0, p.flops[i] = 0.0;
    p.on = true;
  } else {
    EXA_TRY(exa_prof_flush(c));
    p.on = false;
  }
  return EXA_OK;
}

void exa_prof_free(ExaCtx& c) {
  for (auto& e : c.prof.ev) cudaEventDestroy(e);
  c.prof.ev.clear();
  c.prof.on = false;
  c.prof.used = 0;
}

// Profiling is best effort: a failed event record leaves the slot unused and the solver
// call unaffected.
ExaProfScope::ExaProfScope(ExaCtx& ctx, int phase) : c(ctx) {
  ExaProf& p = c.prof;
  if (!p.on) return;
  if (p.used == PROF_SLOTS && exa_prof_flush(c) != EXA_OK) return;
  if (cudaEventRecord(p.ev[2 * p.used], c.st) != cudaSuccess) return;
  slot = p.used++;
  p.phase[slot] = phase;
}

ExaProfScope::~ExaProfScope() {
  if (slot >= 0 && cudaEventRecord(c.prof.ev[2 * slot + 1], c.st) != cudaSuccess) {
    // drop the unfinished slot if it is the last one, otherwise time it to the next record
    if (slot == c.prof.used - 1) c.prof.used--;
  }
}

int exa_drv_norm(ExaCtx& c, const double* x, long long n, double* out) {
  EXA_TRY(exa_dot_partials(x, x, n, c.part_a, c.st));
  EXA_TRY(exa_reduce_partials(c.part_a, n, c.scal + 15, 1, c.st));
  EXA_CUDA(cudaMemcpyAsync(c.pinned, c.scal + 15, sizeof(double), cudaMemcpyDeviceToHost, c.st));
  EXA_CUDA(cudaStreamSynchronize(c.st));
  *out = c.pinned[0];
  return EXA_OK;
}

// hdgAssembleRHS + preconditioner setup (discretization.cpp:483-573, matvec.cpp:103-217)
int exa_drv_build_precond(ExaCtx& c) {
  const ExaDims& P = c.P;
  ExaProfScope ps(c, EXA_PH_PRECOND_BUILD);
  if (c.preconditioner == 2) {
    // super-element additive Schwarz with block ILU(0) (matvec.cpp:119-166)
    if (c.precision == 1) return exa_k_bilu_build(P, c.bilu, c.f2e, c.elemcon, c.H32, c.Pc32, c.d_flag, c.st);
    return exa_k_bilu_build(P, c.bilu, c.f2e, c.elemcon, c.H, c.Pc, c.d_flag, c.st);
  }
  if (c.precision == 1) {
    // mixed form: blocks from the FP32 condensed matrix, inverted in FP32
    if (c.preconditioner == 0) {
      const int ncf = P.ncu * P.npf;
      EXA_TRY(exa_k_bj_build(P, c.f2e, c.elemcon, c.H32, c.Pc32, c.st));
      EXA_TRY(exa_inverse(c.Pc32, ncf, (long long)ncf * ncf, P.nf, c.d_flag, c.st));
    } else {
      EXA_TRY(exa_k_eas_build(P, c.f2e, c.elemcon, c.H32, c.Pc32, c.st));
      EXA_TRY(exa_inverse(c.Pc32, P.m, (long long)P.m * P.m, P.ne, c.d_flag, c.st));
    }
    return EXA_OK;
  }
  if (c.preconditioner == 0) {
    EXA_TRY(exa_k_bj_build(P, c.f2e, c.elemcon, c.H, c.Pc, c.st));
    const int ncf = P.ncu * P.npf;
    EXA_TRY(exa_inverse(c.Pc, ncf, (long long)ncf * ncf, P.nf, c.d_flag, c.st));
  } else {
    EXA_TRY(exa_k_eas_build(P, c.f2e, c.elemcon, c.H, c.Pc, c.st));
    EXA_TRY(exa_inverse(c.Pc, P.m, (long long)P.m * P.m, P.ne, c.d_flag, c.st));
  }
  return EXA_OK;
}

int exa_drv_assemble(ExaCtx& c) {
  // d_flag[0]: zero pivot in an inverse; d_flag[1]: a tensor-core kernel's wait ran out
  EXA_CUDA(cudaMemsetAsync(c.d_flag, 0, 2 * sizeof(int), c.st));
  EXA_TRY(exa_model_assemble(c, true));
  EXA_TRY(exa_k_scatter(c.P, c.f2e, c.elemcon, c.Rh, c.b, c.st));
  EXA_TRY(exa_drv_build_precond(c));
  int flag[2] = {0, 0};
  EXA_CUDA(cudaMemcpyAsync(c.pinned, c.d_flag, 2 * sizeof(int), cudaMemcpyDeviceToHost, c.st));
  EXA_CUDA(cudaStreamSynchronize(c.st));
  std::memcpy(flag, c.pinned, 2 * sizeof(int));
  if (flag[1]) {
    exa_set_error("tensor-core element elimination: a wait inside the kernel ran out");
    return EXA_ERR_CUDA;
  }
  if (flag[0]) {
    exa_set_error("singular element or preconditioner block during assembly");
    return EXA_ERR_SINGULAR;
  }
  return EXA_OK;
}

// hdgAssembleResidual: Ru, Rh, b; norm = |b| + |Ru| (solution.cpp:148-157)
int exa_drv_residual(ExaCtx& c, double* norm) {
  if (c.scheme == 0) {
    // LDG: R(u) of the element states (residual.cpp:589-617); norm = |R|
    EXA_TRY(exa_model_ldg_residual(c, c.udg, c.ldg_R));
    if (norm) EXA_TRY(exa_drv_norm(c, c.ldg_R, c.sysN(), norm));
    return EXA_OK;
  }
  EXA_TRY(exa_model_assemble(c, false));
  EXA_TRY(exa_k_scatter(c.P, c.f2e, c.elemcon, c.Rh, c.b, c.st));
  if (norm) {
    double nb = 0.0, nr = 0.0;
    EXA_TRY(exa_drv_norm(c, c.b, c.ndofuhat(), &nb));
    EXA_TRY(exa_drv_norm(c, c.Ru, (long long)c.P.n * c.P.ne, &nr));
    *norm = nb + nr;
  }
  return EXA_OK;
}

// LDG: w = J(u) v by differences of residuals around the current state u = udg with R(u) in
// ldg_R (MatVec, matvec.cpp:41-100): (R(u + eps v) - R(u)) / eps, or the central difference
int ldg_matvec(ExaCtx& c, const double* v, double* w) {
  const long long N = c.sysN();
  const double eps = c.matvec_eps;
  if (c.matvec_order == 1) {
    EXA_TRY(exa_lincomb(c.ldg_w, 1.0, c.udg, eps, v, N, c.st));
    EXA_TRY(exa_model_ldg_residual(c, c.ldg_w, c.ldg_Rw));
    return exa_lincomb(w, 1.0 / eps, c.ldg_Rw, -1.0 / eps, c.ldg_R, N, c.st);
  }
  EXA_TRY(exa_lincomb(c.ldg_w, 1.0, c.udg, -eps, v, N, c.st));
  EXA_TRY(exa_model_ldg_residual(c, c.ldg_w, c.ldg_Rm));
  EXA_TRY(exa_lincomb(c.ldg_w, 1.0, c.udg, eps, v, N, c.st));
  EXA_TRY(exa_model_ldg_residual(c, c.ldg_w, c.ldg_Rw));
  return exa_lincomb(w, 0.5 / eps, c.ldg_Rw, -0.5 / eps, c.ldg_Rm, N, c.st);
}

// w = A v (hdgMatVec, matvec.cpp:240-389)
int exa_drv_matvec(ExaCtx& c, const double* v, double* w) {
  ExaProfScope ps(c, EXA_PH_MATVEC);
  if (c.scheme == 0) return ldg_matvec(c, v, w);
  if (c.precision == 1)
    EXA_TRY(exa_k_elem_matvec(c.P, c.elemcon, c.H32, v, c.we, c.st, c.d_uflag));
  else
    EXA_TRY(exa_k_elem_matvec(c.P, c.elemcon, c.H, v, c.we, c.st));
  EXA_TRY(exa_k_scatter(c.P, c.f2e, c.elemcon, c.we, w, c.st));
  return EXA_OK;
}

// w = P v (ApplyPreconditioner, preconditioner.cpp:273-295); v and w may not alias
int exa_drv_precond(ExaCtx& c, const double* v, double* w) {
  ExaProfScope ps(c, EXA_PH_PRECOND_APPLY);
  if (c.scheme == 0) {
    // LDG (ApplyMatrix, applymatrix.cpp:66-98): the identity (precMatrixType 0) or the
    // element mass inverse applied to each field
    if (c.ldg_prec_matrix == 0) {
      EXA_CUDA(cudaMemcpyAsync(w, v, sizeof(double) * c.sysN(), cudaMemcpyDeviceToDevice, c.st));
      return EXA_OK;
    }
    const ExaDims& P = c.P;
    GemmBatch g{};
    g.M = P.npe; g.N = P.ncu; g.K = P.npe; g.alpha = 1.0; g.beta = 0.0;
    g.A = c.Minv; g.lda = P.npe; g.sA = (long long)P.npe * P.npe;
    g.B = v; g.ldb = P.npe; g.sB = (long long)P.npe * P.ncu;
    g.C = w; g.ldc = P.npe; g.sC = (long long)P.npe * P.ncu;
    g.batch = P.ne; g.batch2 = 1;
    return exa_gemm(g, c.st);
  }
  if (c.preconditioner == 2) {
    if (c.precision == 1) return exa_k_bilu_apply(c.P, c.bilu, c.Pc32, v, w, c.st);
    return exa_k_bilu_apply(c.P, c.bilu, c.Pc, v, w, c.st);
  }
  if (c.precision == 1) {
    if (c.preconditioner == 0) return exa_k_bj_apply(c.P, c.Pc32, v, w, c.st);
    EXA_TRY(exa_k_elem_matvec(c.P, c.elemcon, c.Pc32, v, c.we, c.st, c.d_uflag));
    return exa_k_scatter(c.P, c.f2e, c.elemcon, c.we, w, c.st);
  }
  if (c.preconditioner == 0) return exa_k_bj_apply(c.P, c.Pc, v, w, c.st);
  EXA_TRY(exa_k_elem_matvec(c.P, c.elemcon, c.Pc, v, c.we, c.st));
  return exa_k_scatter(c.P, c.f2e, c.elemcon, c.we, w, c.st);
}

int exa_drv_getq(ExaCtx& c) {
  if (c.P.ncq == 0) return EXA_OK;
  ExaProfScope ps(c, EXA_PH_GETQ);
  if (c.Minv && exa_getq_mf_smem(c.P, c.wq_w != nullptr) <= 227 * 1024) {
    if (c.wq_w) EXA_TRY(exa_k_getq_gemm(c.P, c.shapegt, c.shapegw, c.elemg, c.udg, c.wq_ug, c.wq_v, c.wq_w, c.st));
    return exa_k_getq_mf(c.P, c.shapegt, c.shapegw, c.shapfgt, c.shapfgw, c.perm, c.elemcon, c.elemg, c.faceg, c.Minv,
                         c.uh, c.udg, c.st, c.wq_w);
  }
  return exa_k_getq(c.P, c.elemcon, c.MC, c.ME, c.uh, c.udg, c.st);
}

extern "C" int exa_poly_ritz(const double* H, int m, double* sr, double* si);

namespace {

// out = P A x (x may be out): the matvec into c.w, then the preconditioner
int pa(ExaCtx& c, const double* x, double* out) {
  EXA_TRY(exa_drv_matvec(c, x, c.w));
  return exa_drv_precond(c, c.w, out);
}

// ApplyPoly (backend/Solver/gmres.cpp:319-357): wv <- s(P A) wv, the polynomial whose roots are
// the Leja-ordered Ritz values (complex pairs through one real quadratic factor); uses c.w,
// poly_q and poly_p as work.  Nothing to do without a polynomial preconditioner.
int apply_poly(ExaCtx& c, double* wv) {
  if (c.ppdegree <= 1) return EXA_OK;
  const int m = c.ppdegree;
  const long long N = c.sysN();
  double *q = c.poly_q, *p = c.poly_p;
  const std::vector<double>&sr = c.poly_sr, &si = c.poly_si;
  EXA_CUDA(cudaMemcpyAsync(q, wv, sizeof(double) * N, cudaMemcpyDeviceToDevice, c.st));
  EXA_CUDA(cudaMemsetAsync(wv, 0, sizeof(double) * N, c.st));
  int i = 0;
  while (i < m - 1) {
    if (si[i] == 0.0) {
      EXA_TRY(exa_axpby(wv, q, 1.0 / sr[i], 1.0, N, c.st));
      EXA_TRY(pa(c, q, p));
      EXA_TRY(exa_axpby(q, p, -1.0 / sr[i], 1.0, N, c.st));
      i += 1;
    } else {
      const double a = sr[i], b = si[i], a2b2 = a * a + b * b;
      EXA_TRY(pa(c, q, p));
      EXA_TRY(exa_axpby(p, q, 2.0 * a, -1.0, N, c.st));
      EXA_TRY(exa_axpby(wv, p, 1.0 / a2b2, 1.0, N, c.st));
      if (i < m - 2) {
        EXA_TRY(pa(c, p, p));
        EXA_TRY(exa_axpby(q, p, -1.0 / a2b2, 1.0, N, c.st));
      }
      i += 2;
    }
  }
  if (si[m - 1] == 0.0) EXA_TRY(exa_axpby(wv, q, 1.0 / sr[m - 1], 1.0, N, c.st));
  return EXA_OK;
}

// v_j <- v_j orthogonalised against v_0 .. v_{j-1} by modified Gram-Schmidt and normalised,
// the coefficients into hcol[0 .. j] (MGS, getpoly.cpp:36-45; the pipelined launches of
// arnoldi_ops)
int mgs_column(ExaCtx& c, int j, double* hcol) {
  const long long N = c.sysN();
  double* vn = c.V + (long long)j * N;
  EXA_TRY(exa_dot_partials(vn, c.V, N, c.part_a, c.st));
  double* pin = c.part_a;
  double* pout = c.part_b;
  for (int k = 1; k < j; ++k) {
    EXA_TRY(exa_mgs_step(vn, c.V + (long long)(k - 1) * N, c.V + (long long)k * N, pin, pout, hcol + k - 1, N, c.st));
    std::swap(pin, pout);
  }
  EXA_TRY(exa_mgs_step(vn, c.V + (long long)(j - 1) * N, nullptr, pin, pout, hcol + j - 1, N, c.st));
  return exa_mgs_finish(vn, vn, pout, hcol + j, N, c.st);
}

// getPoly (getpoly.cpp:226-247) and the Ritz-value post-processing of GMRES (gmres.cpp:385-398):
// m = ppdegree Arnoldi steps of P A from randvect (makeH, getpoly.cpp:208-224), then on the
// host the harmonic Ritz values in Leja order (exa_poly_ritz)
int poly_setup(ExaCtx& c) {
  const int m = c.ppdegree, m1 = m + 1, n1 = c.restart + 1;
  const long long N = c.sysN();
  double nr = 0.0;
  EXA_TRY(exa_drv_norm(c, c.randvect, N, &nr));
  EXA_TRY(exa_scale(c.V, c.randvect, 1.0 / nr, N, c.st));
  for (int j = 0; j < m; ++j) {
    EXA_TRY(pa(c, c.V + (long long)j * N, c.V + (long long)(j + 1) * N));
    EXA_TRY(mgs_column(c, j + 1, c.hess + (long long)n1 * j));
  }
  EXA_CUDA(cudaMemcpyAsync(c.pinned, c.hess, sizeof(double) * n1 * m, cudaMemcpyDeviceToHost, c.st));
  EXA_CUDA(cudaStreamSynchronize(c.st));
  std::vector<double> H((size_t)m1 * m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m1; ++i) H[(size_t)i + (size_t)m1 * j] = c.pinned[(size_t)i + (size_t)n1 * j];
  c.poly_sr.assign(m, 0.0);
  c.poly_si.assign(m, 0.0);
  return exa_poly_ritz(H.data(), m, c.poly_sr.data(), c.poly_si.data());
}

// cpuBackSolve (backend/Common/cpuimpl.h:198-208)
void back_solve(double* y, const double* H, const double* s, int i, int n) {
  for (int j = i; j >= 0; j--) y[j] = s[j];
  for (int j = i; j >= 0; j--) {
    y[j] = y[j] / H[j + n * j];
    for (int k = j - 1; k >= 0; k--) y[k] = y[k] - H[k + n * j] * y[j];
  }
}

}  // namespace

namespace {

// The work of Arnoldi step i of a restart cycle, all enqueued on the context stream with
// no host synchronisation: v_{i+1} = P A v_i orthogonalised against v_0..v_i (MGS or CGS),
// the Hessenberg column i, the Givens update and the residual estimate |s_{i+1}| / |b|,
// copied to the pinned slot `rel_pin`.
int arnoldi_ops(ExaCtx& c, int i, const double* d_nrmb, double* d_relerr, double* rel_pin) {
  const long long N = c.sysN();
  const int n1 = c.restart + 1;
  double* vi = c.V + (long long)i * N;
  double* vn = c.V + (long long)(i + 1) * N;
  double* hcol = c.hess + (long long)n1 * i;
  EXA_TRY(exa_drv_matvec(c, vi, c.w));
  EXA_TRY(exa_drv_precond(c, c.w, vn));
  EXA_TRY(apply_poly(c, vn));
  {
    ExaProfScope ps_ortho(c, EXA_PH_ORTHO);
    if (c.ortho == 0) {
      EXA_TRY(exa_dot_partials(vn, c.V, N, c.part_a, c.st));
      double* pin = c.part_a;
      double* pout = c.part_b;
      for (int k = 1; k <= i; ++k) {
        EXA_TRY(exa_mgs_step(vn, c.V + (long long)(k - 1) * N, c.V + (long long)k * N, pin, pout, hcol + k - 1, N, c.st));
        std::swap(pin, pout);
      }
      EXA_TRY(exa_mgs_step(vn, c.V + (long long)i * N, nullptr, pin, pout, hcol + i, N, c.st));
      EXA_TRY(exa_mgs_finish(vn, vn, pout, hcol + i + 1, N, c.st));
    } else {
      EXA_TRY(exa_cgs(vn, c.V, hcol, c.part_m, N, i + 1, c.st));
      EXA_TRY(exa_dot_partials(vn, vn, N, c.part_a, c.st));
      EXA_TRY(exa_mgs_finish(vn, vn, c.part_a, hcol + i + 1, N, c.st));
    }
  }
  EXA_TRY(exa_givens(hcol, c.gs, c.gcs, c.gsn, i, d_nrmb, d_relerr, c.st));
  EXA_CUDA(cudaMemcpyAsync(rel_pin, d_relerr, sizeof(double), cudaMemcpyDeviceToHost, c.st));
  return EXA_OK;
}

// Enqueues Arnoldi step i.  Its first use runs the launches directly; from the second use on
// the step is one CUDA graph, captured then and replayed after, which replaces some 30
// launches (the matvec, the preconditioner, one Gram-Schmidt launch per basis vector, the
// Givens update) by one.  The graph's arguments are fixed per context: the basis column,
// the Hessenberg column, the residual slot.  Phase profiling records events between the
// launches, so it runs the launches directly.  A capture that fails leaves the context on
// direct launches.
int arnoldi_step(ExaCtx& c, int i, const double* d_nrmb, double* d_relerr, double* rel_pin) {
  const int pr = c.precision == 1 ? 1 : 0;
  // a polynomial preconditioner's Ritz values are kernel arguments and change with every
  // GMRES call, so its steps run as direct launches
  if (!c.use_graphs || c.prof.on || c.ppdegree > 1 || i >= (int)c.arnoldi_graph[pr].size())
    return arnoldi_ops(c, i, d_nrmb, d_relerr, rel_pin);
  cudaGraphExec_t& ex = c.arnoldi_graph[pr][i];
  if (ex) {
    EXA_CUDA(cudaGraphLaunch(ex, c.st));
    exa_add_launches(c.arnoldi_launches[pr][i]);
    return EXA_OK;
  }
  if (!c.arnoldi_seen[pr][i]) {
    c.arnoldi_seen[pr][i] = 1;
    return arnoldi_ops(c, i, d_nrmb, d_relerr, rel_pin);
  }
  const long long l0 = exa_thread_launches();
  EXA_CUDA(cudaStreamBeginCapture(c.st, cudaStreamCaptureModeThreadLocal));
  const int st = arnoldi_ops(c, i, d_nrmb, d_relerr, rel_pin);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c.st, &g);
  const long long nl = exa_thread_launches() - l0;
  exa_add_launches(-nl);  // counted again at each replay
  if (st == EXA_OK && e == cudaSuccess && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess) {
    cudaGraphDestroy(g);
    c.arnoldi_launches[pr][i] = nl;
    EXA_CUDA(cudaGraphLaunch(ex, c.st));
    exa_add_launches(nl);
    return EXA_OK;
  }
  if (g) cudaGraphDestroy(g);
  ex = nullptr;
  cudaGetLastError();
  c.use_graphs = 0;
  return arnoldi_ops(c, i, d_nrmb, d_relerr, rel_pin);
}

// ComputeInitialGuessAndPreconditioner (preconditioner.cpp:133-181): the image of the newest
// basis vector under the current condensed operator, U_i = A W_i, then c = (U^T U)^-1 U^T b
// (the small matrix inverted on the host by Gauss-Jordan with partial pivoting, as the
// reference inverts it with getrf/getri) and x = W c.  A singular U^T U leaves x = 0.
int rb_initial_guess(ExaCtx& c) {
  const long long N = c.sysN();
  const int cur = c.rb_cur;
  const int i = c.rb_removed > 0 ? c.rb_removed - 1 : cur - 1;
  EXA_TRY(exa_drv_matvec(c, c.rbW + (long long)i * N, c.rbU + (long long)i * N));
  int nd = 0;
  for (int j = 0; j < cur; ++j) {
    EXA_TRY(exa_dot_partials(c.rbU + (long long)j * N, c.b, N, c.part_a, c.st));
    EXA_TRY(exa_reduce_partials(c.part_a, N, c.rbD + nd++, 0, c.st));
  }
  for (int j = 0; j < cur; ++j)
    for (int k = 0; k <= j; ++k) {
      EXA_TRY(exa_dot_partials(c.rbU + (long long)j * N, c.rbU + (long long)k * N, N, c.part_a, c.st));
      EXA_TRY(exa_reduce_partials(c.part_a, N, c.rbD + nd++, 0, c.st));
    }
  std::vector<double> d(nd);
  EXA_CUDA(cudaMemcpyAsync(d.data(), c.rbD, sizeof(double) * nd, cudaMemcpyDeviceToHost, c.st));
  EXA_CUDA(cudaStreamSynchronize(c.st));
  // H = U^T U (symmetric), inverted in place
  std::vector<double> H((size_t)cur * cur), rhs(d.begin(), d.begin() + cur);
  for (int j = 0, o = cur; j < cur; ++j)
    for (int k = 0; k <= j; ++k, ++o) H[j + cur * k] = H[k + cur * j] = d[o];
  std::vector<int> used(cur, 0), perm(cur);
  for (int k = 0; k < cur; ++k) {
    int p = -1;
    double best = 0.0;
    for (int r = 0; r < cur; ++r)
      if (!used[r] && std::fabs(H[r + cur * k]) > best) { best = std::fabs(H[r + cur * k]); p = r; }
    if (p < 0) return EXA_OK;  // singular: zero initial guess
    used[p] = 1;
    perm[k] = p;
    const double dinv = 1.0 / H[p + cur * k];
    for (int j = 0; j < cur; ++j) H[p + cur * j] = (j == k) ? dinv : H[p + cur * j] * dinv;
    for (int r = 0; r < cur; ++r) {
      if (r == p) continue;
      const double f = H[r + cur * k];
      for (int j = 0; j < cur; ++j) H[r + cur * j] = (j == k) ? -f * dinv : H[r + cur * j] - f * H[p + cur * j];
    }
  }
  // entry (r, c) of the tableau is inverse(pos[r], perm[c]); coef = inverse * rhs
  std::vector<int> pos(cur);
  for (int k = 0; k < cur; ++k) pos[perm[k]] = k;
  std::vector<double> inv((size_t)cur * cur), coef(cur, 0.0);
  for (int r = 0; r < cur; ++r)
    for (int k = 0; k < cur; ++k) inv[pos[r] + cur * perm[k]] = H[r + cur * k];
  for (int r = 0; r < cur; ++r)
    for (int k = 0; k < cur; ++k) coef[r] += inv[r + cur * k] * rhs[k];
  double* cd = c.rbD;  // the dot products are consumed: reuse for the coefficients
  EXA_CUDA(cudaMemcpyAsync(cd, coef.data(), sizeof(double) * cur, cudaMemcpyHostToDevice, c.st));
  EXA_TRY(exa_gemv_add(c.x, c.rbW, cd, N, cur, c.st));
  EXA_CUDA(cudaStreamSynchronize(c.st));  // coef is host memory that goes out of scope
  return EXA_OK;
}

// UpdateRB (ptcsolver.cpp:484-500): the Newton update, scaled by its step length, replaces
// the oldest basis vector
int rb_update(ExaCtx& c, double alpha) {
  const long long N = c.sysN();
  EXA_TRY(exa_scale(c.x, c.x, alpha, N, c.st));
  double nrm = 0.0;
  EXA_TRY(exa_drv_norm(c, c.x, N, &nrm));
  if (nrm > 0.0) {
    EXA_CUDA(cudaMemcpyAsync(c.rbW + (long long)c.rb_removed * N, c.x, sizeof(double) * N, cudaMemcpyDeviceToDevice,
                             c.st));
    if (c.rb_cur < c.RBdim) c.rb_cur += 1;
    c.rb_removed = (c.rb_removed + 1) % c.RBdim;
  }
  return EXA_OK;
}

// UpdateSolution (gmres.cpp:132-137) with the first i + 1 basis vectors: y from the
// Hessenberg back-solve on the host, x += V y on the device.
int update_solution(ExaCtx& c, int i, std::vector<double>& ybuf) {
  const long long N = c.sysN();
  const int n1 = c.restart + 1, nrest = c.restart;
  double* hh = c.pinned;
  double* ss = hh + (size_t)n1 * nrest;
  EXA_CUDA(cudaMemcpyAsync(hh, c.hess, sizeof(double) * n1 * nrest, cudaMemcpyDeviceToHost, c.st));
  EXA_CUDA(cudaMemcpyAsync(ss, c.gs, sizeof(double) * n1, cudaMemcpyDeviceToHost, c.st));
  EXA_CUDA(cudaStreamSynchronize(c.st));
  back_solve(ybuf.data(), hh, ss, i, n1);
  double* yd = c.part_m;  // device copy of the back-solve result (part_m holds >= restart+1 doubles)
  EXA_CUDA(cudaMemcpyAsync(yd, ybuf.data(), sizeof(double) * (i + 1), cudaMemcpyHostToDevice, c.st));
  EXA_TRY(exa_gemv_add(c.x, c.V, yd, N, i + 1, c.st));
  return EXA_OK;
}

}  // namespace

// GMRES (gmres.cpp:361-597): restarted, left-preconditioned, MGS (flag 0) or CGS (flag 1).
// Solves A x = b for the current system; x starts at zero (no reduced basis).
// The host reads each step's residual estimate one step late: step i + 1 is enqueued before
// the estimate of step i is read, so the device does not wait for the host between steps.
// When step i has converged, step i + 1 has run as well; it writes only basis column i + 2,
// Hessenberg column i + 1 and Givens entries i + 1 and i + 2, none of which the solution
// update of step i reads, so the result is that of stopping at step i.
namespace {
int gmres_body(ExaCtx& c, int* iters_out, double* relerr_out) {
  const long long N = c.sysN();
  const int nrest = c.restart, maxit = c.gmres_maxit, n1 = nrest + 1;
  double nrmb = 0.0, nrmr = 0.0;
  // the polynomial's Ritz values, from the current operator (gmres.cpp:385-398)
  if (c.ppdegree > 1) EXA_TRY(poly_setup(c));
  if (!c.gmres_x_preset) EXA_CUDA(cudaMemsetAsync(c.x, 0, sizeof(double) * N, c.st));
  EXA_TRY(exa_drv_norm(c, c.b, N, &nrmb));
  c.last_gmres_converged = true;
  // the HDG solve stops at a right-hand side below the Newton tolerance; the LDG GMRES
  // (gmres.cpp:140-318) has no such test
  if (c.scheme != 0 && nrmb < c.newton_tol) {
    *iters_out = 0;
    *relerr_out = 0.0;
    return EXA_OK;
  }
  // initial guess from the reduced basis (LinearSolver, ptcsolver.cpp:374-379); a guess of
  // norm at most 1e-12 counts as none, as in gmres.cpp:404-421
  if (!c.gmres_x_preset && c.RBdim > 0 && c.rb_cur > 0) EXA_TRY(rb_initial_guess(c));
  double scalar = 0.0;
  if (c.gmres_x_preset || (c.RBdim > 0 && c.rb_cur > 0)) EXA_TRY(exa_drv_norm(c, c.x, N, &scalar));
  if (scalar > 1e-12) {
    EXA_TRY(exa_drv_matvec(c, c.x, c.w));
    EXA_TRY(exa_axpby(c.w, c.b, 1.0, -1.0, N, c.st));  // w = b - A x
    EXA_TRY(exa_drv_norm(c, c.w, N, &nrmr));
  } else {
    nrmr = nrmb;  // r = b
  }
  const double tol = std::min(0.1, c.gmres_tol * (nrmb / nrmr));
  EXA_TRY(exa_drv_precond(c, scalar > 1e-12 ? c.w : c.b, c.r));
  EXA_TRY(apply_poly(c, c.r));
  EXA_TRY(exa_drv_norm(c, c.r, N, &nrmb));
  nrmr = nrmb;
  // device copy of nrmb for the Givens kernel
  double* d_nrmb = c.scal + 14;
  double* d_relerr = c.scal + 13;
  double* rel_pin = c.pinned + (size_t)n1 * (n1 + 2) + 64;  // one slot per step of a cycle
  c.pinned[0] = nrmb;
  EXA_CUDA(cudaMemcpyAsync(d_nrmb, c.pinned, sizeof(double), cudaMemcpyHostToDevice, c.st));
  std::vector<double> ybuf(n1);
  int j = 0;
  double relerr = 1.0;
  while (j < maxit) {
    EXA_TRY(exa_scale(c.V, c.r, 1.0 / nrmr, N, c.st));
    std::vector<double> s0(n1, 0.0);
    s0[0] = nrmr;
    std::copy(s0.begin(), s0.end(), c.pinned);
    EXA_CUDA(cudaMemcpyAsync(c.gs, c.pinned, sizeof(double) * n1, cudaMemcpyHostToDevice, c.st));
    int i = 0, pending = -1;
    for (i = 0; i < nrest && j < maxit; i++, j++) {
      EXA_TRY(arnoldi_step(c, i, d_nrmb, d_relerr, rel_pin + i));
      EXA_CUDA(cudaEventRecord(c.step_ev[i & 1], c.st));
      if (pending >= 0) {
        EXA_CUDA(cudaEventSynchronize(c.step_ev[pending & 1]));
        relerr = rel_pin[pending];
        if (relerr < tol) {
          EXA_TRY(update_solution(c, pending, ybuf));
          EXA_CUDA(cudaStreamSynchronize(c.st));
          *iters_out = j;
          *relerr_out = relerr;
          return EXA_OK;
        }
      }
      pending = i;
    }
    if (pending >= 0) {
      EXA_CUDA(cudaEventSynchronize(c.step_ev[pending & 1]));
      relerr = rel_pin[pending];
      if (relerr < tol) {
        EXA_TRY(update_solution(c, pending, ybuf));
        EXA_CUDA(cudaStreamSynchronize(c.st));
        *iters_out = j;
        *relerr_out = relerr;
        return EXA_OK;
      }
    }
    EXA_TRY(update_solution(c, i - 1, ybuf));
    // r = P (b - A x)
    EXA_TRY(exa_drv_matvec(c, c.x, c.w));
    EXA_TRY(exa_axpby(c.w, c.b, 1.0, -1.0, N, c.st));
    EXA_TRY(exa_drv_precond(c, c.w, c.r));
    EXA_TRY(apply_poly(c, c.r));
    EXA_TRY(exa_drv_norm(c, c.r, N, &nrmr));
    relerr = nrmr / nrmb;
    if (relerr < tol) {
      *iters_out = j;
      *relerr_out = relerr;
      return EXA_OK;
    }
  }
  *iters_out = j;
  *relerr_out = relerr;
  c.last_gmres_converged = false;
  return EXA_OK;  // not converged: the reference warns and continues (gmres.cpp:586-594)
}
}  // namespace

// The mixed form's FP32 block products stream through shared memory with bounded waits
// (d_flag[1] set when one ran out); read after the work that used them.
int exa_drv_check_uflag(ExaCtx& c) {
  if (c.precision != 1 || !c.d_uflag) return EXA_OK;
  int f = 0;
  EXA_CUDA(cudaMemcpyAsync(c.pinned, c.d_uflag, sizeof(int), cudaMemcpyDeviceToHost, c.st));
  EXA_CUDA(cudaStreamSynchronize(c.st));
  std::memcpy(&f, c.pinned, sizeof(int));
  if (f) {
    exa_set_error("FP32 block product: a wait inside the kernel ran out");
    return EXA_ERR_CUDA;
  }
  return EXA_OK;
}

int exa_drv_gmres(ExaCtx& c, int* iters_out, double* relerr_out) {
  if (c.batcher && c.scheme != 0 && exa_batchable(c)) {
    EXA_TRY(exa_batcher_gmres(c.batcher, c, iters_out, relerr_out));
  } else {
    EXA_TRY(gmres_body(c, iters_out, relerr_out));
  }
  return exa_drv_check_uflag(c);
}

int exa_drv_gmres_update(ExaCtx& c, int i) {
  std::vector<double> ybuf(c.restart + 1);
  EXA_TRY(update_solution(c, i, ybuf));
  EXA_CUDA(cudaStreamSynchronize(c.st));  // ybuf's host copy is consumed
  return EXA_OK;
}

// PTCsolver (ptcsolver.cpp:255-330) with LinearSolver (ptcsolver.cpp:53-120) for the LDG
// discretisation: GMRES on J(u) x = -R(u) from x = 0, u += x, until |R(u)| < the tolerance;
// a norm above 1e6 or NaN stops it (the reference writes the state and exits there).
// iters_out counts the PTC steps taken.
int exa_drv_ptc(ExaCtx& c, int* iters_out, double* norm_out) {
  const long long N = c.sysN();
  double nrmr = 0.0;
  EXA_TRY(exa_model_ldg_residual(c, c.udg, c.ldg_R));
  EXA_TRY(exa_drv_norm(c, c.ldg_R, N, &nrmr));
  c.last_norm0 = nrmr;
  c.total_gmres_iters = 0;
  int it = 0;
  for (it = 0; it < c.newton_maxit; ++it) {
    EXA_TRY(exa_scale(c.b, c.ldg_R, -1.0, N, c.st));  // J x = -R(u)
    // LinearSolver (ptcsolver.cpp:53-97): with a reduced basis, its guess x (the HDG solve's
    // formula with b = -R gives the reference's x = -W coef) is kept only if R(u + x) is at most
    // 1.05 |R(u)| (else x = 0 and the basis is emptied); below the tolerance it is the step
    int status = 0;
    const bool rb = c.RBdim > 0 && c.rb_cur > 0;
    if (rb) {
      const double oldnrm = nrmr;
      double nv = 0.0;
      EXA_CUDA(cudaMemsetAsync(c.x, 0, sizeof(double) * N, c.st));
      EXA_TRY(rb_initial_guess(c));
      EXA_TRY(exa_lincomb(c.ldg_w, 1.0, c.udg, 1.0, c.x, N, c.st));
      EXA_TRY(exa_model_ldg_residual(c, c.ldg_w, c.ldg_Rw));
      EXA_TRY(exa_drv_norm(c, c.ldg_Rw, N, &nv));
      if (nv > 1.05 * oldnrm) {
        EXA_TRY(exa_scale(c.x, c.x, 0.0, N, c.st));
        c.rb_removed = 0;
        c.rb_cur = 0;
      }
      if (nv < c.newton_tol) status = 1;
    }
    int gi = 0;
    double ge = 0.0;
    if (status == 0) {
      c.gmres_x_preset = rb ? 1 : 0;
      const int gs = exa_drv_gmres(c, &gi, &ge);
      c.gmres_x_preset = 0;
      EXA_TRY(gs);
    }
    c.last_gmres_iters = gi;
    c.last_gmres_relerr = ge;
    c.total_gmres_iters += gi;
    {
      ExaProfScope ps(c, EXA_PH_UPDATE);
      EXA_TRY(exa_axpby(c.udg, c.x, 1.0, 1.0, N, c.st));
    }
    EXA_TRY(exa_model_ldg_residual(c, c.udg, c.ldg_R));
    EXA_TRY(exa_drv_norm(c, c.ldg_R, N, &nrmr));
    c.last_newton_iters = it + 1;
    if (status == 0 && c.RBdim > 0) EXA_TRY(rb_update(c, 1.0));  // UpdateRB (ptcsolver.cpp:207-226)
    if (!(nrmr <= 1.0e6)) {
      exa_set_error("PTC residual norm %g is above 1e6 or NaN", nrmr);
      *iters_out = it + 1;
      *norm_out = nrmr;
      return std::isnan(nrmr) ? EXA_ERR_NAN : EXA_ERR_NOTCONV;
    }
    if (nrmr < c.newton_tol) {
      *iters_out = it + 1;
      *norm_out = nrmr;
      c.last_norm = nrmr;
      return EXA_OK;
    }
  }
  *iters_out = it;
  *norm_out = nrmr;
  c.last_norm = nrmr;
  return EXA_OK;
}

// NewtonSolver (solution.cpp:125-243)
int exa_drv_newton(ExaCtx& c, int* iters_out, double* norm_out) {
  if (c.scheme == 0) return exa_drv_ptc(c, iters_out, norm_out);
  if (c.precision == 1) return exa_drv_newton_mixed(c, iters_out, norm_out);
  const ExaDims& P = c.P;
  const long long N = c.ndofuhat();
  double nrmr = 0.0;
  EXA_TRY(exa_drv_getq(c));
  EXA_TRY(exa_drv_residual(c, &nrmr));
  c.last_norm0 = nrmr;
  c.total_gmres_iters = 0;
  for (int it = 0; it < c.newton_maxit; ++it) {
    EXA_TRY(exa_drv_assemble(c));
    int gi = 0;
    double ge = 0.0;
    EXA_TRY(exa_drv_gmres(c, &gi, &ge));
    c.last_gmres_iters = gi;
    c.last_gmres_relerr = ge;
    c.total_gmres_iters += gi;
    double alpha = 1.0;
    {
      // u += alpha x; uhat = u; du = Ru + DinvF x; udg(u) += alpha du
      ExaProfScope ps(c, EXA_PH_UPDATE);
      EXA_TRY(exa_axpby(c.uh, c.x, alpha, 1.0, N, c.st));
      EXA_TRY(exa_k_dudg(P, c.elemcon, c.F, c.Ru, c.x, c.du, c.st));
      EXA_TRY(exa_k_udg_update(P, c.udg, c.du, alpha, c.st));
    }
    EXA_TRY(exa_drv_getq(c));
    const double nrm0 = nrmr;
    EXA_TRY(exa_drv_residual(c, &nrmr));
    if (nrmr > nrm0 && nrmr > 1.0e6) {
      exa_set_error("Residual norm increases more than 1e6 (%g -> %g)", nrm0, nrmr);
      *iters_out = it + 1;
      *norm_out = nrmr;
      return EXA_ERR_NOTCONV;
    }
    while ((nrmr > nrm0 && alpha > 0.1) || std::isnan(nrmr)) {
      alpha = alpha / 2.0;
      EXA_TRY(exa_axpby(c.uh, c.x, -alpha, 1.0, N, c.st));
      EXA_TRY(exa_k_udg_update(P, c.udg, c.du, -alpha, c.st));
      EXA_TRY(exa_drv_getq(c));
      EXA_TRY(exa_drv_residual(c, &nrmr));
      if (alpha < 1e-12) break;
    }
    if (c.RBdim > 0) EXA_TRY(rb_update(c, alpha));
    c.last_newton_iters = it + 1;
    if (std::isnan(nrmr)) {
      exa_set_error("Newton residual is NaN");
      *iters_out = it + 1;
      *norm_out = nrmr;
      return EXA_ERR_NAN;
    }
    if (nrmr < c.newton_tol) {
      *iters_out = it + 1;
      *norm_out = nrmr;
      c.last_norm = nrmr;
      return EXA_OK;
    }
  }
  *iters_out = c.newton_maxit;
  *norm_out = nrmr;
  c.last_norm = nrmr;
  return EXA_OK;
}

// Condensed right-hand side of the mixed form from the FP64 residual (Ru, Rh) of the
// current state: Ru <- D^-1 Ru and Rh <- Rh - K Ru with the FP32 factors of the last
// assembly, then b = scatter(Rh).
int exa_drv_condense_mixed(ExaCtx& c) {
  const ExaDims& P = c.P;
  const int n = P.n, m = P.m;
  ExaProfScope ps(c, EXA_PH_UPDATE);
  // in element chunks of the assembly's workspace (c.wRu holds neb element vectors)
  for (int e0 = 0; e0 < P.ne; e0 += c.neb) {
    const int nb = std::min(c.neb, P.ne - e0);
    double* Ruc = c.Ru + (long long)e0 * n;
    EXA_CUDA(cudaMemcpyAsync(c.wRu, Ruc, sizeof(double) * (size_t)n * nb, cudaMemcpyDeviceToDevice, c.st));
    EXA_TRY(exa_k_gemv32(n, n, nb, 1.0, c.Dinv32 + (long long)e0 * n * n, (long long)n * n, c.wRu, n, 0.0, Ruc, n,
                         c.st, c.d_uflag));
    EXA_TRY(exa_k_gemv32(m, n, nb, -1.0, c.K32 + (long long)e0 * m * n, (long long)m * n, Ruc, n, 1.0,
                         c.Rh + (long long)e0 * m, m, c.st, c.d_uflag));
  }
  return exa_k_scatter(P, c.f2e, c.elemcon, c.Rh, c.b, c.st);
}

// Mixed-precision Newton solve: one assembly of the FP32 Jacobian blocks, then steps
//   solve A32 x = b (GMRES to mixed_inner_tol), uhat += x, u += D^-1 Ru + D^-1 F x,
//   FP64 residual, FP64 condensed right-hand side through the FP32 factors,
// until the FP64 residual norm |b| + |Ru| (solution.cpp:148-157) has dropped by the target
// ratio (mixed_rtol, or the GMRES tolerance when it is 0), or has stopped falling below the
// absolute Newton tolerance.  The FP64 residual at every step makes the FP32 solve an
// iterative refinement of the FP64 Newton step.
int exa_drv_newton_mixed(ExaCtx& c, int* iters_out, double* norm_out) {
  const ExaDims& P = c.P;
  const long long N = c.ndofuhat();
  const double rtol = c.mixed_rtol > 0.0 ? c.mixed_rtol : c.gmres_tol;
  double nrmr = 0.0;
  EXA_TRY(exa_drv_getq(c));
  EXA_TRY(exa_drv_residual(c, &nrmr));
  const double nrm0 = nrmr;
  c.last_norm0 = nrm0;
  c.total_gmres_iters = 0;
  if (!(nrm0 > 0.0)) {
    *iters_out = 0;
    *norm_out = nrm0;
    c.last_norm = nrm0;
    return std::isnan(nrm0) ? EXA_ERR_NAN : EXA_OK;
  }
  EXA_TRY(exa_drv_assemble(c));
  const double gtol = c.gmres_tol;
  double prev = nrm0;
  int it = 0;
  for (it = 0; it < c.mixed_maxit; ++it) {
    int gi = 0;
    double ge = 0.0;
    // the inner solves see the small right-hand sides of late steps: no absolute cut-off
    const double ntol = c.newton_tol;
    c.gmres_tol = c.mixed_inner_tol;
    c.newton_tol = 0.0;
    const int st = exa_drv_gmres(c, &gi, &ge);
    c.gmres_tol = gtol;
    c.newton_tol = ntol;
    EXA_TRY(st);
    c.last_gmres_iters = gi;
    c.last_gmres_relerr = ge;
    c.total_gmres_iters += gi;
    {
      ExaProfScope ps(c, EXA_PH_UPDATE);
      EXA_TRY(exa_axpby(c.uh, c.x, 1.0, 1.0, N, c.st));
      EXA_TRY(exa_k_dudg(P, c.elemcon, c.F32, c.Ru, c.x, c.du, c.st, c.d_uflag));
      EXA_TRY(exa_k_udg_update(P, c.udg, c.du, 1.0, c.st));
      if (c.RBdim > 0) EXA_TRY(rb_update(c, 1.0));
    }
    EXA_TRY(exa_drv_getq(c));
    EXA_TRY(exa_drv_residual(c, &nrmr));
    c.last_newton_iters = it + 1;
    if (std::isnan(nrmr)) {
      exa_set_error("mixed-precision refinement: residual is NaN");
      *iters_out = it + 1;
      *norm_out = nrmr;
      c.last_norm = nrmr;
      return EXA_ERR_NAN;
    }
    if (nrmr <= rtol * nrm0) break;
    // a residual already below the absolute Newton tolerance that no longer falls has
    // reached the FP64 round-off floor (a solve started from a converged state)
    const bool floor = nrmr < c.newton_tol && nrmr > 0.5 * prev;
    prev = nrmr;
    if (floor) break;
    EXA_TRY(exa_drv_condense_mixed(c));
  }
  *iters_out = std::min(it + 1, c.mixed_maxit);
  *norm_out = nrmr;
  c.last_norm = nrmr;
  EXA_TRY(exa_drv_check_uflag(c));  // the updates' and condensations' FP32 products
  if (nrmr > rtol * nrm0 && !(nrmr < c.newton_tol)) {
    exa_set_error("mixed-precision refinement stopped at residual ratio %.3e after %d steps", nrmr / nrm0,
                  c.mixed_maxit);
    return EXA_ERR_NOTCONV;
  }
  return EXA_OK;
}

namespace {
// DIRK tables (timestepcoeff.cpp:35-104): c, d (column-major nstage x nstage), t
bool dirk_coeff(int nstage, int torder, std::vector<double>& cc, std::vector<double>& d, std::vector<double>& t) {
  if (nstage == 1 && torder == 1) { cc = {1.0}; d = {1.0}; t = {1.0}; return true; }
  if (nstage == 1 && torder == 2) { cc = {2.0}; d = {2.0}; t = {0.5}; return true; }
  if (nstage == 2 && torder == 2) {
    d = {3.414213562373096, -8.242640687119289, 0.0, 3.414213562373096}; cc = {0.0, 1.0};
    t = {0.292893218813452, 1.0}; return true;
  }
  if (nstage == 2 && torder == 3) {
    d = {1.267949192431123, 0.928203230275509, 0.0, 1.267949192431123}; cc = {1.098076211353316, 0.633974596215561};
    t = {0.788675134594813, 0.211324865405187}; return true;
  }
  if (nstage == 3 && torder == 3) {
    d = {2.294280360323567, -1.484721005721436, -8.556127801733982, 0.0, 2.294280360323568, 3.391748836909791,
         0.0, 0.0, 2.294280360323567};
    cc = {0.0, 0.0, 1.0}; t = {0.435866521500000, 0.717933260750000, 1.000000000000000}; return true;
  }
  if (nstage == 3 && torder == 4) {
    d = {0.935822227524088, 0.497940606760015, -0.345865915800969, 0.0, 0.935822227524088, 2.867525668568206,
         0.0, 0.0, 0.935822227524088};
    cc = {0.445622407287714, 1.064177772475912, 0.120614758428183};
    t = {1.068579021301629, 0.500000000000000, -0.068579021301629}; return true;
  }
  return false;
}

__global__ void extract_u_kernel(ExaDims P, const double* udg, double* u) {
  const long long N = (long long)P.n * P.ne;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N; idx += (long long)gridDim.x * blockDim.x)
    u[idx] = udg[idx % P.n + (long long)P.npe * P.nc * (idx / P.n)];
}
__global__ void insert_u_kernel(ExaDims P, double* udg, const double* u) {
  const long long N = (long long)P.n * P.ne;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N; idx += (long long)gridDim.x * blockDim.x)
    udg[idx % P.n + (long long)P.npe * P.nc * (idx / P.n)] = u[idx];
}
}  // namespace

// One DIRK stage around Newton (exasim.hpp:413-482): PreviousSolutions at stage 0
// (previoussolutions.cpp:23-45), UpdateSourceDIRK (updatesource.cpp:32-80), the Newton
// solve, and the stage accumulation of UpdateSolution (updatesolution.cpp:118-140).
// `time0` is the time at the start of step `istep`.
int exa_drv_dirk_stage(ExaCtx& c, int istep, int j, int* its_out, double* norm_out) {
  if (!c.tdep) { exa_set_error("app.bin is not time dependent"); return EXA_ERR_ARG; }
  std::vector<double> cc, d, t;
  if (!dirk_coeff(c.nstage, c.torder, cc, d, t)) { exa_set_error("DIRK(%d,%d) is not tabulated", c.nstage, c.torder); return EXA_ERR_UNSUPPORTED; }
  if (istep < 0 || istep >= (int)c.dt.size()) { exa_set_error("step %d beyond the dt list", istep); return EXA_ERR_ARG; }
  if (j < 0 || j >= c.nstage) { exa_set_error("stage %d out of range", j); return EXA_ERR_ARG; }
  const ExaDims& P = c.P;
  const int S = c.nstage;
  const long long Nu = (long long)P.n * P.ne;
  const int blocks = 1024;
  const double dt = c.dt[istep];
  if (j == 0) {
    double csum = 1.0;
    for (int k = 0; k < S; ++k) csum -= cc[k];
    extract_u_kernel<<<blocks, 256, 0, c.st>>>(P, c.udg, c.udgprev);
    EXA_LAUNCH_CHECK();
    EXA_TRY(exa_scale(c.utmp, c.udgprev, csum, Nu, c.st));
  }
  c.time = c.time0 + dt * t[j];
  c.dtfactor = d[j * S + j] / dt;
  extract_u_kernel<<<blocks, 256, 0, c.st>>>(P, c.udg, c.du);
  EXA_LAUNCH_CHECK();
  if (j == 0) {
    EXA_TRY(exa_scale(c.sdg, c.du, d[0] / dt, Nu, c.st));
  } else if (j == 1) {
    const double sc = (d[1] + d[S + 1]) / d[0];
    EXA_TRY(exa_axpby(c.sdg, c.du, -d[1] / dt, sc, Nu, c.st));
  } else if (j == 2) {
    const double sc = d[2] / d[1];
    const double pc = d[2] + d[S + 2] + d[2 * S + 2] - sc * (d[1] + d[S + 1]);
    EXA_TRY(exa_axpby(c.sdg, c.du, -d[S + 2] / dt, sc, Nu, c.st));
    EXA_TRY(exa_axpby(c.sdg, c.udgprev, pc / dt, 1.0, Nu, c.st));
  } else {
    exa_set_error("DIRK with more than 3 stages");
    return EXA_ERR_UNSUPPORTED;
  }
  int its = 0;
  double nrm = 0.0;
  EXA_TRY(exa_drv_newton(c, &its, &nrm));
  if (its_out) *its_out = its;
  if (norm_out) *norm_out = nrm;
  extract_u_kernel<<<blocks, 256, 0, c.st>>>(P, c.udg, c.du);
  EXA_LAUNCH_CHECK();
  EXA_TRY(exa_axpby(c.utmp, c.du, cc[j], 1.0, Nu, c.st));
  if (j == S - 1) {
    insert_u_kernel<<<blocks, 256, 0, c.st>>>(P, c.udg, c.utmp);
    EXA_LAUNCH_CHECK();
    c.time0 = c.time0 + dt;
  }
  return EXA_OK;
}

// nsteps DIRK steps (exasim.hpp:413-482)
int exa_drv_dirk(ExaCtx& c, int nsteps, int* its_out, int max_out) {
  int count = 0;
  for (int istep = 0; istep < nsteps; ++istep) {
    for (int j = 0; j < c.nstage; ++j) {
      int its = 0;
      EXA_TRY(exa_drv_dirk_stage(c, istep, j, &its, nullptr));
      if (its_out && count < max_out) its_out[count] = its;
      ++count;
    }
  }
  EXA_CUDA(cudaStreamSynchronize(c.st));
  return EXA_OK;
}

// Model-specific translation unit: instantiates the assembly kernels for one
// generated model (header produced by exasim_b200/modelc.py, selected at build time
// with -DEXA_MODEL_HEADER="..." -DEXA_MODEL_NS=exa_model_<name>) and runs the
// element-block loop of hdgAssembleLinearSystem / hdgAssembleResidual
// (backend/Discretization/uequation.cpp:778-787, 1080-1088).
#include <vector>

#include "exa_assembly.cuh"
#include "exa_ldg.cuh"
#include "exa_solver.cuh"
#include "exa_umma.cuh"
#include EXA_MODEL_HEADER

EXA_BIND_MODEL(EXA_MODEL_NS)

namespace {

AsmArgs make_args(const ExaCtx& c, int e0) {
  AsmArgs A{};
  A.P = c.P;
  A.shapegt = c.shapegt; A.shapegw = c.shapegw; A.shapfgt = c.shapfgt; A.shapfgw = c.shapfgw;
  A.perm = c.perm; A.elemcon = c.elemcon; A.bf = c.bf;
  A.elemg = c.elemg; A.faceg = c.faceg;
  A.uinf = c.uinf; A.param = c.param; A.tau = c.tau;
  A.udg = c.udg; A.uh = c.uh; A.sdg = c.sdg;
  A.time = c.time; A.dtfactor = c.dtfactor;
  A.tdep = c.tdep; A.tdfunc = c.tdfunc; A.sourcefunc = c.sourcefunc; A.modelnumber = c.modelnumber;
  A.e0 = e0;
  return A;
}

int smem_attr(const void* fn, size_t bytes) {
  EXA_TRY(exa_allow_smem(fn, bytes));
  return EXA_OK;
}

// The element inverse needs D alone, so once the q-elimination product into D is done it
// runs on the context's second stream, beside the three products into F, K and H: its pivot
// loop is latency-bound and the products are HBM- or tensor-bound.  With phase profiling on,
// everything stays on the context stream, so the phase events time each step alone.
bool overlap_inverse(const ExaCtx& c) { return c.P.ncq > 0 && c.st2 && !c.prof.on; }

// The context stream joins the second stream before any later work, on every path out of a
// Schur step (an early error return included), so nothing it runs next can overlap it.
struct InverseJoin {
  ExaCtx& c;
  bool pending = false;
  ~InverseJoin() {
    if (pending) cudaStreamWaitEvent(c.st, c.ev_inv, 0);
  }
  int join() {
    pending = false;
    EXA_CUDA(cudaStreamWaitEvent(c.st, c.ev_inv, 0));
    return EXA_OK;
  }
};

template <class Fn>
int inverse_beside(ExaCtx& c, InverseJoin& j, Fn&& fn) {
  EXA_CUDA(cudaEventRecord(c.ev_q, c.st));
  EXA_CUDA(cudaStreamWaitEvent(c.st2, c.ev_q, 0));
  j.pending = true;
  const int st = fn(c.st2);
  // recorded whatever fn returned, so the join covers whatever it enqueued; if the record
  // itself fails, the second stream is drained here, so that nothing left on it can outlive
  // this step (the join would otherwise wait on the previous step's event)
  const cudaError_t e = cudaEventRecord(c.ev_inv, c.st2);
  if (e != cudaSuccess) {
    j.pending = false;
    cudaStreamSynchronize(c.st2);
    exa_set_error("cudaEventRecord on the second stream: %s", cudaGetErrorString(e));
    return EXA_ERR_CUDA;
  }
  return st;
}

// Schur condensation of one chunk (uequation.cpp:559-775): q-elimination, D^-1, DinvF,
// Ru <- D^-1 Ru, H += K DinvF, Rh -= K Ru.
int schur_chunk(ExaCtx& c, int e0, int nb) {
  const ExaDims& P = c.P;
  const int n = P.n, m = P.m, npe = P.npe, nd = P.nd, ncu = P.ncu, ndf = P.ndf;
  const long long nqn = (long long)npe * nd * ncu;
  double* Hc = c.H + (long long)e0 * m * m;
  const bool overlap = overlap_inverse(c);
  InverseJoin join{c};
  if (P.ncq > 0) {
    ExaProfScope ps(c, EXA_PH_QELIM);
    // four GEMMs per trace component with K = npe*nd: (n + m) rows x (npe + ndf) columns in all
    exa_prof_flops(c, EXA_PH_QELIM, 2.0 * nb * ncu * (double)npe * nd * (double)(n + m) * (npe + ndf));
    const double* MC = c.MC + (long long)e0 * npe * npe * nd;
    const double* ME = c.ME + (long long)e0 * npe * ndf * nd;
    // contraction over the stacked (l, d) rows of MinvC / MinvE (K = npe*nd), one GEMM per
    // block and per trace component b (batch2 = ncu)
    const long long kq = (long long)npe * nd;
    GemmBatch g{};
    g.batch = nb; g.batch2 = ncu;
    g.K = (int)kq; g.beta = 1.0;
    // D(:, j + npe*b) += sum_(l,d) B(:, l + npe*d + npe*nd*b) MinvC(l, d, j)
    g.M = n; g.N = npe; g.alpha = 1.0;
    g.A = c.wB; g.lda = n; g.sA = (long long)n * nqn; g.sA2 = (long long)n * kq;
    g.B = MC; g.ldb = kq; g.sB = kq * npe; g.sB2 = 0;
    g.C = c.wD; g.ldc = n; g.sC = (long long)n * n; g.sC2 = (long long)n * npe;
    EXA_TRY(exa_gemm(g, c.st));
    if (overlap) EXA_TRY(inverse_beside(c, join, [&](cudaStream_t s) {
      return exa_inverse_ws(c.wD, n, (long long)n * n, nb, c.wInv, c.d_flag, s);
    }));
    // F(:, b + ncu*jf) -= sum_(l,d) B(:, l + npe*d + npe*nd*b) MinvE(l, d, jf)
    g.N = ndf; g.alpha = -1.0;
    g.B = ME; g.ldb = kq; g.sB = kq * ndf;
    g.C = c.wF; g.ldc = (long long)n * ncu; g.sC = (long long)n * m; g.sC2 = n;
    EXA_TRY(exa_gemm(g, c.st));
    // K(:, j + npe*b) += sum_(l,d) G(:, l + npe*d + npe*nd*b) MinvC(l, d, j)
    g.M = m; g.N = npe; g.alpha = 1.0;
    g.A = c.wG; g.lda = m; g.sA = (long long)m * nqn; g.sA2 = (long long)m * kq;
    g.B = MC; g.ldb = kq; g.sB = kq * npe;
    g.C = c.wK; g.ldc = m; g.sC = (long long)m * n; g.sC2 = (long long)m * npe;
    EXA_TRY(exa_gemm(g, c.st));
    // H(:, b + ncu*jf) -= sum_(l,d) G(:, l + npe*d + npe*nd*b) MinvE(l, d, jf)
    g.N = ndf; g.alpha = -1.0;
    g.B = ME; g.ldb = kq; g.sB = kq * ndf;
    g.C = Hc; g.ldc = (long long)m * ncu; g.sC = (long long)m * m; g.sC2 = m;
    EXA_TRY(exa_gemm(g, c.st));
  }
  if (overlap) {
    EXA_TRY(join.join());
  } else {
    ExaProfScope ps(c, EXA_PH_INVERSE);
    EXA_TRY(exa_inverse_ws(c.wD, n, (long long)n * n, nb, c.wInv, c.d_flag, c.st));
  }
  ExaProfScope ps(c, EXA_PH_SCHUR);
  exa_prof_flops(c, EXA_PH_SCHUR, 2.0 * nb * ((double)n * n * m + (double)n * n + (double)m * m * n + (double)m * n));
  GemmBatch g{};
  g.batch = nb; g.batch2 = 1;
  // DinvF = -Dinv F
  g.M = n; g.N = m; g.K = n; g.alpha = -1.0; g.beta = 0.0;
  g.A = c.wD; g.lda = n; g.sA = (long long)n * n;
  g.B = c.wF; g.ldb = n; g.sB = (long long)n * m;
  g.C = c.F + (long long)e0 * n * m; g.ldc = n; g.sC = (long long)n * m;
  EXA_TRY(exa_gemm(g, c.st));
  // Ru = Dinv Ru
  double* Ruc = c.Ru + (long long)e0 * n;
  EXA_CUDA(cudaMemcpyAsync(c.wRu, Ruc, sizeof(double) * (size_t)n * nb, cudaMemcpyDeviceToDevice, c.st));
  g.N = 1; g.alpha = 1.0;
  g.B = c.wRu; g.ldb = n; g.sB = n;
  g.C = Ruc; g.ldc = n; g.sC = n;
  EXA_TRY(exa_gemm(g, c.st));
  // H += K DinvF
  g.M = m; g.N = m; g.K = n; g.alpha = 1.0; g.beta = 1.0;
  g.A = c.wK; g.lda = m; g.sA = (long long)m * n;
  g.B = c.F + (long long)e0 * n * m; g.ldb = n; g.sB = (long long)n * m;
  g.C = Hc; g.ldc = m; g.sC = (long long)m * m;
  EXA_TRY(exa_gemm(g, c.st));
  // Rh -= K Ru
  g.N = 1; g.alpha = -1.0;
  g.B = Ruc; g.ldb = n; g.sB = n;
  g.C = c.Rh + (long long)e0 * m; g.ldc = m; g.sC = m;
  EXA_TRY(exa_gemm(g, c.st));
  return EXA_OK;
}

// Mixed-precision Schur condensation of one chunk: the steps of schur_chunk with the
// products in 3xTF32 on the tensor cores (FP32 accumulation) over operands packed in the
// tensor-core layout, and the results kept in FP32: Dinv32 = D^-1, F32 = -D^-1 F,
// K32 = K, H32 = H + K D^-1 F.  The GEMM epilogues write each result both where the
// solver reads it and packed for the next product.  Ru <- D^-1 Ru and Rh <- Rh - K Ru stay
// FP64 vectors (FP32 matrices, FP64 accumulation).
int schur_chunk_mixed(ExaCtx& c, int e0, int nb) {
  const ExaDims& P = c.P;
  const int n = P.n, m = P.m, npe = P.npe, nd = P.nd, ncu = P.ncu, ndf = P.ndf;
  const long long nqn = (long long)npe * nd * ncu;
  float* D32 = c.Dinv32 + (long long)e0 * n * n;
  float* K32 = c.K32 + (long long)e0 * m * n;
  float* H32 = c.H32 + (long long)e0 * m * m;
  float* F32 = c.F32 + (long long)e0 * n * m;
  const double* Hc = c.fp64_full ? c.H + (long long)e0 * m * m : c.H;  // per-chunk staging in the mixed form
  const bool overlap = overlap_inverse(c);
  InverseJoin join{c};
  // D^-1 in FP32 (the recursive blocked form with its products on the tensor cores where
  // the order exceeds the register kernel's, else the register kernel), then packed
  auto inverse = [&](cudaStream_t s) -> int {
    if (c.wInvPk)
      EXA_TRY(exa_inverse_tc32(D32, n, (long long)n * n, nb, c.wInv32, c.wInvPk, c.d_flag, c.d_uflag, s));
    else
      EXA_TRY(exa_inverse_ws(D32, n, (long long)n * n, nb, reinterpret_cast<float*>(c.wInv), c.d_flag, s));
    return EXA_OK;
  };
  auto pack_dinv = [&](cudaStream_t s) { return exa_pack(D32, 0, 1, n, (long long)n * n, 0, nb, 1, c.Dinvp, s); };
  auto at = [](UPacked u, long long e) {  // operand of element e of the set
    u.hi += e * u.sb;
    if (u.lo) u.lo += e * u.sb;
    return u;
  };
  UPackOut toF{c.wFp, 1, 1, 0}, toK{c.Kp, 0, 1, 0};
  if (P.ncq > 0) {
    const long long kq = (long long)npe * nd;   // the contraction, and B's columns per component
    const int kg = exa_tc::qk_group(npe);       // packed K: a group of kg per gradient component
    if (!c.Sp.hi) {
      // B per trace component b: row r, packed k = l + kg*d from column l + npe*d + npe*nd*b.
      // With the tensor-core volume kernel B is already packed (volume and face kernels write
      // it so), and G always is (the face kernel writes it in this layout in the mixed form)
      ExaProfScope pp(c, EXA_PH_PACK);
      EXA_TRY(exa_pack(c.wB, 1, 1, n, (long long)n * nqn, (long long)n * kq, nb, ncu, c.wBp, c.st, kg, npe));
    }
    ExaProfScope ps(c, EXA_PH_QELIM);
    exa_prof_flops(c, EXA_PH_QELIM, 2.0 * nb * ncu * (double)npe * nd * (double)(n + m) * (npe + ndf));
    UGemmP u{};
    u.batch = nb; u.batch2 = ncu; u.K = kg * nd; u.beta = 1.0;
    u.tci = EXA_T_F64; u.tco = EXA_T_F32;
    // D(:, j + npe*b) = D + B_b MinvC
    u.M = n; u.N = npe; u.alpha = 1.0;
    u.A = c.wBp; u.B = at(c.MCp, e0); u.B.sb2 = 0;
    u.Cin = c.wD; u.ldci = n; u.sCi = (long long)n * n; u.sCi2 = (long long)n * npe;
    u.C = D32; u.ldc = n; u.sC = (long long)n * n; u.sC2 = (long long)n * npe;
    u.nout = 0;
    EXA_TRY(exa_gemm_3xtf32(u, c.d_uflag, c.st));
    if (overlap) EXA_TRY(inverse_beside(c, join, [&](cudaStream_t s) {
      EXA_TRY(inverse(s));
      return pack_dinv(s);
    }));
    // F(:, b + ncu*jf) = F - B_b MinvE, packed only (B operand of D^-1 F)
    u.N = ndf; u.alpha = -1.0;
    u.B = at(c.MEp, e0); u.B.sb2 = 0;
    u.Cin = c.wF; u.ldci = (long long)n * ncu; u.sCi = (long long)n * m; u.sCi2 = n;
    u.C = nullptr;
    toF.cmul = ncu; toF.cadd = 1;
    u.out[0] = toF; u.nout = 1;
    EXA_TRY(exa_gemm_3xtf32(u, c.d_uflag, c.st));
    // K(:, j + npe*b) = K + G_b MinvC, plain and packed (A operand of K D^-1 F)
    u.M = m; u.N = npe; u.alpha = 1.0;
    u.A = c.wGp; u.B = at(c.MCp, e0); u.B.sb2 = 0;
    u.Cin = c.wK; u.ldci = m; u.sCi = (long long)m * n; u.sCi2 = (long long)m * npe;
    u.C = K32; u.ldc = m; u.sC = (long long)m * n; u.sC2 = (long long)m * npe;
    toK.cmul = 1; toK.cadd = npe;
    u.out[0] = toK; u.nout = 1;
    EXA_TRY(exa_gemm_3xtf32(u, c.d_uflag, c.st));
    // H(:, b + ncu*jf) = H - G_b MinvE
    u.N = ndf; u.alpha = -1.0;
    u.B = at(c.MEp, e0); u.B.sb2 = 0;
    u.Cin = Hc; u.ldci = (long long)m * ncu; u.sCi = (long long)m * m; u.sCi2 = m;
    u.C = H32; u.ldc = (long long)m * ncu; u.sC = (long long)m * m; u.sC2 = m;
    u.nout = 0;
    EXA_TRY(exa_gemm_3xtf32(u, c.d_uflag, c.st));
  } else {
    EXA_TRY(exa_k_to_f32(c.wD, D32, (long long)nb * n * n, c.st));
    EXA_TRY(exa_k_to_f32(c.wK, K32, (long long)nb * m * n, c.st));
    EXA_TRY(exa_k_to_f32(Hc, H32, (long long)nb * m * m, c.st));
    // F as the B operand of D^-1 F (row = column of F, k = row), K as an A operand
    EXA_TRY(exa_pack(c.wF, 1, n, 1, (long long)n * m, 0, nb, 1, c.wFp, c.st));
    EXA_TRY(exa_pack(c.wK, 1, 1, m, (long long)m * n, 0, nb, 1, c.Kp, c.st));
  }
  if (overlap) {
    EXA_TRY(join.join());
  } else {
    {
      ExaProfScope ps(c, EXA_PH_INVERSE);
      EXA_TRY(inverse(c.st));
    }
    ExaProfScope pp(c, EXA_PH_PACK);
    EXA_TRY(pack_dinv(c.st));
  }
  ExaProfScope ps(c, EXA_PH_SCHUR);
  exa_prof_flops(c, EXA_PH_SCHUR, 2.0 * nb * ((double)n * n * m + (double)n * n + (double)m * m * n + (double)m * n));
  UGemmP u{};
  u.batch = nb; u.batch2 = 1;
  u.tci = EXA_T_F32; u.tco = EXA_T_F32;
  // DinvF = -Dinv F: plain (Newton update) and packed (B operand of K DinvF)
  u.M = n; u.N = m; u.K = n; u.alpha = -1.0; u.beta = 0.0;
  u.A = c.Dinvp; u.B = c.wFp;
  u.Cin = nullptr;
  u.C = F32; u.ldc = n; u.sC = (long long)n * m;
  u.out[0] = UPackOut{c.DinvFp, 1, 1, 0}; u.nout = 1;
  EXA_TRY(exa_gemm_3xtf32(u, c.d_uflag, c.st));
  // H += K DinvF
  u.M = m; u.N = m; u.K = n; u.alpha = 1.0; u.beta = 1.0;
  u.A = c.Kp; u.B = c.DinvFp;
  u.Cin = H32; u.ldci = m; u.sCi = (long long)m * m;
  u.C = H32; u.ldc = m; u.sC = (long long)m * m;
  u.nout = 0;
  EXA_TRY(exa_gemm_3xtf32(u, c.d_uflag, c.st));
  // Ru = Dinv Ru; Rh -= K Ru
  double* Ruc = c.Ru + (long long)e0 * n;
  EXA_CUDA(cudaMemcpyAsync(c.wRu, Ruc, sizeof(double) * (size_t)n * nb, cudaMemcpyDeviceToDevice, c.st));
  EXA_TRY(exa_k_gemv32(n, n, nb, 1.0, D32, (long long)n * n, c.wRu, n, 0.0, Ruc, n, c.st, c.d_uflag));
  EXA_TRY(exa_k_gemv32(m, n, nb, -1.0, K32, (long long)m * n, Ruc, n, 1.0, c.Rh + (long long)e0 * m, m, c.st,
                       c.d_uflag));
  return EXA_OK;
}

}  // namespace

namespace {

// udg (and the stage source) at the Gauss points of elements e0 .. e0 + nb - 1 by GEMMs with the
// shared basis shapegt: the volume kernel then reads them instead of forming them per element
int volume_gauss_values(ExaCtx& c, AsmArgs& A, int e0, int nb) {
  const ExaDims& P = c.P;
  GemmBatch g{};
  g.M = P.nge; g.K = P.npe; g.alpha = 1.0; g.beta = 0.0;
  g.A = c.shapegt; g.lda = P.nge;
  g.B = c.udg + (long long)e0 * P.npe * P.nc; g.ldb = P.npe; g.N = P.nc * nb;
  g.C = c.wUG; g.ldc = P.nge;
  g.batch = 1; g.batch2 = 1;
  EXA_TRY(exa_gemm(g, c.st));
  A.ugpre = c.wUG;
  if (c.tdep) {
    g.B = c.sdg + (long long)e0 * P.npe * P.ncu; g.N = P.ncu * nb;
    g.C = c.wSG;
    EXA_TRY(exa_gemm(g, c.st));
    A.sgpre = c.wSG;
  }
  A.rgout = c.wRG;
  return EXA_OK;
}

// The FP64 volume blocks D and B of the chunk on the DMMA tensor cores: for each field c, the
// products T_(k,c) shapegt[:, :, 0] of all (element, k) pairs in one batched GEMM, written into
// the columns of D (c < ncu) or B, elements in parts of c.wT_elems (vol_mat_kernel's sums).
int volume_blocks_gemm(ExaCtx& c, int nb) {
  const ExaDims& P = c.P;
  const int npe = P.npe, nge = P.nge, ncu = P.ncu, nd = P.nd, n = P.n, nblk = P.ncu * P.nc;
  const long long nqn = (long long)npe * nd * ncu, blk = (long long)npe * nge;
  for (int le0 = 0; le0 < nb; le0 += c.wT_elems) {
    const int nbs = std::min(c.wT_elems, nb - le0);
    const long long tot = blk * nblk * nbs;
    vol_t_kernel<<<(unsigned)std::min<long long>((tot + 255) / 256, 8192), 256, 0, c.st>>>(P, c.shapegw, c.wRg, le0,
                                                                                         nbs, c.wT);
    EXA_LAUNCH_CHECK();
    for (int cc = 0; cc < P.nc; ++cc) {
      GemmBatch g{};
      g.M = npe; g.N = npe; g.K = nge; g.alpha = 1.0; g.beta = 0.0;
      g.A = c.wT + (long long)ncu * cc * blk; g.lda = npe; g.sA = nblk * blk; g.sA2 = blk;
      g.B = c.shapegt; g.ldb = nge;
      if (cc < ncu) {
        g.C = c.wD + (long long)le0 * n * n + (long long)n * npe * cc;
        g.ldc = n; g.sC = (long long)n * n;
      } else {
        const int qc = cc - ncu, nq = qc % ncu, d = qc / ncu;
        g.C = c.wB + (long long)le0 * n * nqn + (long long)n * ((long long)npe * d + (long long)npe * nd * nq);
        g.ldc = n; g.sC = (long long)n * nqn;
      }
      g.sC2 = npe;  // trace component k: rows npe k
      g.batch = nbs; g.batch2 = ncu;
      EXA_TRY(exa_gemm(g, c.st));
    }
  }
  return EXA_OK;
}

// Ru of the chunk = shapegw (npe x nge (nd + 1)) times the volume kernel's integrands
int volume_residual_gemm(ExaCtx& c, double* Ruc, int nb) {
  const ExaDims& P = c.P;
  GemmBatch g{};
  g.M = P.npe; g.K = P.nge * (P.nd + 1); g.N = P.ncu * nb; g.alpha = 1.0; g.beta = 0.0;
  g.A = c.shapegw; g.lda = P.npe;
  g.B = c.wRG; g.ldb = (long long)P.nge * (P.nd + 1);
  g.C = Ruc; g.ldc = P.npe;
  g.batch = 1; g.batch2 = 1;
  return exa_gemm(g, c.st);
}

}  // namespace

int exa_model_assemble(ExaCtx& c, bool jacobian) {
  const ExaDims& P = c.P;
  const int n = P.n, m = P.m;
  const long long nqn = (long long)P.npe * P.nd * P.ncu;
  const size_t vs = jacobian ? vol_points_smem<true>(P) : vol_points_smem<false>(P);
  const size_t fs = face_smem(P, jacobian);
  if (jacobian) {
    EXA_TRY(smem_attr((const void*)vol_points_kernel<ExaModel, true>, vs));
    EXA_TRY(smem_attr((const void*)face_kernel<ExaModel, true>, fs));
  } else {
    EXA_TRY(smem_attr((const void*)vol_points_kernel<ExaModel, false>, vs));
    EXA_TRY(smem_attr((const void*)face_kernel<ExaModel, false>, fs));
  }
  const int tpb_v = P.nge <= 64 ? 64 : (P.nge <= 128 ? 128 : 256);
  const int tpb_f = 128;
  for (int e0 = 0; e0 < P.ne; e0 += c.neb) {
    const int nb = std::min(c.neb, P.ne - e0);
    AsmArgs A = make_args(c, e0);
    double* Ruc = c.Ru + (long long)e0 * n;
    double* Rhc = c.Rh + (long long)e0 * m;
    if (jacobian) {
      {
        ExaProfScope ps(c, EXA_PH_VOLUME);
        if (c.wRG) EXA_TRY(volume_gauss_values(c, A, e0, nb));
        vol_points_kernel<ExaModel, true><<<nb, tpb_v, vs, c.st>>>(A, Ruc, c.wRg);
        EXA_LAUNCH_CHECK();
        if (c.wRG) EXA_TRY(volume_residual_gemm(c, Ruc, nb));
        if (c.precision == 1 && c.Sp.hi) {
          // B straight into its packed FP32 form (the face kernel adds its terms there too).
          // The volume kernel assigns every entry of B, so only the layout's padding needs
          // zeros, and nothing writes there after the zeroing at allocation.
          UPacked bp{};
          if (nqn > 0 && P.ncq > 0) {
            bp = c.wBp;
            A.Bp = c.wBp;
          }
          EXA_TRY(exa_k_vol_mat_tc(P, c.shapegw32, c.Sp, c.wRg, c.wD, c.wB, bp, nb, c.d_uflag, c.st));
        } else if (c.wT) {
          EXA_TRY(volume_blocks_gemm(c, nb));
        } else {
          const int tiles = exa_ceil_div(P.npe, 64);
          dim3 grid(tiles * tiles, nb, P.ncu * P.nc);
          vol_mat_kernel<<<grid, 256, 0, c.st>>>(P, c.shapegw, c.shapegt, c.wRg, c.wD, c.wB);
          EXA_LAUNCH_CHECK();
        }
      }
      double* Hc = c.fp64_full ? c.H + (long long)e0 * m * m : c.H;
      {
        ExaProfScope ps(c, EXA_PH_FACE);
        // F, K and H of the chunk: the face kernel assigns their face blocks, at the same
        // positions at every assembly (face l's rows or columns, the same master-face node
        // lists for every element); the rest is structurally zero.  The plain form's products
        // overwrite these arrays, so it zeroes them each time; in the mixed form the products
        // only read them, and the zeros of the switch to that form (exa_ctx_set_precision) stay.
        const bool zero_blocks = c.precision != 1;
        if (zero_blocks) {
          EXA_CUDA(cudaMemsetAsync(c.wF, 0, sizeof(double) * (size_t)nb * n * m, c.st));
          EXA_CUDA(cudaMemsetAsync(c.wK, 0, sizeof(double) * (size_t)nb * m * n, c.st));
        }
        if (nqn > 0 && P.ncq > 0) {
          if (c.precision == 1 && c.wGp.hi) {
            // G written packed by the face kernel.  Each element slot gets the same entries
            // assigned at every assembly (face l's trace rows against face l's nodes, the same
            // master-face node lists for every element); the rest of G is structurally zero and
            // keeps the zeros of the allocation, since nothing else writes there.
            A.Gp = c.wGp;
          } else {
            EXA_CUDA(cudaMemsetAsync(c.wG, 0, sizeof(double) * (size_t)nb * m * nqn, c.st));
          }
        }
        if (zero_blocks) EXA_CUDA(cudaMemsetAsync(Hc, 0, sizeof(double) * (size_t)nb * m * m, c.st));
        face_kernel<ExaModel, true><<<nb, tpb_f, fs, c.st>>>(A, Ruc, Rhc, c.wD, c.wB, c.wF, c.wK, c.wG, Hc);
        EXA_LAUNCH_CHECK();
      }
      EXA_TRY(c.precision == 1 ? schur_chunk_mixed(c, e0, nb) : schur_chunk(c, e0, nb));
    } else {
      ExaProfScope ps(c, EXA_PH_RESIDUAL);
      if (c.wRG) EXA_TRY(volume_gauss_values(c, A, e0, nb));
      if (!launch_vol_pointwise<ExaModel>(A, nb, c.st))
        vol_points_kernel<ExaModel, false><<<nb, tpb_v, vs, c.st>>>(A, Ruc, nullptr);
      EXA_LAUNCH_CHECK();
      if (c.wRG) EXA_TRY(volume_residual_gemm(c, Ruc, nb));
      face_kernel<ExaModel, false><<<nb, tpb_f, fs, c.st>>>(A, Ruc, Rhc, nullptr, nullptr, nullptr, nullptr, nullptr,
                                                           nullptr);
      EXA_LAUNCH_CHECK();
    }
  }
  return EXA_OK;
}

bool exa_model_has_ldg_boundary() { return ExaModel::has_ldg_boundary; }

// The LDG residual of the element states u (the layout of udg: nc = ncu without q): the volume
// integrals of the HDG residual (RuElem, uresidual.cpp:45-130, is the same quadrature), the
// face residuals of every face, and their sum into the elements with the sign and scaling of
// Residual (residual.cpp:589-617).
int exa_model_ldg_residual(ExaCtx& c, const double* u, double* Ru) {
  const ExaDims& P = c.P;
  ExaProfScope ps(c, EXA_PH_RESIDUAL);
  double* saved = c.udg;
  c.udg = const_cast<double*>(u);
  auto body = [&]() -> int {
    const size_t vs = vol_points_smem<false>(P);
    EXA_TRY(smem_attr((const void*)vol_points_kernel<ExaModel, false>, vs));
    const int tpb_v = P.nge <= 64 ? 64 : (P.nge <= 128 ? 128 : 256);
    for (int e0 = 0; e0 < P.ne; e0 += c.neb) {
      const int nb = std::min(c.neb, P.ne - e0);
      AsmArgs A = make_args(c, e0);
      double* Ruc = c.Ru + (long long)e0 * P.n;
      if (c.wRG) EXA_TRY(volume_gauss_values(c, A, e0, nb));
      if (!launch_vol_pointwise<ExaModel>(A, nb, c.st))
        vol_points_kernel<ExaModel, false><<<nb, tpb_v, vs, c.st>>>(A, Ruc, nullptr);
      EXA_LAUNCH_CHECK();
      if (c.wRG) EXA_TRY(volume_residual_gemm(c, Ruc, nb));
    }
    LdgArgs L{};
    L.P = P;
    L.shapfgt = c.shapfgt; L.shapfgw = c.shapfgw; L.shapfnt = c.shapfnt;
    L.f2e = c.f2e; L.perm = c.perm; L.bf = c.bf; L.fcon = c.ldg_fcon;
    L.xdg = c.xdg; L.faceg = c.faceg; L.uinf = c.uinf; L.param = c.param; L.tau = c.tau;
    L.ntau = c.ntau; L.modelnumber = c.modelnumber; L.time = c.time;
    L.u = u; L.Rh = c.ldg_Rh;
    const size_t fs = ldg_face_smem(P);
    EXA_TRY(smem_attr((const void*)ldg_face_kernel<ExaModel>, fs));
    // interior faces by the pointwise kernel where the model's (nd, ncu) has one, the boundary
    // faces (and otherwise all) by the general one
    int fgen = 0;
    if (c.ldg_split && launch_ldg_face_inner<ExaModel>(L, P.nf0, c.st)) {
      EXA_LAUNCH_CHECK();
      fgen = P.nf0;
    }
    if (P.nf > fgen) {
      L.f0 = fgen;
      ldg_face_kernel<ExaModel><<<P.nf - fgen, 64, fs, c.st>>>(L);
      EXA_LAUNCH_CHECK();
    }
    return exa_k_ldg_gather(P, c.f2e, c.perm, c.elemcon, c.Ru, c.ldg_Rh, Ru, c.tdep, c.dtfactor, c.st);
  };
  const int st = body();
  c.udg = saved;
  return st;
}

// initial u from the model's cpuInitu at the element nodes (readsolstruct, readbinaryfiles.cpp:546-556)
int exa_model_init_udg(ExaCtx& c, double* host_udg) {
  const ExaDims& P = c.P;
  const int np = P.npe * P.ne;
  std::vector<double> f((size_t)np * P.nc, 0.0);
  EXA_MODEL_NS::cpuInitu(f.data(), c.h_xdg.data(), c.h_uinf.data(), c.h_param.data(), c.modelnumber, np, P.ncx,
                         P.nc, P.npe, P.ne);
  for (int e = 0; e < P.ne; ++e)
    for (int k = 0; k < P.ncu; ++k)
      for (int i = 0; i < P.npe; ++i)
        host_udg[i + P.npe * k + P.npe * P.nc * e] = f[i + P.npe * k + (size_t)P.npe * P.nc * e];
  return EXA_OK;
}

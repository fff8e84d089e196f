// Context setup from Exasim's input blobs and the C ABI of the solver
// (declarations and reference citations: include/exasim_b200.h).
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "exa_solver.cuh"
#include "exa_bilu0.h"
#include "exa_tc.cuh"
#include "exa_umma.cuh"
#include "../../include/exasim_b200.h"

namespace {

// Exasim *.bin layout: [lsize, nsize(lsize), part_0(nsize[0]), part_1(nsize[1]), ...]
struct Blob {
  std::vector<long long> nsize;
  std::vector<const double*> part;
  bool ok = false;
};

Blob split_blob(const double* a, long long n) {
  Blob b;
  if (!a || n < 1) return b;
  const long long ls = (long long)a[0];
  if (ls < 1 || 1 + ls > n) return b;
  long long o = 1 + ls;
  for (long long i = 0; i < ls; ++i) {
    const long long s = (long long)a[1 + i];
    if (s < 0 || o + s > n) return b;
    b.nsize.push_back(s);
    b.part.push_back(a + o);
    o += s;
  }
  b.ok = true;
  return b;
}

template <class T>
int dev_upload(ExaCtx& c, T** dst, const T* src, size_t count) {
  if (count == 0) {
    *dst = nullptr;
    return EXA_OK;
  }
  // stream-ordered allocation on the context stream: unlike cudaMalloc / cudaFree it does not
  // synchronize the device, so contexts can come and go while others are solving
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, count * sizeof(T), c.st);
  if (e != cudaSuccess) {
    exa_set_error("device allocation of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
    return EXA_ERR_NOMEM;
  }
  c.allocs.push_back(p);
  c.alloc_bytes += (long long)(count * sizeof(T));
  *dst = (T*)p;
  // from pageable memory the call returns once the source has been staged
  if (src) EXA_CUDA(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, c.st));
  return EXA_OK;
}

// Zeroed on the context stream: that stream is non-blocking, so a legacy-stream memset
// would not be ordered before the kernels that later fill the array on it.
template <class T>
int dev_alloc(ExaCtx& c, T** dst, size_t count) {
  EXA_TRY(dev_upload<T>(c, dst, nullptr, count));
  if (count) EXA_CUDA(cudaMemsetAsync(*dst, 0, count * sizeof(T), c.st));
  return EXA_OK;
}

std::vector<int> to_int(const double* p, long long n) {
  std::vector<int> v((size_t)n);
  for (long long i = 0; i < n; ++i) v[(size_t)i] = (int)llround(p[i]);
  return v;
}

// udg from sol.bin (full or u only) or the model's initial condition; uhat from sol.bin or
// from u at the face nodes (readsolstruct, readbinaryfiles.cpp:499-618)
int init_solution(ExaCtx& c, const Blob& S) {
  const ExaDims& P = c.P;
  {
    std::vector<double> u((size_t)P.ne * P.npe * P.nc, 0.0);
    const long long nu = S.nsize.size() > 2 ? S.nsize[2] : 0;
    if (nu == (long long)(size_t)P.ne * P.npe * P.nc) {
      std::memcpy(u.data(), S.part[2], sizeof(double) * u.size());
    } else if (nu == (long long)(size_t)P.ne * P.npe * P.ncu) {
      for (size_t e = 0; e < (size_t)P.ne; ++e)
        for (int k = 0; k < P.ncu; ++k)
          for (int i = 0; i < P.npe; ++i) u[i + P.npe * k + P.npe * P.nc * e] = S.part[2][i + P.npe * k + P.npe * P.ncu * e];
    } else if (nu == 0) {
      EXA_TRY(exa_model_init_udg(c, u.data()));
    } else {
      exa_set_error("sol.bin udg size %lld matches neither npe*nc*ne nor npe*ncu*ne", nu);
      return EXA_ERR_ARG;
    }
    // on the context stream, after the zeroing queued there (pageable sources are staged
    // before the calls return)
    EXA_CUDA(cudaMemcpyAsync(c.udg, u.data(), sizeof(double) * u.size(), cudaMemcpyHostToDevice, c.st));
    const long long nuh = S.nsize.size() > 5 ? S.nsize[5] : 0;
    if (nuh == c.ndofuhat()) {
      EXA_CUDA(cudaMemcpyAsync(c.uh, S.part[5], sizeof(double) * nuh, cudaMemcpyHostToDevice, c.st));
    } else {
      EXA_TRY(exa_k_face_nodes(P, c.f2e, c.perm, c.udg, c.uh, c.st));
    }
  }

  return EXA_OK;
}

}  // namespace

int exa_ctx_init(ExaCtx& c, const double* app, long long napp, const double* master, long long nmaster,
                 const double* mesh, long long nmesh, const double* sol, long long nsol, int device) {
  Blob A = split_blob(app, napp), M = split_blob(master, nmaster), Me = split_blob(mesh, nmesh),
       S = split_blob(sol, nsol);
  if (!A.ok || !M.ok || !Me.ok || !S.ok) {
    exa_set_error("malformed input blob (app %d, master %d, mesh %d, sol %d)", A.ok, M.ok, Me.ok, S.ok);
    return EXA_ERR_ARG;
  }
  if (A.nsize.size() < 9 || M.nsize.size() < 15 || Me.nsize.size() < 28 || S.nsize.size() < 3) {
    exa_set_error("input blobs are shorter than Exasim's formats");
    return EXA_ERR_ARG;
  }
  // ---- app.bin (readappstruct, readbinaryfiles.cpp:65-152; setcommonstruct, setstructs.cpp:45-200)
  const double* nd_app = A.part[0];
  const double* flag = A.part[1];
  const double* prob = A.part[2];
  ExaDims& P = c.P;
  const int mpiprocs = (int)nd_app[0];
  P.nc = (int)nd_app[5];
  P.ncu = (int)nd_app[6];
  P.ncq = (int)nd_app[7];
  P.nco = (int)nd_app[9];
  P.ncx = (int)nd_app[11];
  P.ncw = (int)nd_app[13];
  c.tdep = (int)flag[0];
  c.wave = (int)flag[1];
  c.ortho = (int)flag[5];
  c.preconditioner = (int)flag[6];
  c.tdfunc = (int)flag[10];
  c.sourcefunc = (int)flag[11];
  c.modelnumber = (int)flag[12];
  const int spatial = (int)prob[0];
  c.torder = (int)prob[3];
  c.nstage = (int)prob[4];
  c.newton_maxit = (int)prob[13];
  c.gmres_maxit = (int)prob[14];
  c.restart = (int)prob[15];
  c.RBdim = (int)prob[16];
  c.ppdegree = A.nsize[2] > 27 ? (int)prob[27] : 0;
  const int coupled = A.nsize[2] > 28 ? (int)prob[28] : 0;
  c.h_uinf.assign(A.part[3], A.part[3] + A.nsize[3]);
  c.dt.assign(A.part[4], A.part[4] + A.nsize[4]);
  const double* factor = A.part[5];
  c.h_param.assign(A.part[6], A.part[6] + A.nsize[6]);
  const double* solvers = A.part[7];
  if (A.nsize[7] < 2 || A.nsize[8] < 1) {
    exa_set_error("app.bin lacks solver parameters or tau");
    return EXA_ERR_ARG;
  }
  c.newton_tol = solvers[0];
  c.gmres_tol = solvers[1];
  c.time0 = (c.tdep == 1 && A.nsize[5] > 0) ? factor[0] : 0.0;
  c.time = c.time0;
  if (spatial != 0 && spatial != 1) {
    exa_set_error("discretization problem[0]=%d: LDG (0) or HDG (1)", spatial);
    return EXA_ERR_UNSUPPORTED;
  }
  c.scheme = spatial;
  c.ntau = (int)A.nsize[8];
  if (c.scheme == 0) {
    // LDG with the pseudo-transient solver: models without q, the finite-difference Jacobian
    // (flag[4], solversparam[2]), the identity or mass-inverse preconditioner (flag[7]), the
    // reduced-basis initial guess (problem[16]) and the polynomial preconditioner (problem[27])
    c.matvec_order = (int)flag[4];
    c.matvec_eps = A.nsize[7] > 2 ? solvers[2] : 1e-3;
    c.ldg_prec_matrix = (int)flag[7];
    if (P.ncq != 0) {
      exa_set_error("LDG with q (ncq=%d) is not supported: the reference's GetQ calls RuFace for the q face term",
                    P.ncq);
      return EXA_ERR_UNSUPPORTED;
    }
    if (c.matvec_order != 1 && c.matvec_order != 2) {
      exa_set_error("LDG matrix-vector product of order %d: 1 or 2", c.matvec_order);
      return EXA_ERR_UNSUPPORTED;
    }
    if (!(c.matvec_eps > 0.0)) { exa_set_error("LDG finite-difference step %g is not positive", c.matvec_eps); return EXA_ERR_ARG; }
  }
  if (mpiprocs > 1) { exa_set_error("multi-rank inputs: this solver runs one GPU per mesh"); return EXA_ERR_UNSUPPORTED; }
  if (P.nco > 0 || P.ncw > 0) { exa_set_error("odg/wdg fields (nco=%d, ncw=%d) are outside the HDG hot path", P.nco, P.ncw); return EXA_ERR_UNSUPPORTED; }
  if (c.wave) { exa_set_error("wave (ModelW) problems are not supported"); return EXA_ERR_UNSUPPORTED; }
  if (coupled > 0) { exa_set_error("coupled interfaces are not supported"); return EXA_ERR_UNSUPPORTED; }
  if (c.RBdim < 0 || c.RBdim > 64) { exa_set_error("reduced-basis dimension %d outside 0..64", c.RBdim); return EXA_ERR_UNSUPPORTED; }
  if (c.ppdegree > 1 && c.ppdegree > c.restart) {
    exa_set_error("polynomial preconditioner of degree %d needs a GMRES restart of at least that (restart %d)",
                  c.ppdegree, c.restart);
    return EXA_ERR_UNSUPPORTED;
  }
  if (c.preconditioner < 0 || c.preconditioner > 2) { exa_set_error("preconditioner %d: block Jacobi (0), elemental additive Schwarz (1) or block ILU(0) on Cartesian sub-domains (2)", c.preconditioner); return EXA_ERR_UNSUPPORTED; }
  if (c.restart < 1 || c.gmres_maxit < 1) { exa_set_error("GMRES restart/iterations must be positive"); return EXA_ERR_ARG; }

  // ---- master.bin (readmasterstruct, readbinaryfiles.cpp:208-268)
  const double* mnd = M.part[0];
  P.nd = (int)mnd[0];
  c.elemtype = (int)mnd[1];
  c.porder = (int)mnd[3];
  P.npe = (int)mnd[5];
  P.npf = (int)mnd[6];
  P.nge = (int)mnd[7];
  P.ngf = (int)mnd[8];
  if (P.ncx != P.nd) { exa_set_error("ncx (%d) differs from the dimension (%d)", P.ncx, P.nd); return EXA_ERR_UNSUPPORTED; }
  if (P.nc != P.ncu && P.nc != P.ncu * (P.nd + 1)) { exa_set_error("nc=%d is neither ncu nor ncu*(nd+1)", P.nc); return EXA_ERR_UNSUPPORTED; }
  if ((long long)M.nsize[1] != (long long)P.nge * P.npe * (P.nd + 1) || (long long)M.nsize[3] != (long long)P.ngf * P.npf * P.nd) {
    exa_set_error("master.bin shape tables do not match its sizes");
    return EXA_ERR_ARG;
  }

  // ---- mesh.bin (readmeshstruct, readbinaryfiles.cpp:321-409)
  const double* mdims = Me.part[0];
  P.ne = (int)mdims[1];
  P.nfe = (int)mdims[4];
  P.ndf = P.npf * P.nfe;
  P.n = P.npe * P.ncu;
  P.m = P.ncu * P.ndf;
  if (Me.nsize[23] != (long long)P.npf * P.nfe || Me.nsize[24] != (long long)P.nfe * P.ne) {
    exa_set_error("mesh.bin perm/bf sizes do not match the master element");
    return EXA_ERR_ARG;
  }
  std::vector<int> perm = to_int(Me.part[23], Me.nsize[23]);
  std::vector<int> bfv = to_int(Me.part[24], Me.nsize[24]);
  ExaConn conn;
  if (Me.nsize[1] == 0) {
    if (Me.nsize[26] != (long long)P.ne * ((c.elemtype == 0) ? P.nd + 1 : (1 << P.nd))) {
      exa_set_error("mesh.bin has neither connectivity nor element vertex lists");
      return EXA_ERR_ARG;
    }
    std::vector<int> t = to_int(Me.part[26], Me.nsize[26]);
    const int nf = exa_build_connectivity(t.data(), bfv.data(), perm.data(), M.part[12], P.nd, c.elemtype, P.ne,
                                          P.npe, P.npf, conn);
    if (nf < 0) { exa_set_error("mesh connectivity is wrong (unmatched face)"); return EXA_ERR_MESH; }
  } else {
    // pre-connected mesh: f2e [4,nf], elemcon [npf*nfe, ne]; interior faces are the fblks with code 0
    conn.nf = (int)mdims[2];
    conn.nfe = P.nfe;
    conn.f2e = to_int(Me.part[21], Me.nsize[21]);
    conn.elemcon = to_int(Me.part[22], Me.nsize[22]);
    conn.nf0 = 0;
    for (long long j = 0; j + 2 < Me.nsize[3]; j += 3)
      if ((int)Me.part[3][j + 2] == 0) conn.nf0 += (int)Me.part[3][j + 1] - (int)Me.part[3][j] + 1;
    if ((long long)conn.f2e.size() != 4LL * conn.nf || (long long)conn.elemcon.size() != (long long)P.ndf * P.ne) {
      exa_set_error("mesh.bin f2e/elemcon sizes are inconsistent");
      return EXA_ERR_ARG;
    }
  }
  P.nf = conn.nf;
  P.nf0 = conn.nf0;
  if (P.n > exa_inverse_max_n()) {
    exa_set_error("element blocks of order %d exceed the dense inverse's limit %d", P.n, exa_inverse_max_n());
    return EXA_ERR_UNSUPPORTED;
  }
  if ((c.preconditioner == 0 && P.ncu * P.npf > 160) || (c.preconditioner == 1 && P.m > 160)) {
    exa_set_error("preconditioner %d: its blocks (order %d) exceed 160", c.preconditioner,
                  c.preconditioner == 0 ? P.ncu * P.npf : P.m);
    return EXA_ERR_UNSUPPORTED;
  }

  // ---- sol.bin (readsolstruct, readbinaryfiles.cpp:499-618)
  if (S.nsize[1] != (long long)P.npe * P.ncx * P.ne) { exa_set_error("sol.bin xdg size mismatch"); return EXA_ERR_ARG; }
  c.h_xdg.assign(S.part[1], S.part[1] + S.nsize[1]);

  // ---- device
  c.device = device;
  EXA_CUDA(cudaSetDevice(device));
  EXA_CUDA(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
  EXA_CUDA(cudaStreamCreateWithFlags(&c.st2, cudaStreamNonBlocking));
  EXA_CUDA(cudaEventCreateWithFlags(&c.ev_q, cudaEventDisableTiming));
  EXA_CUDA(cudaEventCreateWithFlags(&c.ev_inv, cudaEventDisableTiming));
  EXA_TRY(dev_upload(c, &c.shapegt, M.part[1], (size_t)M.nsize[1]));
  EXA_TRY(dev_upload(c, &c.shapegw, M.part[2], (size_t)M.nsize[2]));
  EXA_TRY(dev_upload(c, &c.shapfgt, M.part[3], (size_t)M.nsize[3]));
  EXA_TRY(dev_upload(c, &c.shapfgw, M.part[4], (size_t)M.nsize[4]));
  EXA_TRY(dev_upload(c, &c.perm, perm.data(), perm.size()));
  EXA_TRY(dev_upload(c, &c.bf, bfv.data(), bfv.size()));
  EXA_TRY(dev_upload(c, &c.f2e, conn.f2e.data(), conn.f2e.size()));
  EXA_TRY(dev_upload(c, &c.elemcon, conn.elemcon.data(), conn.elemcon.size()));
  if (c.preconditioner == 2) {
    // block ILU(0) on the Cartesian sub-domains of mesh.bin's cartgridpart (discretization.cpp:296-311)
    c.cartgridpart = to_int(Me.part[25], Me.nsize[25]);
    if (c.cartgridpart.empty()) {
      exa_set_error("block ILU(0) (preconditioner 2) needs cartgridpart in mesh.bin");
      return EXA_ERR_UNSUPPORTED;
    }
    ExaBilu hb;
    char msg[256] = "";
    if (exa_bilu_setup(c.cartgridpart.data(), (int)c.cartgridpart.size(), conn.f2e.data(), conn.nf, P.nfe, P.ne, hb,
                       msg, sizeof(msg)) != 0) {
      exa_set_error("block ILU(0): %s", msg);
      return EXA_ERR_UNSUPPORTED;
    }
    const int ncf = P.ncu * P.npf;
    if (ncf > 64 || exa_bilu_apply_smem(ncf, hb.nfse) > 227 * 1024) {
      exa_set_error("block ILU(0): %d faces of %d rows per sub-domain exceed shared memory", hb.nfse, ncf);
      return EXA_ERR_UNSUPPORTED;
    }
    ExaBiluDev& d = c.bilu;
    d.nse = hb.nse; d.nfse = hb.nfse; d.nnz = hb.nnz;
    EXA_TRY(dev_upload(c, &d.row_ptr, hb.row_ptr.data(), hb.row_ptr.size()));
    EXA_TRY(dev_upload(c, &d.col_ind, hb.col_ind.data(), hb.col_ind.size()));
    EXA_TRY(dev_upload(c, &d.face, hb.face.data(), hb.face.size()));
    EXA_TRY(dev_upload(c, &d.row_of, hb.row_of.data(), hb.row_of.size()));
    EXA_TRY(dev_upload(c, &d.fac_ptr, hb.fac_ptr.data(), hb.fac_ptr.size()));
    EXA_TRY(dev_upload(c, &d.fac_ji, hb.fac_ji.data(), std::max<size_t>(1, hb.fac_ji.size())));
    EXA_TRY(dev_upload(c, &d.upd_ptr, hb.upd_ptr.data(), hb.upd_ptr.size()));
    EXA_TRY(dev_upload(c, &d.upd_jl, hb.upd_jl.data(), std::max<size_t>(1, hb.upd_jl.size())));
    EXA_TRY(dev_upload(c, &d.upd_il, hb.upd_il.data(), std::max<size_t>(1, hb.upd_il.size())));
    EXA_TRY(dev_upload(c, &d.gf_ptr, hb.gf_ptr.data(), hb.gf_ptr.size()));
    EXA_TRY(dev_upload(c, &d.gf_pos, hb.gf_pos.data(), hb.gf_pos.size()));
    EXA_TRY(dev_alloc(c, &d.out, (size_t)hb.nse * hb.nfse * ncf));
  }
  EXA_TRY(dev_upload(c, &c.xdg, S.part[1], (size_t)S.nsize[1]));
  std::vector<double> one_zero(1, 0.0);
  EXA_TRY(dev_upload(c, &c.uinf, c.h_uinf.empty() ? one_zero.data() : c.h_uinf.data(), std::max<size_t>(1, c.h_uinf.size())));
  EXA_TRY(dev_upload(c, &c.param, c.h_param.empty() ? one_zero.data() : c.h_param.data(), std::max<size_t>(1, c.h_param.size())));
  EXA_TRY(dev_upload(c, &c.tau, A.part[8], (size_t)A.nsize[8]));
  const size_t ne = P.ne;
  EXA_TRY(dev_alloc(c, &c.elemg, ne * P.elemg_stride()));
  EXA_TRY(dev_alloc(c, &c.faceg, ne * P.nfe * P.faceg_stride()));
  EXA_TRY(exa_k_geometry(P, c.shapegt, c.shapfgt, c.perm, c.xdg, c.elemg, c.faceg, c.st));
  if (c.scheme == 0) {
    // LDG: both sides' face-node table, the face nodal basis for the boundary's Ubou, and
    // the residual buffers of the finite-difference Jacobian
    const bool boundary = conn.nf0 < conn.nf;
    c.ldg_has_boundary = boundary ? 1 : 0;
    if (boundary && !exa_model_has_ldg_boundary()) {
      exa_set_error("LDG on a mesh with boundary faces needs the model's Ubou and Fbou (KokkosUbou, KokkosFbou)");
      return EXA_ERR_UNSUPPORTED;
    }
    if (M.nsize.size() < 8 || M.nsize[7] != (long long)P.npf * P.npf * P.nd) {
      exa_set_error("master.bin lacks the face nodal basis shapfnt");
      return EXA_ERR_ARG;
    }
    EXA_TRY(dev_upload(c, &c.shapfnt, M.part[7], (size_t)M.nsize[7]));
    {
      bool split = true;
      for (int f = 0; f < conn.nf && split; ++f) split = (conn.f2e[4 * f + 2] >= 0) == (f < conn.nf0);
      c.ldg_split = split ? 1 : 0;
    }
    EXA_TRY(dev_alloc(c, &c.ldg_fcon, 2 * (size_t)P.npf * P.nf));
    EXA_TRY(exa_k_ldg_fcon(P, c.f2e, c.perm, c.elemcon, c.ldg_fcon, c.st));
    const size_t nl = (size_t)P.npe * P.ncu * ne;
    EXA_TRY(dev_alloc(c, &c.ldg_R, nl));
    EXA_TRY(dev_alloc(c, &c.ldg_w, nl));
    EXA_TRY(dev_alloc(c, &c.ldg_Rw, nl));
    EXA_TRY(dev_alloc(c, &c.ldg_Rm, nl));
    EXA_TRY(dev_alloc(c, &c.ldg_Rh, (size_t)P.npf * P.ncu * std::max(1, P.nf)));
  }

  // solution: udg from sol.bin (full or u only) or the model's initial condition; uhat from sol.bin or u
  EXA_TRY(dev_alloc(c, &c.udg, ne * P.npe * P.nc));
  EXA_TRY(dev_alloc(c, &c.uh, (size_t)c.ndofuhat()));
  EXA_TRY(dev_alloc(c, &c.sdg, ne * P.npe * P.ncu));
  EXA_TRY(init_solution(c, S));

  // q-equation matrices Minv*C, Minv*E (qequation.cpp:66-338)
  if (P.ncq > 0) {
    double *mass = nullptr, *cw = nullptr, *ew = nullptr;
    EXA_TRY(dev_alloc(c, &mass, ne * P.npe * P.npe));
    EXA_TRY(dev_alloc(c, &cw, ne * P.npe * P.npe * P.nd));
    EXA_TRY(dev_alloc(c, &ew, ne * P.npe * P.ndf * P.nd));
    EXA_TRY(dev_alloc(c, &c.MC, ne * P.npe * P.npe * P.nd));
    EXA_TRY(dev_alloc(c, &c.ME, ne * P.npe * P.ndf * P.nd));
    EXA_TRY(dev_alloc(c, &c.d_flag, 4));
    EXA_TRY(exa_k_qmats(P, c.shapegt, c.shapegw, c.shapfgt, c.shapfgw, c.perm, c.elemg, c.faceg, mass, cw, ew, c.st));
    EXA_TRY(exa_inverse_tune(P.npe, (int)std::min<size_t>(ne, 4096), 1, c.st));
    EXA_TRY(exa_inverse(mass, P.npe, (long long)P.npe * P.npe, P.ne, c.d_flag, c.st));
    c.Minv = mass;  // kept: q recovery applies it to C u - E uhat
    EXA_TRY(dev_alloc(c, &c.wq_ug, ne * P.nge * P.ncu));
    EXA_TRY(dev_alloc(c, &c.wq_v, ne * P.nge * P.nd * P.nd * P.ncu));
    EXA_TRY(dev_alloc(c, &c.wq_w, ne * P.npe * P.nd * P.ncu));
    // the two products of q recovery over all elements: u at the Gauss points (one batch entry
    // per field) and the gradient moments C_d u (large meshes only, as above)
    if ((long long)ne * P.nge * P.npe >= (1LL << 25)) {
      EXA_TRY(exa_gemm_tune(P.nge, (int)ne, P.npe, P.ncu, c.st));
      EXA_TRY(exa_gemm_tune(P.npe, P.ncu * P.nd * (int)ne, P.nge * P.nd, 1, c.st));
    }
    GemmBatch g{};
    g.M = P.npe; g.N = P.npe; g.K = P.npe; g.alpha = 1.0; g.beta = 0.0;
    g.A = mass; g.lda = P.npe; g.sA = (long long)P.npe * P.npe; g.sA2 = 0;
    g.B = cw; g.ldb = P.npe; g.sB = (long long)P.npe * P.npe * P.nd; g.sB2 = (long long)P.npe * P.npe;
    // stored with rows (l, d) stacked: MinvC(l, d, j) = MC[l + npe*d + npe*nd*j], so the Schur
    // q-elimination contracts over (l, d) in one GEMM per block
    g.C = c.MC; g.ldc = (long long)P.npe * P.nd; g.sC = (long long)P.npe * P.npe * P.nd; g.sC2 = P.npe;
    g.batch = P.ne; g.batch2 = P.nd;
    EXA_TRY(exa_gemm(g, c.st));
    g.N = P.ndf;
    g.B = ew; g.sB = (long long)P.npe * P.ndf * P.nd; g.sB2 = (long long)P.npe * P.ndf;
    g.C = c.ME; g.sC = (long long)P.npe * P.ndf * P.nd; g.sC2 = P.npe;
    EXA_TRY(exa_gemm(g, c.st));
    EXA_CUDA(cudaStreamSynchronize(c.st));
    int flag_h = 0;
    EXA_CUDA(cudaMemcpy(&flag_h, c.d_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag_h) { exa_set_error("singular element mass matrix"); return EXA_ERR_SINGULAR; }
  } else {
    EXA_TRY(dev_alloc(c, &c.d_flag, 4));
  }

  if (c.scheme == 0 && c.ldg_prec_matrix != 0) {
    // the LDG preconditioner: the inverse element mass matrices, applied per field
    // (ApplyMassInv, applymatrix.cpp:66-85)
    EXA_TRY(dev_alloc(c, &c.Minv, ne * P.npe * P.npe));
    EXA_TRY(exa_k_ldg_mass(P, c.shapegt, c.shapegw, c.elemg, c.Minv, c.st));
    EXA_TRY(exa_inverse(c.Minv, P.npe, (long long)P.npe * P.npe, P.ne, c.d_flag, c.st));
    int flag_h = 0;
    EXA_CUDA(cudaStreamSynchronize(c.st));
    EXA_CUDA(cudaMemcpy(&flag_h, c.d_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag_h) { exa_set_error("singular element mass matrix"); return EXA_ERR_SINGULAR; }
  }

  // condensed system and workspace (the HDG arrays; an LDG context needs the element
  // residual, the volume residual's chunk workspace and the Krylov vectors only)
  // B and G (the q columns) exist only for models with q
  const bool hdg = c.scheme != 0;
  const size_t n = P.n, m = P.m, nqn = P.ncq > 0 ? (size_t)P.npe * P.nd * P.ncu : 0;
  if (hdg) {
    EXA_TRY(dev_alloc(c, &c.H, ne * m * m));
    EXA_TRY(dev_alloc(c, &c.F, ne * n * m));
  }
  EXA_TRY(dev_alloc(c, &c.Ru, ne * n));
  if (hdg) EXA_TRY(dev_alloc(c, &c.Rh, ne * m));
  const size_t N = (size_t)std::max(c.ndofuhat(), c.sysN());
  EXA_TRY(dev_alloc(c, &c.b, N));
  if (!hdg) {
  } else if (c.preconditioner == 0) {
    EXA_TRY(dev_alloc(c, &c.Pc, (size_t)P.ncu * P.npf * P.ncu * P.npf * P.nf));
  } else if (c.preconditioner == 2) {
    EXA_TRY(dev_alloc(c, &c.Pc, (size_t)P.ncu * P.npf * P.ncu * P.npf * c.bilu.nse * c.bilu.nnz));
  } else {
    EXA_TRY(dev_alloc(c, &c.Pc, ne * m * m));
  }
  // element chunk: bounded workspace (about 8 GB at most)
  const size_t inv_ws = hdg && exa_inverse_needs_ws((int)n) ? n * n : 0;
  const size_t vol_ws = (size_t)P.nge * P.nc + (size_t)P.nge * P.ncu + (size_t)P.nge * (P.nd + 1) * P.ncu;
  const size_t per_elem = hdg ? sizeof(double) * (n * n + n * nqn + n * m + m * n + m * nqn +
                                                  (size_t)P.nge * (P.nd + 1) * P.ncu * P.nc + n + inv_ws)
                              : sizeof(double) * (vol_ws + n);
  size_t cap = (size_t)8 << 30;
  c.neb = (int)std::max<size_t>(1, std::min<size_t>(std::min<size_t>(ne, cap / per_elem), 65535));
  const size_t nb = c.neb;
  if (hdg) {
    EXA_TRY(dev_alloc(c, &c.wD, nb * n * n));
    EXA_TRY(dev_alloc(c, &c.wB, std::max<size_t>(1, nb * n * nqn)));
    EXA_TRY(dev_alloc(c, &c.wF, nb * n * m));
    EXA_TRY(dev_alloc(c, &c.wK, nb * m * n));
    EXA_TRY(dev_alloc(c, &c.wG, std::max<size_t>(1, nb * m * nqn)));
    EXA_TRY(dev_alloc(c, &c.wRg, nb * P.nge * (P.nd + 1) * P.ncu * P.nc));
    EXA_TRY(dev_alloc(c, &c.wRu, nb * n));
  }
  EXA_TRY(dev_alloc(c, &c.wUG, nb * P.nge * P.nc));
  EXA_TRY(dev_alloc(c, &c.wSG, nb * P.nge * P.ncu));
  EXA_TRY(dev_alloc(c, &c.wRG, nb * P.nge * (P.nd + 1) * P.ncu));
  if (hdg) {
    // T factors of the FP64 volume products: at most 512 MB, the chunk taken in parts
    const size_t per = (size_t)P.npe * P.nge * P.ncu * P.nc;
    c.wT_elems = (int)std::max<size_t>(1, std::min<size_t>(nb, (512u << 20) / (8 * per)));
    EXA_TRY(dev_alloc(c, &c.wT, (size_t)c.wT_elems * per));
  }
  if (inv_ws) EXA_TRY(dev_alloc(c, &c.wInv, nb * inv_ws));
  if ((long long)nb * P.nge * P.npe >= (1LL << 25)) {
    // the chunk-wide GEMMs of the residual: udg and the stage source at the Gauss points, and
    // the integrand's contraction with shapegw (one product each over the whole chunk); small
    // meshes (the served stream's) keep the padding heuristic rather than pay for the timing
    EXA_TRY(exa_gemm_tune(P.nge, P.nc * (int)nb, P.npe, 1, c.st));
    if (c.tdep) EXA_TRY(exa_gemm_tune(P.nge, P.ncu * (int)nb, P.npe, 1, c.st));
    EXA_TRY(exa_gemm_tune(P.npe, P.ncu * (int)nb, P.nge * (P.nd + 1), 1, c.st));
  }
  if (hdg) {
    // the FP64 element products of the assembly: the fastest GEMM tile of each shape is
    // measured once per process and device (q elimination, D^-1 F, K D^-1 F)
    const int kq = P.npe * P.nd, nbt = (int)std::min<size_t>(nb, 512);
    if (P.ncq > 0) {
      EXA_TRY(exa_gemm_tune((int)n, P.npe, kq, nbt, c.st));
      EXA_TRY(exa_gemm_tune((int)n, P.ndf, kq, nbt, c.st));
      EXA_TRY(exa_gemm_tune((int)m, P.npe, kq, nbt, c.st));
      EXA_TRY(exa_gemm_tune((int)m, P.ndf, kq, nbt, c.st));
    }
    EXA_TRY(exa_gemm_tune((int)n, (int)m, (int)n, nbt, c.st));
    EXA_TRY(exa_gemm_tune((int)m, (int)m, (int)n, nbt, c.st));
    EXA_TRY(exa_gemm_tune(P.npe, P.npe, P.nge, nbt, c.st));  // the FP64 volume products
    // and the element inverse (FP64 D of the plain form)
    EXA_TRY(exa_inverse_tune((int)n, (int)std::min<size_t>(nb, 4096), 1, c.st));
  }
  EXA_TRY(dev_alloc(c, &c.V, N * (size_t)(c.restart + 1)));
  EXA_TRY(dev_alloc(c, &c.x, N));
  EXA_TRY(dev_alloc(c, &c.r, N));
  EXA_TRY(dev_alloc(c, &c.w, N));
  if (hdg) EXA_TRY(dev_alloc(c, &c.we, ne * m));
  EXA_TRY(dev_alloc(c, &c.du, ne * n));
  const int VB = exa_vec_blocks();
  EXA_TRY(dev_alloc(c, &c.part_a, VB));
  EXA_TRY(dev_alloc(c, &c.part_b, VB));
  EXA_TRY(dev_alloc(c, &c.part_m, (size_t)VB * (c.restart + 1)));
  const size_t n1 = c.restart + 1;
  EXA_TRY(dev_alloc(c, &c.hess, n1 * c.restart));
  EXA_TRY(dev_alloc(c, &c.gs, n1));
  EXA_TRY(dev_alloc(c, &c.gcs, n1));
  EXA_TRY(dev_alloc(c, &c.gsn, n1));
  EXA_TRY(dev_alloc(c, &c.scal, 16));
  if (c.ppdegree > 1) {
    // start vector of the polynomial's Arnoldi process: seeded normal values on the trace
    // nodes, normalised (the reference draws rand() normals on the element nodes, averages
    // them to a continuous field and takes the face values, setsysstruct.cpp:84-203, 338-352;
    // exa_set_field("randvect") replaces it)
    EXA_TRY(dev_alloc(c, &c.randvect, N));
    EXA_TRY(dev_alloc(c, &c.poly_q, N));
    EXA_TRY(dev_alloc(c, &c.poly_p, N));
    // the system's length (the trace, or the element states of an LDG context)
    const size_t Nr = (size_t)c.sysN();
    std::vector<double> rv(Nr);
    unsigned long long st = 0x9E3779B97F4A7C15ull;
    auto next = [&]() {  // splitmix64, then a uniform in (0, 1)
      st += 0x9E3779B97F4A7C15ull;
      unsigned long long z = st;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z ^= z >> 31;
      return ((double)(z >> 11) + 0.5) / 9007199254740992.0;
    };
    double nrm = 0.0;
    for (size_t i = 0; i < Nr; i += 2) {  // Box-Muller pairs
      const double u1 = next(), u2 = next(), rr = std::sqrt(-2.0 * std::log(u1));
      rv[i] = rr * std::cos(6.283185307179586 * u2);
      if (i + 1 < Nr) rv[i + 1] = rr * std::sin(6.283185307179586 * u2);
    }
    for (double v : rv) nrm += v * v;
    nrm = std::sqrt(nrm);
    for (double& v : rv) v /= nrm;
    EXA_CUDA(cudaMemcpyAsync(c.randvect, rv.data(), sizeof(double) * Nr, cudaMemcpyHostToDevice, c.st));
    EXA_CUDA(cudaStreamSynchronize(c.st));
  }
  if (c.RBdim > 0) {
    EXA_TRY(dev_alloc(c, &c.rbW, N * (size_t)c.RBdim));
    EXA_TRY(dev_alloc(c, &c.rbU, N * (size_t)c.RBdim));
    EXA_TRY(dev_alloc(c, &c.rbD, (size_t)c.RBdim * (c.RBdim + 1)));
  }
  if (c.tdep) {
    EXA_TRY(dev_alloc(c, &c.udgprev, ne * n));
    EXA_TRY(dev_alloc(c, &c.utmp, ne * n));
  }
  // staging for the Hessenberg matrix and Givens vector, then one residual slot per step
  EXA_CUDA(cudaMallocHost((void**)&c.pinned, sizeof(double) * (n1 * (n1 + 3) + 64)));
  for (int k = 0; k < 2; ++k) {
    EXA_CUDA(cudaEventCreateWithFlags(&c.step_ev[k], cudaEventDisableTiming));
    c.arnoldi_graph[k].assign(c.restart, nullptr);
    c.arnoldi_launches[k].assign(c.restart, 0);
    c.arnoldi_seen[k].assign(c.restart, 0);
  }
  EXA_CUDA(cudaStreamSynchronize(c.st));
  return EXA_OK;
}

namespace {
// Frees one allocation of the context (stream-ordered) and takes it off its list.
void dev_release(ExaCtx& c, void* p, size_t bytes) {
  if (!p) return;
  for (size_t i = 0; i < c.allocs.size(); ++i)
    if (c.allocs[i] == p) {
      c.allocs.erase(c.allocs.begin() + (long long)i);
      c.alloc_bytes -= (long long)bytes;
      break;
    }
  cudaFreeAsync(p, c.st);
}

size_t precond_blocks(const ExaCtx& c) {
  const ExaDims& P = c.P;
  const size_t ncf = (size_t)P.ncu * P.npf;
  if (c.preconditioner == 0) return ncf * ncf * P.nf;
  if (c.preconditioner == 2) return ncf * ncf * c.bilu.nse * c.bilu.nnz;
  return (size_t)P.ne * P.m * P.m;
}

// The FP64 condensed blocks for all elements (full) or the mixed form's staging only: H for
// one element chunk, no F and no FP64 preconditioner blocks.  At 32^3 hexahedra of 3D Euler
// (p = 3) the full set is 105 GB, which the mixed form cannot hold beside its FP32 copies.
// The plain form's captured GMRES steps name the freed arrays, so they are dropped.
int fp64_blocks(ExaCtx& c, bool full) {
  if (full == c.fp64_full) return EXA_OK;
  const ExaDims& P = c.P;
  const size_t ne = P.ne, n = P.n, m = P.m, nb = c.neb;
  if (c.st2) EXA_CUDA(cudaStreamSynchronize(c.st2));
  EXA_CUDA(cudaStreamSynchronize(c.st));
  for (cudaGraphExec_t& g : c.arnoldi_graph[0]) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  std::fill(c.arnoldi_seen[0].begin(), c.arnoldi_seen[0].end(), 0);
  dev_release(c, c.H, sizeof(double) * (full ? nb : ne) * m * m);
  c.H = nullptr;
  if (full) {
    EXA_TRY(dev_alloc(c, &c.H, ne * m * m));
    EXA_TRY(dev_alloc(c, &c.F, ne * n * m));
    EXA_TRY(dev_alloc(c, &c.Pc, precond_blocks(c)));
  } else {
    dev_release(c, c.F, sizeof(double) * ne * n * m);
    dev_release(c, c.Pc, sizeof(double) * precond_blocks(c));
    c.F = nullptr;
    c.Pc = nullptr;
    EXA_TRY(dev_alloc(c, &c.H, nb * m * m));
  }
  c.fp64_full = full;
  return EXA_OK;
}
}  // namespace

// Switch between the plain FP64 form (0) and the mixed-precision form (1).  The FP32
// arrays of the mixed form are allocated on the first switch to it and kept afterwards;
// the FP64 blocks that the new form does not read are freed (fp64_blocks).
int exa_ctx_set_precision(ExaCtx& c, int mode) {
  if (mode != 0 && mode != 1) {
    exa_set_error("precision mode %d: 0 (FP64) or 1 (FP32/TF32 elimination with FP64 refinement)", mode);
    return EXA_ERR_ARG;
  }
  if (mode == 1 && c.scheme == 0) {
    exa_set_error("the mixed-precision form condenses the HDG system; the LDG path runs in FP64");
    return EXA_ERR_UNSUPPORTED;
  }
  if (c.scheme == 0) return EXA_OK;  // LDG: FP64 already, no condensed arrays
  if (mode == 1) {
    EXA_TRY(fp64_blocks(c, false));
    // the mixed assembly writes only the face blocks of the chunk arrays F, K and H (its
    // products read them): their other entries must be zero, which a plain assembly may
    // have overwritten
    const ExaDims& P = c.P;
    const size_t nb = c.neb, n = P.n, m = P.m;
    EXA_CUDA(cudaMemsetAsync(c.wF, 0, sizeof(double) * nb * n * m, c.st));
    EXA_CUDA(cudaMemsetAsync(c.wK, 0, sizeof(double) * nb * m * n, c.st));
    EXA_CUDA(cudaMemsetAsync(c.H, 0, sizeof(double) * nb * m * m, c.st));
  }
  if (mode == 1 && c.H32 == nullptr) {
    const ExaDims& P = c.P;
    const size_t ne = P.ne, n = P.n, m = P.m, nb = c.neb;
    const int kq = P.npe * P.nd, kg = exa_tc::qk_group(P.npe), kq4 = kg * P.nd;
    // a packed operand for `count` elements with `per` parts each (batch strides sb = per
    // parts, sb2 = one part); split: hi and lo TF32 parts in HBM, else FP32 values split by
    // the GEMM in shared memory
    auto packed = [&](UPacked& u, int R, int K, int TR, size_t count, int per, bool split) -> int {
      const long long sz = exa_pack_size(R, K);
      u.R = R; u.K = K; u.TR = TR;
      u.sb = sz * per;
      u.sb2 = sz;
      EXA_TRY(dev_alloc(c, &u.hi, (size_t)sz * per * count));
      if (split) EXA_TRY(dev_alloc(c, &u.lo, (size_t)sz * per * count));
      else u.lo = nullptr;
      return EXA_OK;
    };
    const int r16m = (P.m + 15) / 16 * 16;
    if (P.ncq > 0) {
      // Minv C, Minv E as B operands: row j (column of the product), k = (l, d) at
      // l + qk_group(npe) d (zeros between the groups)
      EXA_TRY(packed(c.MCp, P.npe, kq4, (P.npe + 15) / 16 * 16, ne, 1, false));
      EXA_TRY(packed(c.MEp, P.ndf, kq4, (P.ndf + 15) / 16 * 16, ne, 1, false));
      EXA_TRY(exa_pack(c.MC, 1, kq, 1, (long long)kq * P.npe, 0, (int)ne, 1, c.MCp, c.st, kg, P.npe));
      EXA_TRY(exa_pack(c.ME, 1, kq, 1, (long long)kq * P.ndf, 0, (int)ne, 1, c.MEp, c.st, kg, P.npe));
      // B and G as A operands, one part per trace component b, with the same K
      EXA_TRY(packed(c.wBp, P.n, kq4, 128, nb, P.ncu, false));
      EXA_TRY(packed(c.wGp, P.m, kq4, 128, nb, P.ncu, false));
    }
    if (exa_vol_mat_tc_fits(P)) {
      // basis at the Gauss points: row j (node), k = g
      EXA_TRY(packed(c.Sp, P.npe, P.nge, 128, 1, 1, true));
      EXA_TRY(exa_pack(c.shapegt, 1, P.nge, 1, 0, 0, 1, 1, c.Sp, c.st));
      const long long nw = (long long)P.npe * P.nge * (P.nd + 1);
      EXA_TRY(dev_alloc(c, &c.shapegw32, (size_t)nw));
      EXA_TRY(exa_k_to_f32(c.shapegw, c.shapegw32, nw, c.st));
    }
    EXA_TRY(packed(c.Dinvp, P.n, P.n, 128, nb, 1, false));
    EXA_TRY(packed(c.wFp, P.m, P.n, r16m, nb, 1, false));
    EXA_TRY(packed(c.Kp, P.m, P.n, 128, nb, 1, false));
    EXA_TRY(packed(c.DinvFp, P.m, P.n, r16m, nb, 1, false));
    EXA_TRY(dev_alloc(c, &c.H32, ne * m * m));
    EXA_TRY(dev_alloc(c, &c.F32, ne * n * m));
    EXA_TRY(dev_alloc(c, &c.K32, ne * m * n));
    EXA_TRY(dev_alloc(c, &c.Dinv32, ne * n * n));
    EXA_TRY(exa_inverse_tune((int)n, (int)std::min<size_t>(nb, 4096), 0, c.st));
    if (exa_inverse_tc32_pk((int)n) > 0) {
      EXA_TRY(dev_alloc(c, &c.wInv32, nb * (size_t)exa_inverse_tc32_ws((int)n)));
      EXA_TRY(dev_alloc(c, &c.wInvPk, nb * (size_t)exa_inverse_tc32_pk((int)n)));
    }
    if (c.preconditioner == 0)
      EXA_TRY(dev_alloc(c, &c.Pc32, (size_t)P.ncu * P.npf * P.ncu * P.npf * P.nf));
    else if (c.preconditioner == 2)
      EXA_TRY(dev_alloc(c, &c.Pc32, (size_t)P.ncu * P.npf * P.ncu * P.npf * c.bilu.nse * c.bilu.nnz));
    else
      EXA_TRY(dev_alloc(c, &c.Pc32, ne * m * m));
    c.d_uflag = c.d_flag + 1;
    EXA_CUDA(cudaStreamSynchronize(c.st));
  }
  if (mode == 0) EXA_TRY(fp64_blocks(c, true));
  c.precision = mode;
  return EXA_OK;
}

// Puts a context back to the start of a new solve of the same mesh and discretization with the
// physical parameters, tau and initial state of `app` / `sol` (the serving path reuses contexts
// this way, keeping master, mesh, geometry and q matrices resident).
int exa_ctx_reset(ExaCtx& c, const double* app, long long napp, const double* sol, long long nsol) {
  Blob A = split_blob(app, napp), S = split_blob(sol, nsol);
  if (!A.ok || !S.ok || A.nsize.size() < 9 || S.nsize.size() < 3) {
    exa_set_error("reset: malformed app or sol blob");
    return EXA_ERR_ARG;
  }
  if ((size_t)A.nsize[6] != c.h_param.size() || A.nsize[8] < 1) {
    exa_set_error("reset: %lld physical parameters, the context has %zu", A.nsize[6], c.h_param.size());
    return EXA_ERR_ARG;
  }
  EXA_CUDA(cudaSetDevice(c.device));
  c.h_param.assign(A.part[6], A.part[6] + A.nsize[6]);
  if (!c.h_param.empty())
    EXA_CUDA(cudaMemcpyAsync(c.param, c.h_param.data(), sizeof(double) * c.h_param.size(), cudaMemcpyHostToDevice,
                             c.st));
  EXA_CUDA(cudaMemcpyAsync(c.tau, A.part[8], sizeof(double) * (size_t)A.nsize[8], cudaMemcpyHostToDevice, c.st));
  c.time0 = (c.tdep == 1 && A.nsize[5] > 0) ? A.part[5][0] : 0.0;
  c.time = c.time0;
  c.dtfactor = 0.0;
  c.last_gmres_iters = c.last_newton_iters = c.total_gmres_iters = 0;
  c.last_norm0 = c.last_norm = 0.0;
  c.rb_cur = c.rb_removed = 0;
  EXA_CUDA(cudaMemsetAsync(c.sdg, 0, sizeof(double) * (size_t)c.P.npe * c.P.ncu * c.P.ne, c.st));
  EXA_TRY(init_solution(c, S));
  EXA_CUDA(cudaStreamSynchronize(c.st));
  return EXA_OK;
}

// 64-bit FNV-1a over the blobs that fix a context's resident data: master, mesh, sol, and app
// without its physical parameters and tau (parts 6 and 8), which exa_ctx_reset replaces.
unsigned long long exa_ctx_key(const double* app, long long napp, const double* master, long long nmaster,
                               const double* mesh, long long nmesh, const double* sol, long long nsol) {
  unsigned long long h = 1469598103934665603ULL;
  auto mix = [&](const void* p, size_t n) {
    const unsigned char* b = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) {
      h ^= b[i];
      h *= 1099511628211ULL;
    }
  };
  Blob A = split_blob(app, napp);
  if (A.ok) {
    mix(app, sizeof(double) * (size_t)(1 + A.nsize.size()));  // the part sizes
    for (size_t i = 0; i < A.part.size(); ++i)
      if (i != 6 && i != 8) mix(A.part[i], sizeof(double) * (size_t)A.nsize[i]);
  } else {
    mix(app, sizeof(double) * (size_t)std::max(0LL, napp));
  }
  mix(master, sizeof(double) * (size_t)std::max(0LL, nmaster));
  mix(mesh, sizeof(double) * (size_t)std::max(0LL, nmesh));
  mix(sol, sizeof(double) * (size_t)std::max(0LL, nsol));
  return h;
}

// Device bytes a context for these blobs will hold (the arrays exa_ctx_init allocates, with
// nf bounded by ne * nfe), for admission before it exists; 0 for malformed blobs.
long long exa_ctx_estimate_bytes(const double* app, long long napp, const double* master, long long nmaster,
                                 const double* mesh, long long nmesh, int precision) {
  Blob A = split_blob(app, napp), M = split_blob(master, nmaster), Me = split_blob(mesh, nmesh);
  if (!A.ok || !M.ok || !Me.ok || A.nsize.size() < 9 || M.nsize.size() < 1 || Me.nsize.size() < 1) return 0;
  const double ncu = A.part[0][6], nc = A.part[0][5], ncq = A.part[0][7];
  const double restart = A.part[2][15], precond = A.part[1][6];
  const double nd = M.part[0][0], npe = M.part[0][5], npf = M.part[0][6], nge = M.part[0][7], ngf = M.part[0][8];
  const double ne = Me.part[0][1], nfe = Me.part[0][4];
  const double nf = ne * nfe, n = npe * ncu, ndf = npf * nfe, m = ndf * ncu, N = ncu * npf * nf;
  const double nqn = ncq > 0 ? npe * nd * ncu : 0;
  double per_elem = m * m + n * m + n + m + npe * nc + npe * ncu + nge * (nd + nd * nd + 1) + nfe * ngf * (2 * nd + 1) +
                    (ncq > 0 ? npe * npe * nd + npe * ndf * nd + npe * npe * (2 + nd) + npe * ndf * nd : 0) + m + n;
  // q recovery workspace (Gauss-point u, its geometric products, C u)
  per_elem += ncq > 0 ? nge * ncu * (1 + nd * nd) + npe * nd * ncu : 0;
  per_elem += precond == 1 ? m * m : 0;
  // element chunk workspace (the whole mesh when it fits in 8 GB)
  per_elem += n * n + n * nqn + 2 * n * m + m * nqn + nge * (nd + 1) * ncu * nc + n + (n > 160 ? n * n : 0);
  per_elem += nge * (nc + ncu + (nd + 1) * ncu);  // Gauss-point values and Ru integrand of a chunk
  // preconditioner blocks: block Jacobi one per face; block ILU(0) one per stored block of the
  // sub-domain face graph, at most the face itself and the other faces of its two elements
  const double ncf2 = ncu * npf * ncu * npf;
  const double pblocks = precond == 0 ? ncf2 * nf : (precond == 2 ? ncf2 * nf * (1 + 2 * (nfe - 1)) : 0.0);
  // volume-product T factors: at most 512 MB
  const double wt = std::min(ne * npe * nge * ncu * nc, (double)(64 << 20));
  double words = ne * per_elem + N * (restart + 6) + pblocks + wt;
  if (precision == 1) words *= 1.75;
  return (long long)(8.0 * words) + (16LL << 20);
}

void exa_ctx_free(ExaCtx& c) {
  if (c.device >= 0) cudaSetDevice(c.device);
  // the second stream first: after an error it may still use arrays that are freed below
  if (c.st2) cudaStreamSynchronize(c.st2);
  if (c.st) cudaStreamSynchronize(c.st);
  exa_prof_free(c);
  for (void* p : c.allocs) {
    if (c.st) cudaFreeAsync(p, c.st);
    else cudaFree(p);
  }
  if (c.st) cudaStreamSynchronize(c.st);
  c.allocs.clear();
  c.alloc_bytes = 0;
  if (c.pinned) cudaFreeHost(c.pinned);
  c.pinned = nullptr;
  for (int k = 0; k < 2; ++k) {
    for (cudaGraphExec_t g : c.arnoldi_graph[k])
      if (g) cudaGraphExecDestroy(g);
    c.arnoldi_graph[k].clear();
    if (c.step_ev[k]) cudaEventDestroy(c.step_ev[k]);
    c.step_ev[k] = nullptr;
  }
  if (c.st2) cudaStreamDestroy(c.st2);
  c.st2 = nullptr;
  if (c.ev_q) cudaEventDestroy(c.ev_q);
  if (c.ev_inv) cudaEventDestroy(c.ev_inv);
  c.ev_q = c.ev_inv = nullptr;
  if (c.st) cudaStreamDestroy(c.st);
  c.st = nullptr;
}

// ==================================================================================
// C ABI
// ==================================================================================
struct exa_ctx {
  ExaCtx c;
};

namespace {

struct FieldRef {
  double* p;
  long long n;
  float* p32 = nullptr;  // FP32 arrays of the mixed-precision form (p is null then)
};

bool field(ExaCtx& c, const char* name, FieldRef& f) {
  const ExaDims& P = c.P;
  const long long ne = P.ne, n = P.n, m = P.m, N = c.sysN();
  const std::string s(name ? name : "");
  if (c.scheme == 0 && s != "udg" && s != "uh" && s != "Ru" && s != "b" && s != "x" && s != "sdg" && s != "elemg" &&
      s != "faceg" && s != "randvect")
    return false;  // an LDG context holds no condensed or preconditioner arrays
  if (s == "udg") f = {c.udg, (long long)P.npe * P.nc * ne};
  else if (s == "uh") f = {c.uh, c.ndofuhat()};
  else if (s == "Ru" && c.scheme == 0) f = {c.ldg_R, N};  // the LDG residual of the last exa_residual
  else if (s == "H" && c.fp64_full) f = {c.H, m * m * ne};
  else if (s == "F" && c.fp64_full) f = {c.F, n * m * ne};
  else if (s == "Ru") f = {c.Ru, n * ne};
  else if (s == "Rh") f = {c.Rh, m * ne};
  else if (s == "b") f = {c.b, N};
  else if (s == "x") f = {c.x, N};
  else if (s == "sdg") f = {c.sdg, n * ne};
  else if (s == "randvect" && c.randvect) f = {c.randvect, N};
  else if (s == "P" && c.fp64_full)
    f = {c.Pc, c.preconditioner == 0   ? (long long)P.ncu * P.npf * P.ncu * P.npf * P.nf
               : c.preconditioner == 2 ? (long long)P.ncu * P.npf * P.ncu * P.npf * c.bilu.nse * c.bilu.nnz
                                       : m * m * ne};
  else if (s == "MinvC") f = {c.MC, P.ncq > 0 ? (long long)P.npe * P.npe * P.nd * ne : 0};
  else if (s == "MinvE") f = {c.ME, P.ncq > 0 ? (long long)P.npe * P.ndf * P.nd * ne : 0};
  else if (s == "elemg") f = {c.elemg, (long long)P.elemg_stride() * ne};
  else if (s == "faceg") f = {c.faceg, (long long)P.faceg_stride() * P.nfe * ne};
  else if (s == "K" && c.neb == P.ne) f = {c.wK, m * n * ne};
  else if (s == "B" && c.neb == P.ne && !(c.precision == 1 && c.Sp.hi))  // else B exists only packed in FP32
    f = {c.wB, n * (long long)P.npe * P.nd * P.ncu * ne};
  else if (s == "Dinv" && c.neb == P.ne) f = {c.wD, n * n * ne};
  else if (s == "H32" && c.H32) f = {nullptr, m * m * ne, c.H32};
  else if (s == "F32" && c.F32) f = {nullptr, n * m * ne, c.F32};
  else if (s == "K32" && c.K32) f = {nullptr, m * n * ne, c.K32};
  else if (s == "Dinv32" && c.Dinv32) f = {nullptr, n * n * ne, c.Dinv32};
  else return false;
  return true;
}

int guard(exa_ctx* h) {
  if (!h) {
    exa_set_error("null context");
    return EXA_ERR_ARG;
  }
  cudaError_t e = cudaSetDevice(h->c.device);
  if (e != cudaSuccess) {
    exa_set_error("cudaSetDevice(%d): %s", h->c.device, cudaGetErrorString(e));
    return EXA_ERR_CUDA;
  }
  return EXA_OK;
}

}  // namespace

extern "C" {

const char* exa_last_error(void) { return exa_get_error(); }

int exa_create(const double* app, long long napp, const double* master, long long nmaster, const double* mesh,
               long long nmesh, const double* sol, long long nsol, int device, exa_ctx** out) {
  if (!out) {
    exa_set_error("null output handle");
    return EXA_ERR_ARG;
  }
  *out = nullptr;
  exa_ctx* h = new exa_ctx();
  int s = exa_ctx_init(h->c, app, napp, master, nmaster, mesh, nmesh, sol, nsol, device);
  if (s != EXA_OK) {
    exa_ctx_free(h->c);
    delete h;
    return s;
  }
  *out = h;
  return EXA_OK;
}

void exa_destroy(exa_ctx* h) {
  if (!h) return;
  exa_ctx_free(h->c);
  delete h;
}

int exa_sizes(exa_ctx* h, long long* out) {
  EXA_TRY(guard(h));
  const ExaDims& P = h->c.P;
  const long long v[16] = {P.ne, P.nf, P.nf0, P.npe, P.npf, P.nfe, P.nc, P.ncu, P.nd,
                           P.n,  P.m,  h->c.ndofuhat(), P.nge, P.ngf, h->c.neb, h->c.preconditioner};
  for (int i = 0; i < 16; ++i) out[i] = v[i];
  return EXA_OK;
}

int exa_get_field(exa_ctx* h, const char* name, double* host, long long n) {
  EXA_TRY(guard(h));
  FieldRef f{};
  if (!field(h->c, name, f) || !host || n != f.n) {
    exa_set_error("get_field('%s'): unknown name or size %lld != %lld", name ? name : "", n, f.n);
    return EXA_ERR_ARG;
  }
  EXA_CUDA(cudaStreamSynchronize(h->c.st));
  if (n && f.p32) {
    std::vector<float> t((size_t)n);
    EXA_CUDA(cudaMemcpy(t.data(), f.p32, sizeof(float) * n, cudaMemcpyDeviceToHost));
    for (long long i = 0; i < n; ++i) host[i] = t[(size_t)i];
  } else if (n) {
    EXA_CUDA(cudaMemcpy(host, f.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
  }
  return EXA_OK;
}

int exa_set_field(exa_ctx* h, const char* name, const double* host, long long n) {
  EXA_TRY(guard(h));
  FieldRef f{};
  if (!field(h->c, name, f) || !host || n != f.n) {
    exa_set_error("set_field('%s'): unknown name or size %lld != %lld", name ? name : "", n, f.n);
    return EXA_ERR_ARG;
  }
  EXA_CUDA(cudaStreamSynchronize(h->c.st));
  if (n && f.p32) {
    std::vector<float> t(host, host + n);
    EXA_CUDA(cudaMemcpy(f.p32, t.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  } else if (n) {
    EXA_CUDA(cudaMemcpy(f.p, host, sizeof(double) * n, cudaMemcpyHostToDevice));
  }
  return EXA_OK;
}

int exa_field_ptr(exa_ctx* h, const char* name, double** dev, long long* n) {
  EXA_TRY(guard(h));
  FieldRef f{};
  if (!field(h->c, name, f) || !dev || !n) {
    exa_set_error("field_ptr('%s'): unknown name", name ? name : "");
    return EXA_ERR_ARG;
  }
  *dev = f.p32 ? reinterpret_cast<double*>(f.p32) : f.p;
  *n = f.n;
  return EXA_OK;
}

int exa_get_connectivity(exa_ctx* h, int* f2e, int* elemcon) {
  EXA_TRY(guard(h));
  EXA_CUDA(cudaStreamSynchronize(h->c.st));
  const ExaDims& P = h->c.P;
  if (f2e) EXA_CUDA(cudaMemcpy(f2e, h->c.f2e, sizeof(int) * 4 * (size_t)P.nf, cudaMemcpyDeviceToHost));
  if (elemcon) EXA_CUDA(cudaMemcpy(elemcon, h->c.elemcon, sizeof(int) * (size_t)P.ndf * P.ne, cudaMemcpyDeviceToHost));
  return EXA_OK;
}

int exa_set_time(exa_ctx* h, double time, double dtfactor) {
  EXA_TRY(guard(h));
  h->c.time = time;
  h->c.dtfactor = dtfactor;
  return EXA_OK;
}

int exa_set_step_time(exa_ctx* h, double time0) {
  EXA_TRY(guard(h));
  if (!std::isfinite(time0)) {
    exa_set_error("set_step_time: time %g is not finite", time0);
    return EXA_ERR_ARG;
  }
  h->c.time0 = time0;
  h->c.time = time0;
  return EXA_OK;
}

int exa_assemble(exa_ctx* h) {
  EXA_TRY(guard(h));
  return exa_drv_assemble(h->c);
}

int exa_residual(exa_ctx* h, double* norm) {
  EXA_TRY(guard(h));
  EXA_TRY(exa_drv_residual(h->c, norm));
  EXA_CUDA(cudaStreamSynchronize(h->c.st));
  return EXA_OK;
}

int exa_matvec(exa_ctx* h, const double* v, double* w) {
  EXA_TRY(guard(h));
  EXA_TRY(exa_drv_matvec(h->c, v, w));
  EXA_CUDA(cudaStreamSynchronize(h->c.st));
  return EXA_OK;
}

int exa_precond(exa_ctx* h, const double* v, double* w) {
  EXA_TRY(guard(h));
  if (v == w) {
    exa_set_error("precond: input and output must differ");
    return EXA_ERR_ARG;
  }
  EXA_TRY(exa_drv_precond(h->c, v, w));
  EXA_CUDA(cudaStreamSynchronize(h->c.st));
  return EXA_OK;
}

int exa_gmres(exa_ctx* h, int* iters, double* relerr) {
  EXA_TRY(guard(h));
  int it = 0;
  double re = 0.0;
  EXA_TRY(exa_drv_gmres(h->c, &it, &re));
  if (iters) *iters = it;
  if (relerr) *relerr = re;
  if (!h->c.last_gmres_converged) {
    // the reference prints a warning with the relative error and goes on (gmres.cpp:586-594);
    // a standalone call reports it, with the iterations and error filled in
    exa_set_error("GMRES(%d) does not converge to the tolerance within %d iterations: relative error %.6e",
                  h->c.restart, it, re);
    return EXA_ERR_NOTCONV;
  }
  return EXA_OK;
}

int exa_getq(exa_ctx* h) {
  EXA_TRY(guard(h));
  EXA_TRY(exa_drv_getq(h->c));
  EXA_CUDA(cudaStreamSynchronize(h->c.st));
  return EXA_OK;
}

int exa_newton(exa_ctx* h, int* iters, double* norm) {
  EXA_TRY(guard(h));
  int it = 0;
  double nr = 0.0;
  int s = exa_drv_newton(h->c, &it, &nr);
  if (iters) *iters = it;
  if (norm) *norm = nr;
  EXA_CUDA(cudaStreamSynchronize(h->c.st));
  return s;
}

int exa_dirk(exa_ctx* h, int nsteps, int* newton_iters, int max_out) {
  EXA_TRY(guard(h));
  return exa_drv_dirk(h->c, nsteps, newton_iters, max_out);
}

int exa_dirk_stage(exa_ctx* h, int istep, int stage, int* iters, double* norm) {
  EXA_TRY(guard(h));
  EXA_TRY(exa_drv_dirk_stage(h->c, istep, stage, iters, norm));
  EXA_CUDA(cudaStreamSynchronize(h->c.st));
  return EXA_OK;
}

int exa_stream(exa_ctx* h, void** stream) {
  EXA_TRY(guard(h));
  *stream = (void*)h->c.st;
  return EXA_OK;
}

int exa_solve(exa_ctx* h, const double* udg_in, const double* uh_in, double* udg_out, double* uh_out, int* iters,
              double* norm) {
  EXA_TRY(guard(h));
  ExaCtx& c = h->c;
  const size_t nu = (size_t)c.P.npe * c.P.nc * c.P.ne, nh = (size_t)c.ndofuhat();
  if (udg_in) EXA_CUDA(cudaMemcpyAsync(c.udg, udg_in, sizeof(double) * nu, cudaMemcpyHostToDevice, c.st));
  if (uh_in) EXA_CUDA(cudaMemcpyAsync(c.uh, uh_in, sizeof(double) * nh, cudaMemcpyHostToDevice, c.st));
  int it = 0;
  double nr = 0.0;
  int s = exa_drv_newton(c, &it, &nr);
  if (iters) *iters = it;
  if (norm) *norm = nr;
  if (s != EXA_OK) return s;
  if (udg_out) EXA_CUDA(cudaMemcpyAsync(udg_out, c.udg, sizeof(double) * nu, cudaMemcpyDeviceToHost, c.st));
  if (uh_out) EXA_CUDA(cudaMemcpyAsync(uh_out, c.uh, sizeof(double) * nh, cudaMemcpyDeviceToHost, c.st));
  EXA_CUDA(cudaStreamSynchronize(c.st));
  return EXA_OK;
}

int exa_set_precision(exa_ctx* h, int mode, double inner_tol, double rtol) {
  EXA_TRY(guard(h));
  if (!(inner_tol > 0.0 && inner_tol < 1.0) || !(rtol >= 0.0 && rtol < 1.0)) {
    exa_set_error("set_precision: inner_tol must lie in (0, 1) and rtol in [0, 1)");
    return EXA_ERR_ARG;
  }
  EXA_TRY(exa_ctx_set_precision(h->c, mode));
  h->c.mixed_inner_tol = inner_tol;
  h->c.mixed_rtol = rtol;
  return EXA_OK;
}

int exa_last_residual(exa_ctx* h, double* initial, double* final_norm) {
  EXA_TRY(guard(h));
  if (initial) *initial = h->c.last_norm0;
  if (final_norm) *final_norm = h->c.last_norm;
  return EXA_OK;
}

int exa_profile(exa_ctx* h, int enable) {
  EXA_TRY(guard(h));
  return exa_prof_enable(h->c, enable);
}

int exa_profile_read(exa_ctx* h, int nphase, double* ms, long long* count, double* flops) {
  EXA_TRY(guard(h));
  if (nphase < 0 || nphase > EXA_NPHASE) {
    exa_set_error("profile: nphase = %d, at most %d phases", nphase, (int)EXA_NPHASE);
    return EXA_ERR_ARG;
  }
  EXA_TRY(exa_prof_flush(h->c));
  for (int i = 0; i < nphase; ++i) {
    if (ms) ms[i] = h->c.prof.ms[i];
    if (count) count[i] = h->c.prof.count[i];
    if (flops) flops[i] = h->c.prof.flops[i];
  }
  return EXA_OK;
}

int exa_stats(exa_ctx* h, long long* out) {
  EXA_TRY(guard(h));
  out[0] = h->c.last_gmres_iters;
  out[1] = h->c.last_newton_iters;
  out[2] = h->c.total_gmres_iters;
  out[3] = 0;
  return EXA_OK;
}

int exa_synchronize(exa_ctx* h) {
  EXA_TRY(guard(h));
  EXA_CUDA(cudaStreamSynchronize(h->c.st));
  return EXA_OK;
}

}  // extern "C"

extern "C" int exa_connectivity_host(const int* t, const int* bf, const int* perm, const double* xpf, int dim,
                                     int elemtype, int ne, int npe, int npf, int* f2e, int* elemcon, int* nf0) {
  ExaConn conn;
  const int nf = exa_build_connectivity(t, bf, perm, xpf, dim, elemtype, ne, npe, npf, conn);
  if (nf < 0) {
    exa_set_error("mesh connectivity is wrong (unmatched face)");
    return -EXA_ERR_MESH;
  }
  std::memcpy(f2e, conn.f2e.data(), sizeof(int) * conn.f2e.size());
  std::memcpy(elemcon, conn.elemcon.data(), sizeof(int) * conn.elemcon.size());
  *nf0 = conn.nf0;
  return nf;
}

extern "C" int exa_bilu0_ordering(const int* cartgridpart, int ncgp, const int* f2e, int nf, int nfe, int ne,
                                  int* row_ptr, int cap_row_ptr, int* col_ind, int cap_col_ind, int* face,
                                  int cap_face, int* nse) {
  ExaBilu b;
  char msg[256] = "";
  if (exa_bilu_setup(cartgridpart, ncgp, f2e, nf, nfe, ne, b, msg, sizeof(msg)) != 0) {
    exa_set_error("block ILU(0): %s", msg);
    return -EXA_ERR_ARG;
  }
  if (b.nfse + 1 > cap_row_ptr || b.nnz > cap_col_ind || (long long)b.nse * b.nfse > cap_face) {
    exa_set_error("block ILU(0) ordering: output buffers too small");
    return -EXA_ERR_ARG;
  }
  std::memcpy(row_ptr, b.row_ptr.data(), sizeof(int) * b.row_ptr.size());
  std::memcpy(col_ind, b.col_ind.data(), sizeof(int) * b.col_ind.size());
  std::memcpy(face, b.face.data(), sizeof(int) * b.face.size());
  *nse = b.nse;
  return b.nfse;
}

// Batched FP64 primitives on device pointers (the kernels the assembly uses).
extern "C" int exa_dgemm_batched(int M, int N, int K, double alpha, const double* A, long long lda, long long sA,
                                 const double* B, long long ldb, long long sB, double beta, double* C, long long ldc,
                                 long long sC, int batch, void* stream) {
  GemmBatch g{};
  g.M = M; g.N = N; g.K = K; g.alpha = alpha; g.beta = beta;
  g.A = A; g.lda = lda; g.sA = sA; g.sA2 = 0;
  g.B = B; g.ldb = ldb; g.sB = sB; g.sB2 = 0;
  g.C = C; g.ldc = ldc; g.sC = sC; g.sC2 = 0;
  g.batch = batch; g.batch2 = 1;
  return exa_gemm(g, (cudaStream_t)stream);
}

extern "C" int exa_gemm_tf32_batched(int M, int N, int K, double alpha, const void* A, int a_f64, long long lda,
                                     long long sA, const void* B, int b_f64, long long ldb, long long sB,
                                     double beta, void* C, int c_f64, long long ldc, long long sC, int batch,
                                     int* flag_dev, void* stream) {
  UGemm g{};
  g.M = M; g.N = N; g.K = K; g.alpha = alpha; g.beta = beta;
  g.A = A; g.ta = a_f64 ? EXA_T_F64 : EXA_T_F32; g.lda = lda; g.sA = sA; g.sA2 = 0;
  g.B = B; g.tb = b_f64 ? EXA_T_F64 : EXA_T_F32; g.ldb = ldb; g.sB = sB; g.sB2 = 0;
  g.Cin = C; g.tci = c_f64 ? EXA_T_F64 : EXA_T_F32; g.ldci = ldc; g.sCi = sC; g.sCi2 = 0;
  g.C = C; g.tco = g.tci; g.ldc = ldc; g.sC = sC; g.sC2 = 0;
  g.batch = batch; g.batch2 = 1;
  return exa_gemm_tf32(g, flag_dev, (cudaStream_t)stream);
}

// 3xTF32 product through packed copies of A and B (allocated for the call and freed after
// it, so the call synchronises the stream); C is FP32.
extern "C" int exa_gemm_3xtf32_batched(int M, int N, int K, double alpha, const void* A, int a_f64, long long lda,
                                       long long sA, const void* B, int b_f64, long long ldb, long long sB,
                                       double beta, float* C, long long ldc, long long sC, int batch, int* flag_dev,
                                       void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || batch <= 0 || N > 1024) {
    exa_set_error("3xtf32 gemm: sizes M %d N %d K %d batch %d (N <= 1024)", M, N, K, batch);
    return EXA_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long long pa = exa_pack_size(M, K), pb = exa_pack_size(N, K);
  float* buf = nullptr;
  EXA_CUDA(cudaMalloc(&buf, sizeof(float) * 2 * (size_t)(pa + pb) * batch));
  UPacked Ap{buf, buf + pa * batch, pa, 0, M, K, 128};
  UPacked Bp{buf + 2 * pa * batch, buf + 2 * pa * batch + pb * batch, pb, 0, N, K, (N + 15) / 16 * 16};
  int s = exa_pack(A, a_f64, 1, lda, sA, 0, batch, 1, Ap, st);
  if (s == EXA_OK) s = exa_pack(B, b_f64, ldb, 1, sB, 0, batch, 1, Bp, st);
  if (s == EXA_OK) {
    UGemmP g{};
    g.M = M; g.N = N; g.K = K; g.alpha = alpha; g.beta = beta;
    g.A = Ap; g.B = Bp;
    g.Cin = C; g.tci = EXA_T_F32; g.ldci = ldc; g.sCi = sC; g.sCi2 = 0;
    g.C = C; g.tco = EXA_T_F32; g.ldc = ldc; g.sC = sC; g.sC2 = 0;
    g.nout = 0; g.batch = batch; g.batch2 = 1;
    s = exa_gemm_3xtf32(g, flag_dev, st);
  }
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(buf);
  if (s != EXA_OK) return s;
  if (e != cudaSuccess) {
    exa_set_error("3xtf32 gemm: %s", cudaGetErrorString(e));
    return EXA_ERR_CUDA;
  }
  return EXA_OK;
}

extern "C" void exa_debug_umma_wait_polls(long long polls) { exa_umma_set_wait_polls(polls); }

extern "C" int exa_dgemm_tune(int M, int N, int K, int batch, void* stream, int* tile) {
  EXA_TRY(exa_gemm_tune(M, N, K, batch, (cudaStream_t)stream));
  if (tile) *tile = exa_gemm_tile_of(M, N, K);
  return EXA_OK;
}

extern "C" int exa_inverse_autotune(int n, int fp64, int batch, void* stream, int* variant) {
  EXA_TRY(exa_inverse_tune(n, batch, fp64, (cudaStream_t)stream));
  if (variant) *variant = exa_inverse_variant_of(n, fp64);
  return EXA_OK;
}

extern "C" int exa_sinverse_batched(float* A, int n, long long stride, int batch, int* info_dev, void* stream) {
  if (exa_inverse_tc32_pk(n) == 0 || batch <= 0) return exa_inverse(A, n, stride, batch, info_dev, (cudaStream_t)stream);
  if (n > exa_inverse_max_n()) {
    exa_set_error("dense inverse of order %d exceeds %d", n, exa_inverse_max_n());
    return EXA_ERR_UNSUPPORTED;
  }
  // the blocks of every level and the packed operands per matrix, freed after the stream drains
  cudaStream_t st = (cudaStream_t)stream;
  const size_t nblk = ((size_t)exa_inverse_tc32_ws(n) * batch + 63) / 64 * 64;  // packed operands start 256-byte aligned
  float* ws = nullptr;
  EXA_CUDA(cudaMallocAsync((void**)&ws, sizeof(float) * (nblk + (size_t)exa_inverse_tc32_pk(n) * batch), st));
  const int s = exa_inverse_tc32(A, n, stride, batch, ws, ws + nblk, info_dev, info_dev, st);
  cudaFreeAsync(ws, st);
  return s;
}

extern "C" int exa_dinverse_batched(double* A, int n, long long stride, int batch, int* info_dev, void* stream) {
  if (!exa_inverse_needs_ws(n) || batch <= 0) return exa_inverse(A, n, stride, batch, info_dev, (cudaStream_t)stream);
  if (n > exa_inverse_max_n()) {
    exa_set_error("dense inverse of order %d exceeds %d", n, exa_inverse_max_n());
    return EXA_ERR_UNSUPPORTED;
  }
  // blocked orders: a temporary workspace of n^2 per matrix, freed after the stream drains
  cudaStream_t st = (cudaStream_t)stream;
  double* ws = nullptr;
  EXA_CUDA(cudaMallocAsync((void**)&ws, sizeof(double) * (size_t)n * n * batch, st));
  const int s = exa_inverse_ws(A, n, stride, batch, ws, info_dev, st);
  cudaFreeAsync(ws, st);
  return s;
}

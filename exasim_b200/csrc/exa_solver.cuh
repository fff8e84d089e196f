// Host-side solver context: inputs parsed from Exasim's app/master/mesh/sol blobs,
// device-resident mesh, master, solution and condensed system, and the workspace of
// the assembly and Krylov loops.  The drivers mirror Exasim's call structure:
//   hdgAssembleLinearSystem / hdgAssembleResidual (discretization.cpp:483-592),
//   GMRES (gmres.cpp:361-597), NewtonSolver (solution.cpp:125-243), DIRK stepping
//   (exasim.hpp:413-482).
#pragma once
#include <string>
#include <vector>

#include "exa_kernels.cuh"
#include "exa_conn.h"
#include "exa_umma.cuh"

// Device time by solver phase (exa_profile / exa_profile_read in the C ABI): CUDA event
// pairs recorded on the context stream around each phase, summed when read.
enum ExaPhase {
  EXA_PH_VOLUME = 0, EXA_PH_FACE, EXA_PH_QELIM, EXA_PH_INVERSE, EXA_PH_SCHUR, EXA_PH_PRECOND_BUILD,
  EXA_PH_MATVEC, EXA_PH_PRECOND_APPLY, EXA_PH_ORTHO, EXA_PH_GETQ, EXA_PH_RESIDUAL, EXA_PH_PACK, EXA_PH_UPDATE,
  EXA_NPHASE
};

struct ExaProf {
  bool on = false;
  std::vector<cudaEvent_t> ev;  // two per slot: start, end
  std::vector<int> phase;       // phase of each slot
  int used = 0;
  double ms[EXA_NPHASE] = {};
  long long count[EXA_NPHASE] = {};
  double flops[EXA_NPHASE] = {};
};

struct ExaCtx {
  ExaDims P{};
  int device = 0;
  cudaStream_t st = nullptr;
  // second stream of the assembly: the element inverse runs there beside the q-elimination
  // products that do not need it (ev_q: D ready; ev_inv: D^-1 ready)
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_q = nullptr, ev_inv = nullptr;
  // app flags (app.bin flag/problem/solversparam, setstructs.cpp:45-322)
  int tdep = 0, wave = 0, preconditioner = 0, ortho = 0, tdfunc = 1, sourcefunc = 1, modelnumber = 0;
  int newton_maxit = 20, gmres_maxit = 200, restart = 25, torder = 1, nstage = 1, ppdegree = 0, RBdim = 0;
  double newton_tol = 1e-6, gmres_tol = 1e-3, time0 = 0.0;
  std::vector<double> dt;
  int elemtype = 0, porder = 0;
  // host copies needed by the host-side initial condition
  std::vector<double> h_xdg, h_uinf, h_param;
  // device data
  double *shapegt = nullptr, *shapegw = nullptr, *shapfgt = nullptr, *shapfgw = nullptr;
  int *perm = nullptr, *elemcon = nullptr, *f2e = nullptr, *bf = nullptr;
  double *xdg = nullptr, *elemg = nullptr, *faceg = nullptr, *uinf = nullptr, *param = nullptr, *tau = nullptr;
  double *udg = nullptr, *uh = nullptr, *sdg = nullptr;
  double *MC = nullptr, *ME = nullptr;
  double* Minv = nullptr;  // inverse element mass matrices [npe, npe, ne] (q recovery by quadrature)
  // q recovery workspace: Gauss-point u, its geometric products and C_d u for all elements
  double *wq_ug = nullptr, *wq_v = nullptr, *wq_w = nullptr;
  double *H = nullptr, *F = nullptr, *Ru = nullptr, *Rh = nullptr, *b = nullptr, *Pc = nullptr;
  // assembly workspace for a chunk of `neb` elements
  int neb = 0;
  double *wD = nullptr, *wB = nullptr, *wF = nullptr, *wK = nullptr, *wG = nullptr, *wRg = nullptr, *wRu = nullptr;
  // per chunk: udg and sdg at the Gauss points and the Ru integrand (the volume kernel's GEMMs)
  double *wUG = nullptr, *wSG = nullptr, *wRG = nullptr;
  // the volume blocks' left factors T = -(shapegw . rgJ) of up to wT_elems elements, for the
  // FP64 volume products on the DMMA tensor cores
  double* wT = nullptr;
  int wT_elems = 0;
  double* wInv = nullptr;  // blocked-inverse workspace (n^2 per element) when n exceeds the register kernel
  // Krylov / Newton workspace
  double *V = nullptr, *x = nullptr, *r = nullptr, *w = nullptr, *we = nullptr, *du = nullptr;
  double *part_a = nullptr, *part_b = nullptr, *part_m = nullptr, *hess = nullptr, *gs = nullptr, *gcs = nullptr,
         *gsn = nullptr, *scal = nullptr, *udgprev = nullptr, *utmp = nullptr;
  int* d_flag = nullptr;
  double* pinned = nullptr;  // small host staging buffer
  // reduced-basis initial guess of GMRES (RBdim > 0): the last RBdim Newton updates W, their
  // images U under the condensed operator, a ring position, and the dot products of a guess
  double *rbW = nullptr, *rbU = nullptr, *rbD = nullptr;
  int rb_cur = 0, rb_removed = 0;
  // polynomial preconditioner (ppdegree > 1, getpoly.cpp / gmres.cpp:91-130): the start vector
  // of its Arnoldi process, two work vectors, and the Leja-ordered Ritz values (real and
  // imaginary parts) of the last GMRES call
  double *randvect = nullptr, *poly_q = nullptr, *poly_p = nullptr;
  std::vector<double> poly_sr, poly_si;
  // GMRES: each Arnoldi step index i of the restart cycle (and each precision) runs as one
  // captured CUDA graph from its second use on; none while phase profiling records events
  std::vector<cudaGraphExec_t> arnoldi_graph[2];
  std::vector<long long> arnoldi_launches[2];
  std::vector<unsigned char> arnoldi_seen[2];
  cudaEvent_t step_ev[2] = {nullptr, nullptr};
  int use_graphs = 1;
  // state
  double time = 0.0, dtfactor = 0.0;
  int nf_total = 0;
  std::vector<void*> allocs;
  long long alloc_bytes = 0;  // device bytes held by the context
  // statistics of the last solve
  int last_gmres_iters = 0, last_newton_iters = 0, total_gmres_iters = 0;
  double last_gmres_relerr = 0.0;
  bool last_gmres_converged = true;  // the last GMRES call reached its tolerance
  long long kernel_launches = 0;
  ExaProf prof;
  // residual norms of the last Newton / refinement solve: at its start and at its end
  double last_norm0 = 0.0, last_norm = 0.0;

  // mixed-precision form (exa_set_precision): the element elimination, the condensed
  // blocks and the preconditioner in FP32 (TF32 tensor-core products, FP32 accumulation);
  // the residual, the Newton update and GMRES stay FP64 and iterate the FP32 solve to the
  // FP64 residual tolerance.
  int precision = 0;              // 0 plain FP64, 1 mixed
  // FP64 H, F (D^-1 F) and preconditioner blocks held for all elements (the plain form); the
  // mixed form holds neither F nor the FP64 preconditioner, and H for one element chunk only
  bool fp64_full = true;
  double mixed_inner_tol = 1e-4;  // GMRES tolerance of each refinement step
  double mixed_rtol = 0.0;        // target residual ratio of a mixed solve (0: GMRES tolerance)
  int mixed_maxit = 30;           // refinement steps per mixed solve
  float *H32 = nullptr, *F32 = nullptr, *K32 = nullptr;    // condensed block, D^-1 F, K
  float *Dinv32 = nullptr, *Pc32 = nullptr;
  // blocks and packed operands of the recursive tensor-core inverse, per element chunk
  float *wInv32 = nullptr, *wInvPk = nullptr;
  int* d_uflag = nullptr;         // tensor-core kernel wait flag
  // operands of the 3xTF32 products, packed in the tensor-core layout (hi and lo parts):
  // Minv C, Minv E as B operands (all elements); per element chunk: B and G (A operands of
  // the q elimination), D^-1 (A), F (B of D^-1 F), K (A) and D^-1 F (B of K D^-1 F)
  UPacked MCp{}, MEp{}, wBp{}, wGp{}, Dinvp{}, wFp{}, Kp{}, DinvFp{};
  UPacked Sp{};  // shapegt[:, :, 0] as the B operand of the tensor-core volume kernel
  float* shapegw32 = nullptr;  // shapegw in FP32, the weights of that kernel's T tiles
  // block ILU(0) on Cartesian sub-domains (preconditioner 2): blocks in Pc / Pc32
  std::vector<int> cartgridpart;
  ExaBiluDev bilu;

  // batched GMRES (exa_batch.cu): when set, GMRES calls of this context run through the batcher
  struct ExaBatcher* batcher = nullptr;

  // LDG discretisation (app.bin problem[0] = 0) and its pseudo-transient solver: the
  // residual of the element states, its Jacobian by residual differences (flag[4]: one- or
  // two-sided, solversparam[2]: the step), the identity preconditioner (flag[7] = 0)
  int scheme = 1;  // 0 LDG, 1 HDG
  int matvec_order = 1, ntau = 1, ldg_prec_matrix = 0;  // flag[7]: 0 identity, else the element mass inverse
  double matvec_eps = 1e-3;
  double* shapfnt = nullptr;  // face nodal basis and its derivatives at the face nodes [npf, npf, nd]
  int* ldg_fcon = nullptr;    // [2, npf, nf]: e npe + node of face node i on each side (side 1 twice on the boundary)
  // R(u), a perturbed state, its residual, the face residuals [npf, ncu, nf], R at u - eps v
  double *ldg_R = nullptr, *ldg_w = nullptr, *ldg_Rw = nullptr, *ldg_Rh = nullptr, *ldg_Rm = nullptr;
  int ldg_has_boundary = 0;
  // interior faces are faces [0, nf0) and boundary faces the rest (the pointwise interior-face
  // kernel relies on it)
  int ldg_split = 0;
  // set by the PTC solver: GMRES starts from the x it finds (the reduced-basis guess it has
  // checked) instead of zero, and computes no guess of its own
  int gmres_x_preset = 0;

  long long ndofuhat() const { return (long long)P.ncu * P.npf * P.nf; }
  // unknowns of the linear systems GMRES solves: the trace (HDG) or the element states (LDG)
  long long sysN() const { return scheme == 0 ? (long long)P.npe * P.ncu * P.ne : ndofuhat(); }
};

// setup and teardown (exa_api.cu)
int exa_ctx_init(ExaCtx& c, const double* app, long long napp, const double* master, long long nmaster,
                 const double* mesh, long long nmesh, const double* sol, long long nsol, int device);
void exa_ctx_free(ExaCtx& c);
int exa_ctx_reset(ExaCtx& c, const double* app, long long napp, const double* sol, long long nsol);
unsigned long long exa_ctx_key(const double* app, long long napp, const double* master, long long nmaster,
                               const double* mesh, long long nmesh, const double* sol, long long nsol);
long long exa_ctx_estimate_bytes(const double* app, long long napp, const double* master, long long nmaster,
                                 const double* mesh, long long nmesh, int precision);

// model-specific steps (instantiated per model)
int exa_model_assemble(ExaCtx& c, bool jacobian);
int exa_model_init_udg(ExaCtx& c, double* host_udg);
// LDG residual (residual.cpp:589-617) of the element states u [npe, ncu, ne] into Ru
int exa_model_ldg_residual(ExaCtx& c, const double* u, double* Ru);
// whether the model carries the LDG boundary functions (Ubou, Fbou)
bool exa_model_has_ldg_boundary();

// model-independent drivers (exa_drivers.cu)
int exa_drv_assemble(ExaCtx& c);
int exa_drv_residual(ExaCtx& c, double* norm);
int exa_drv_matvec(ExaCtx& c, const double* v, double* w);
int exa_drv_precond(ExaCtx& c, const double* v, double* w);
int exa_drv_build_precond(ExaCtx& c);
int exa_drv_gmres(ExaCtx& c, int* iters, double* relerr);
int exa_drv_getq(ExaCtx& c);
int exa_drv_newton(ExaCtx& c, int* iters, double* norm);
int exa_drv_dirk(ExaCtx& c, int nsteps, int* newton_iters_out, int max_out);
int exa_drv_dirk_stage(ExaCtx& c, int istep, int stage, int* its_out, double* norm_out);
int exa_drv_norm(ExaCtx& c, const double* x, long long n, double* out);
// x += V y with y from the back-solve of the Hessenberg system of steps 0..i (gmres.cpp:132-137)
int exa_drv_gmres_update(ExaCtx& c, int i);
// mixed-precision form (exa_drivers.cu, exa_api.cu)
int exa_ctx_set_precision(ExaCtx& c, int mode);
int exa_drv_newton_mixed(ExaCtx& c, int* iters, double* norm);
int exa_drv_condense_mixed(ExaCtx& c);

// phase profile (exa_drivers.cu)
int exa_prof_enable(ExaCtx& c, int on);
int exa_prof_flush(ExaCtx& c);
void exa_prof_free(ExaCtx& c);
inline void exa_prof_flops(ExaCtx& c, int phase, double f) {
  if (c.prof.on) c.prof.flops[phase] += f;
}
// Records the start event on construction and the end event on destruction.
struct ExaProfScope {
  ExaCtx& c;
  int slot = -1;
  ExaProfScope(ExaCtx& ctx, int phase);
  ~ExaProfScope();
};

/* C ABI of the B200 HDG solver (libexasim_b200_<model>.so).
 *
 * One shared library per PDE model, as Exasim builds one libpdemodel<backend>.so per
 * model (backend/Model/libpdemodel.hpp).  A context owns all device memory: mesh,
 * master element, solution (udg, uhat) and the condensed HDG system.  Pointers named
 * *_dev are CUDA device pointers; every other pointer is host memory owned by the caller.
 * Every function returns 0 on success or an ExaStatus code (1 bad argument,
 * 2 unsupported input, 3 CUDA error, 4 singular block, 5 mesh error, 6 not converged,
 * 7 NaN residual, 8 out of device memory, 9 wait timed out); exa_last_error() describes the
 * calling thread's last failure.
 * The reference prints and exits instead (backend/Common/common.h:527-555).
 * One host thread per context; calls are synchronous unless noted.
 *
 * Array layouts are Exasim's (column-major):  udg [npe, nc, ne], uhat [ncu, npf, nf].
 */
#ifndef EXASIM_B200_H
#define EXASIM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct exa_ctx exa_ctx;

/* Message of the calling host thread's last failed call. */
const char* exa_last_error(void);

/* Build a context from the four input files Exasim's preprocessor writes
 * (datain/app.bin, master.bin, mesh.bin, sol.bin), passed as their float64 words.
 * Replaces CDiscretization's constructor: readInput (backend/Discretization/readbinaryfiles.cpp:625),
 * buildConn for raw element lists (connectivity.cpp:1212), compGeometry (geometry.cpp:87-222),
 * qEquation (qequation.cpp:365) and the HDG allocations (discretization.cpp:245-428).
 * app.bin's problem[0] selects the discretization: 1 HDG, 0 LDG (setstructs.cpp:145).  An LDG
 * context solves for the element states u (udg without q: models with ncq = 0) with the
 * pseudo-transient solver: exa_residual, exa_matvec, exa_precond, exa_gmres, exa_newton,
 * exa_dirk and exa_solve run the LDG forms named at each of them, on vectors of length
 * npe*ncu*ne, with the reduced-basis guess of problem[16] as the PTC solver has it and the
 * polynomial preconditioner of problem[27].  It refuses (EXA_ERR_UNSUPPORTED) models with q
 * and the mixed-precision form, and boundary faces without the model's KokkosUbou/KokkosFbou. */
int exa_create(const double* app, long long napp, const double* master, long long nmaster,
               const double* mesh, long long nmesh, const double* sol, long long nsol, int device,
               exa_ctx** out);
void exa_destroy(exa_ctx* ctx);

/* out[16] = {ne, nf, nf0, npe, npf, nfe, nc, ncu, nd, n=npe*ncu, m=ncu*npf*nfe,
 *            ndofuhat, nge, ngf, element chunk, preconditioner} */
int exa_sizes(exa_ctx* ctx, long long* out);

/* Host copies of named device arrays: "udg", "uh", "H", "F" (D^-1 F after assembly),
 * "Ru", "Rh", "b", "x", "sdg", "P" (preconditioner), "MinvC", "MinvE", "elemg", "faceg", and with
 * a polynomial preconditioner "randvect" (the start vector of its Arnoldi process, length ndofuhat;
 * npe*ncu*ne on an LDG context).
 * n must equal the array length.  MinvC and MinvE hold, per element, Minv*C_d and Minv*E_d
 * with the dimension index next to the row index: [npe, nd, npe] and [npe, nd, npf*nfe].
 * "K", "B" and "Dinv" (the FP64 K and B blocks, and D^-1 after an FP64 assembly) exist when the whole
 * mesh is one assembly chunk (exa_sizes element chunk == ne).
 * After exa_set_precision(ctx, 1, ...) the FP32 arrays "H32", "F32" (D^-1 F), "K32" and
 * "Dinv32" are available too: exa_get_field/exa_set_field convert them to and from double,
 * and exa_field_ptr returns their device address (pointing at floats). */
int exa_get_field(exa_ctx* ctx, const char* name, double* host, long long n);
int exa_set_field(exa_ctx* ctx, const char* name, const double* host, long long n);
/* Device pointer and length of a named array (zero-copy access, e.g. from torch). */
int exa_field_ptr(exa_ctx* ctx, const char* name, double** dev, long long* n);
/* f2e [4, nf] and elemcon [npf*nfe, ne] (0-based), either may be NULL. */
int exa_get_connectivity(exa_ctx* ctx, int* f2e, int* elemcon);

/* Current time and DIRK factor d_jj/dt used by time-dependent assembly (UpdateSourceDIRK,
 * backend/Solution/updatesource.cpp:32-50). */
int exa_set_time(exa_ctx* ctx, double time, double dtfactor);
/* The time at the start of the next DIRK step (exa_dirk_stage step 0 starts from it; each
 * completed step adds its dt).  A restart at step R sets it to R dt[0], as the reference does
 * with its restart argument or timestepOffset (backend/Main/exasim.hpp:387-393, 425). */
int exa_set_step_time(exa_ctx* ctx, double time0);

/* hdgAssembleLinearSystem (backend/Discretization/discretization.cpp:483-573): element
 * residuals and Jacobians (uequation.cpp:45-557), static condensation (:559-775),
 * RHS b (matvec.cpp:103) and the preconditioner (matvec.cpp:119-217). */
int exa_assemble(exa_ctx* ctx);
/* hdgAssembleResidual (discretization.cpp:576-592); *norm = |b| + |Ru| (solution.cpp:148-157).
 * LDG: R(u) of the current udg into field "Ru" (Residual, residual.cpp:589-617: element and
 * face integrals, uresidual.cpp:45-334), *norm = |R|. */
int exa_residual(exa_ctx* ctx, double* norm);
/* w = A v, hdgMatVec (matvec.cpp:240-389); device vectors of length ndofuhat.
 * LDG: w = J(u) v by residual differences around the udg and R of the last exa_residual
 * (MatVec, matvec.cpp:41-100; flag[4] one- or two-sided, solversparam[2] the step). */
int exa_matvec(exa_ctx* ctx, const double* v_dev, double* w_dev);
/* w = P v, ApplyPreconditioner (Preconditioning/preconditioner.cpp:273-295); v != w.
 * LDG: the identity (precMatrixType 0) or the element mass inverse per field
 * (preconditioner.cpp:130-137, applymatrix.cpp:66-98). */
int exa_precond(exa_ctx* ctx, const double* v_dev, double* w_dev);
/* Solve A x = b by restarted GMRES (Solver/gmres.cpp:361-597); x is field "x".  When it stops at
 * the iteration cap above its tolerance it returns EXA_ERR_NOTCONV (6) with *iters and *relerr
 * filled in; the reference prints a warning with that error instead (gmres.cpp:586-594).
 * Inside exa_newton an unconverged GMRES call continues the Newton step, as in the reference. */
int exa_gmres(exa_ctx* ctx, int* iters, double* relerr);
/* q from u and uhat, hdgGetQ (qequation.cpp:372-484). */
int exa_getq(exa_ctx* ctx);
/* Damped Newton on the HDG residual, NewtonSolver (Solution/solution.cpp:125-243).
 * LDG: PTCsolver (Solver/ptcsolver.cpp:255-330): GMRES on J(u) x = -R(u), u += x, until
 * |R(u)| < NewtonTol; *iters counts the steps, a norm above 1e6 returns EXA_ERR_NOTCONV
 * (NaN: EXA_ERR_NAN) where the reference writes the state and exits. */
int exa_newton(exa_ctx* ctx, int* iters, double* norm);
/* nsteps DIRK steps around Newton (Main/exasim.hpp:413-482); newton_iters[0..max_out) receives
 * the Newton count of each stage. */
int exa_dirk(exa_ctx* ctx, int nsteps, int* newton_iters, int max_out);
/* One DIRK stage of step istep (0-based, < number of dt entries): source update from the
 * stage history (updatesource.cpp:32-80), Newton solve, stage accumulation
 * (updatesolution.cpp:118-140); the last stage of a step advances the time. */
int exa_dirk_stage(exa_ctx* ctx, int istep, int stage, int* iters, double* norm);
/* The CUDA stream the context launches on (cudaStream_t), for events and interop. */
int exa_stream(exa_ctx* ctx, void** stream);
/* One Newton solve from host buffers: copies udg/uhat in (NULL keeps the current state),
 * solves, copies them out (NULL skips).  The end-to-end form of exa_newton. */
int exa_solve(exa_ctx* ctx, const double* udg_in, const double* uh_in, double* udg_out,
              double* uh_out, int* iters, double* norm);
/* Face connectivity of a raw element list on the host, buildConn / connectivity()
 * (backend/Discretization/connectivity.cpp:426-497, 1212-1385): t [nve, ne] 0-based vertices,
 * bf [nfe, ne] boundary codes, perm [npf, nfe], xpf [npf, dim-1]; f2e (4*nfe*ne ints) and
 * elemcon (npf*nfe*ne ints) receive the result.  Returns nf (>= 0) or a negated status. */
int exa_connectivity_host(const int* t, const int* bf, const int* perm, const double* xpf, int dim,
                          int elemtype, int ne, int npe, int npf, int* f2e, int* elemcon, int* nf0);
/* Precision form of the Newton solves (exa_newton, exa_dirk, exa_dirk_stage, exa_solve).
 * mode 0: plain FP64 (the reference's arithmetic).  mode 1: mixed precision, with no
 * counterpart in the reference: the element elimination (q elimination, D^-1, Schur
 * products) runs on the TF32 tensor cores with FP32 accumulation, and the condensed blocks
 * and the preconditioner are kept in FP32.  The residual, the Newton update and GMRES stay
 * FP64: each step solves the FP32 system to inner_tol and recomputes the FP64 residual,
 * until the FP64 residual norm has dropped by rtol (0: by the GMRES tolerance of app.bin).
 * The first switch to mode 1 allocates the FP32 arrays.  Mode 1 frees the FP64 "H", "F" and
 * "P" arrays, which it does not read (their fields are unavailable until a switch back to
 * mode 0 reallocates them; the next assembly fills them). */
int exa_set_precision(exa_ctx* ctx, int mode, double inner_tol, double rtol);
/* Residual norm |b| + |Ru| at the start and at the end of the last Newton solve. */
int exa_last_residual(exa_ctx* ctx, double* initial, double* final_norm);
/* Device time by solver phase, from CUDA events recorded on the context stream around each
 * phase (the reference prints its own phase timers instead, e.g. Solver/ptcsolver.cpp:361).
 * exa_profile(ctx, 1) resets the totals and starts recording; exa_profile(ctx, 0) stops.
 * Phases: 0 volume assembly, 1 face assembly, 2 q-elimination GEMMs, 3 element inverse,
 * 4 Schur GEMMs, 5 preconditioner build, 6 matvec, 7 preconditioner apply,
 * 8 Gram-Schmidt + Givens, 9 q recovery, 10 residual-only assembly, 11 packing of tensor-core
 * operands (mixed-precision form), 12 Newton update of uhat and u (and, in the mixed form, the
 * refinement's condensed right-hand side).
 * exa_profile_read fills ms, count (timed regions) and flops (algorithmic FLOPs of the GEMM
 * phases 2 and 4, 0 elsewhere) for the first nphase (<= 13) phases; any may be NULL.  It
 * synchronises the context stream. */
int exa_profile(exa_ctx* ctx, int enable);
int exa_profile_read(exa_ctx* ctx, int nphase, double* ms, long long* count, double* flops);
/* Sub-domain face ordering of the block ILU(0) preconditioner (preconditioner 2) on the host:
 * the Cartesian partition of cartgridpart ([2, Nx, Ny, Mx, My, opt] or [3, Nx, Ny, Nz, Mx, My,
 * Mz, opt], gridpartition2d/3d, backend/Common/cpuimpl.h:1332-1496) and the face ordering of a
 * sub-domain (crs_faceordering, cpuimpl.h:1266-1330) for the face connectivity f2e [4, nf]:
 * row_ptr [nfse + 1] and col_ind (CRS, diagonal first) and face [nse, nfse] (column-major).
 * Returns nfse, or a negated status. */
int exa_bilu0_ordering(const int* cartgridpart, int ncgp, const int* f2e, int nf, int nfe, int ne, int* row_ptr,
                       int cap_row_ptr, int* col_ind, int cap_col_ind, int* face, int cap_face, int* nse);
/* out[4] = {last GMRES iterations, last Newton iterations, GMRES iterations of the last solve, 0} */
int exa_stats(exa_ctx* ctx, long long* out);
int exa_synchronize(exa_ctx* ctx);
/* Batched FP64 building blocks on device pointers, enqueued on `stream` (cudaStream_t, may
 * be NULL): C_b = alpha A_b B_b + beta C_b (column-major, batch strides sA, sB, sC) as used for
 * Exasim's PGEMNMStridedBached (backend/Common/pblas.h:695); and the in-place explicit
 * inverse of `batch` n x n blocks `stride` doubles apart (pblas.h:163 Inverse), n <= 320
 * (above 160 by 2 x 2 blocks with a temporary stream-ordered workspace of n^2 doubles per
 * block), *info_dev set non-zero on a zero pivot. */
int exa_dgemm_batched(int M, int N, int K, double alpha, const double* A, long long lda, long long sA,
                      const double* B, long long ldb, long long sB, double beta, double* C, long long ldc,
                      long long sC, int batch, void* stream);
int exa_dinverse_batched(double* A, int n, long long stride, int batch, int* info_dev, void* stream);
/* FP32 counterpart of exa_dinverse_batched, the mixed-precision form's element inverse
 * (an FP32 restatement of pblas.h:163 Inverse; the reference has FP64 only).  Above order 160
 * the 2 x 2 block products run on the tcgen05 3xTF32 GEMM, with a temporary stream-ordered
 * workspace.  *info_dev is set to 1 on a zero pivot and to 2 if a tensor-core wait ran out. */
int exa_sinverse_batched(float* A, int n, long long stride, int batch, int* info_dev, void* stream);
/* No counterpart in the reference.  Times the candidate CTA tiles of exa_dgemm_batched for
 * one M x N x K shape on `batch` (at most 512) scratch blocks, allocated stream-ordered on
 * `stream`, and keeps the fastest for this device and shape; *tile (may be NULL) gets its
 * index.  exa_create tunes the shapes of its element products this way.  Every tile sums
 * each entry over k in the same order, so the choice changes the time, not the result.
 * Synchronizes `stream`; not for use inside stream capture. */
int exa_dgemm_tune(int M, int N, int K, int batch, void* stream, int* tile);
/* The same autotuner for the batched element inverse of order 32 < n <= 128 (FP64 when fp64 is
 * nonzero, else FP32): times the column-by-warp Gauss-Jordan shapes on min(batch, 4096)
 * scratch blocks (once per process, device, order and type; later calls return at once) and
 * keeps the fastest; *variant (optional) receives the shape used for order n (0-3; -1 outside
 * 33..128).  Every shape gives the same bits.  Synchronizes `stream`; not inside stream capture.
 * exa_create and exa_set_precision tune the orders they invert. */
int exa_inverse_autotune(int n, int fp64, int batch, void* stream, int* variant);
/* C_b = alpha A_b B_b + beta C_b with FP32 C, the products split as hi*hi + hi*lo + lo*hi over
 * TF32 parts (3xTF32, about FP32 accuracy) on the tcgen05 tensor cores with FP32
 * accumulation: the product the mixed-precision form uses.  A and B are FP64 or FP32,
 * column-major.  N <= 1024 (above 256 in column chunks of 256, one launch each).  The call
 * packs A and B into temporary device buffers (allocated
 * and freed inside) and synchronises the stream.  *flag_dev as for exa_gemm_tf32_batched. */
int exa_gemm_3xtf32_batched(int M, int N, int K, double alpha, const void* A, int a_f64, long long lda, long long sA,
                            const void* B, int b_f64, long long ldb, long long sB, double beta, float* C, long long ldc,
                            long long sC, int batch, int* flag_dev, void* stream);
/* C_b = alpha A_b B_b + beta C_b on the TF32 tensor cores (tcgen05) with FP32 accumulation,
 * the product the mixed-precision form uses for PGEMNMStridedBached (pblas.h:695).  Each of
 * A, B and C is FP32 or FP64 (a_f64, b_f64, c_f64); the instantiated combinations are all
 * FP32, and FP64 A with FP32 B and C.  N <= 256.  *flag_dev is set to 2 if a wait inside the
 * kernel ran out (the result is then not valid). */
int exa_gemm_tf32_batched(int M, int N, int K, double alpha, const void* A, int a_f64, long long lda, long long sA,
                          const void* B, int b_f64, long long ldb, long long sB, double beta, void* C, int c_f64,
                          long long ldc, long long sC, int batch, int* flag_dev, void* stream);
/* No counterpart in the reference: a test hook for the timeout path of the 3xTF32 tensor-core
 * GEMM (exa_gemm_3xtf32_batched and the mixed form's element products).  Sets the polls of each
 * main-loop mbarrier wait in that kernel, process-wide (negative restores the normal 2^22).  With
 * 0 every such wait gives up at once: the kernel waits (at the normal limit) for the bulk copies
 * and MMAs it already started, frees its tensor memory, sets its flag to 2 and returns, and the
 * caller sees the flag (status 3 from the mixed-form solvers).  Not for use while another thread
 * runs the mixed form. */
void exa_debug_umma_wait_polls(long long polls);
/* Host part of the polynomial preconditioner (ppdegree > 1 in app.bin): from the Hessenberg matrix
 * H [(m+1) x m, column-major] of m Arnoldi steps of the preconditioned operator, the harmonic Ritz
 * values in Leja order, sr[m] + i si[m] (getPoly and its post-processing in GMRES,
 * backend/Solver/getpoly.cpp:111-173, 226-247, gmres.cpp:385-398; eigenvalues by the Francis QR
 * iteration where the reference calls LAPACK dgeev).  GMRES applies the polynomial with these
 * roots after the preconditioner (ApplyPoly, gmres.cpp:319-357).  2 <= m <= 64; no GPU needed. */
int exa_poly_ritz(const double* H, int m, double* sr, double* si);
/* Number of CUDA kernels this library has launched since it was loaded (all contexts). */
long long exa_launch_count(void);
/* Euclidean norms of `ncols` device columns of length n, column j at X + j*ldx, written to
 * out_dev[0..ncols) on `stream` (cudaStream_t, may be NULL) without allocating anything.
 * No counterpart in the reference: it exists for callers that cannot allocate device memory
 * at the call (a host framework's memory pool owns the free memory, or the step loop cannot
 * take cudaFree's device-wide synchronisation).  Its partial sums live in one fixed device
 * array per device (64 columns x 296 blocks of doubles, 151,552 bytes); ncols > 64 returns
 * EXA_ERR_ARG (1).  The first call on each device, with that device current, looks up the
 * array's address (which can load this library's device code), so make it before any stream
 * capture starts.  That address is kept for the life of the process and belongs to the device's
 * primary context: after cudaDeviceReset, or from another driver context on the same device,
 * calls are not valid.  Nothing needs zeroing beforehand.  Calls whose kernels can overlap (other
 * streams with no ordering, several host threads) race on the shared array: order them. */
int exa_dnrm2_cols_fixed(const double* X, long long n, long long ldx, int ncols, double* out_dev, void* stream);

/* ---- Serving: continuous batching of independent solves of this library's model ----
 * No counterpart in the reference, which runs one problem per process.  A server owns
 * `slots` host threads on one device.  Each submitted request (the four datain blobs, copied
 * at submit) waits in arrival order until a slot is free and its context fits in
 * hbm_budget_bytes (estimated from the blobs before it exists, its actual size after); it
 * then runs on its own context and CUDA stream, so admitted solves overlap on the device.
 * Steady problems run Newton (exa_newton); time-dependent ones every DIRK step of their app
 * (exa_dirk).  With reuse_contexts, a finished request's context stays resident, keyed by
 * master, mesh, sol and app without the physical parameters and tau; a later request with
 * the same key reuses it after a reset of parameters and initial state, and contexts held
 * for reuse are evicted least recently used first when memory is needed.  A solve's result
 * does not depend on what else runs: every reduction is in a fixed order.
 * precision, inner_tol and rtol are those of exa_set_precision.  Contexts use stream-ordered
 * allocation, so creating and freeing one does not synchronise the device. */
typedef struct exa_server exa_server;
int exa_server_create(int device, long long hbm_budget_bytes, int slots, int reuse_contexts, exa_server** out);
int exa_server_submit(exa_server* s, const double* app, long long napp, const double* master, long long nmaster,
                      const double* mesh, long long nmesh, const double* sol, long long nsol, int precision,
                      double inner_tol, double rtol, long long* id);
/* Blocks until request `id` has finished (timeout_s < 0: no limit; else EXA_ERR_TIMEOUT) and
 * gives its result sizes (udg npe*nc*ne, uhat ndofuhat); returns the solve's status. */
int exa_server_wait(exa_server* s, long long id, double timeout_s, long long* nudg, long long* nuh);
/* Copies a finished request's udg and uhat (either may be NULL) and info[8] = {queued ms,
 * run ms (set-up or reset, solve, read-back), latency ms (submit to finish), Newton steps,
 * GMRES iterations, first and last residual norm, 1 if its context was reused}, then
 * forgets the request. */
int exa_server_fetch(exa_server* s, long long id, double* udg, long long nudg, double* uh, long long nuh,
                     double* info);
/* out[10] = {queued, running, done, failed, device bytes held, peak bytes held, contexts
 * created, contexts reused, contexts kept idle, contexts evicted} */
int exa_server_stats(exa_server* s, long long* out);
/* Finishes the running solves, drops queued requests and frees every context. */
void exa_server_destroy(exa_server* s);
/* No counterpart in the reference.  Batched Krylov steps across the server's solves: with
 * capacity > 0 (up to 1024 job slots), every GMRES call of a running solve that uses block
 * Jacobi, MGS and no reduced basis (condensed blocks up to 64 x 64) joins one batch, whose
 * Arnoldi steps run as one set of launches (a captured CUDA graph per highest step index) for
 * all of its jobs; calls join and leave at any step.  Each job's reductions have their own
 * fixed order, so a result does not depend on the other jobs.  Set before the first submit;
 * 0 turns batching off. */
int exa_server_set_batching(exa_server* s, int capacity);
/* out[4] = {batched steps, kernel launches of those steps, GMRES calls served, elements per warp
 * of the batched matvec chosen by its autotuner} */
int exa_server_batch_stats(exa_server* s, long long* out);

#ifdef __cplusplus
}
#endif
#endif

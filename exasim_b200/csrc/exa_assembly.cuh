// HDG element assembly kernels, templated on the pointwise model (device functions
// produced by exasim_b200/modelc.py from Exasim's generated sources).  Included once by
// each model's translation unit.
//
// Reference steps (backend/Discretization/uequation.cpp):
//   volume   :45-203   uq at quadrature points, Source/Flux with Jacobians, the DIRK
//                      term, ApplyXxJac, then Ru (Gauss2Node with shapegw) and D, B
//                      (Gauss2Node with shapegw x shapegt, negated)
//   faces    :206-557  (uhat, q) at face points, numerical flux f(uhat,q).n + tau(u-uhat)
//                      for Ru, D, B, F on every face; boundary faces replace the flux by
//                      Fbou for the trace rows Rh, K, G, H
//   residual :790-1088 the same without Jacobians (Flux/Source/Fbouonly)
// One block per element; all of an element's faces are handled by the same block in
// sequence, so face contributions accumulate into D, B and Ru without atomics.
#pragma once
#include <algorithm>

#include "exa_kernels.cuh"
#include "exa_tc.cuh"
#include "exa_umma.cuh"

struct AsmArgs {
  ExaDims P;
  const double *shapegt, *shapegw, *shapfgt, *shapfgw;
  const int *perm, *elemcon, *bf;
  const double *elemg, *faceg;
  const double *uinf, *param, *tau;
  const double *udg, *uh, *sdg;
  double time, dtfactor;
  int tdep, tdfunc, sourcefunc, modelnumber;
  int e0;  // first element of the chunk; per-chunk outputs are indexed from it
  // mixed form: G goes straight into the packed 3xTF32 operand of the q elimination (one
  // part per trace component) instead of the FP64 G; unused when Gp.hi is null
  UPacked Gp;
  // mixed form with the tensor-core volume kernel: B is packed the same way (written by the
  // volume kernel, face terms added here) instead of the FP64 B; unused when Bp.hi is null
  UPacked Bp;
  // Gauss-point values computed for the whole chunk by GEMMs (null: per element here): udg at
  // the Gauss points [nge, nc] and the stage source sdg at them [nge, ncu] per chunk element
  const double *ugpre, *sgpre;
  // when set, the volume kernel leaves its Ru integrand [nge, nd + 1, ncu] per chunk element
  // here and the contraction with shapegw runs as one GEMM over the chunk
  double* rgout;
};

// ----------------------------------------------------------------------------------
// volume: quadrature-point values, Ru (volume part) and the Jacobian integrands rgJ
// rgJ per element: [nge, nd+1, ncu, nc]
// ----------------------------------------------------------------------------------
// The residual-only volume integrand with the Gauss-point values precomputed (ugpre, sgpre;
// rgout set): one thread per Gauss point of the chunk, the model evaluated at that point alone
// (N = 1), so with the dimension and the number of fields fixed at compile time its inputs and
// outputs stay in registers.  The same arithmetic as vol_points_kernel<Mdl, false> (the model's
// sums do not depend on N), with no shared memory and no barriers.  For nc <= VP_NC.
constexpr int VP_NC = 32;
template <class Mdl, int ND, int NCU>
__global__ void __launch_bounds__(128) vol_pointwise_kernel(AsmArgs A, int nb) {
  const ExaDims& P = A.P;
  const int nge = P.nge, nc = P.nc, ncx = P.ncx;
  const long long total = (long long)nb * nge;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(t % nge);
    const long long le = t / nge, e = A.e0 + le;
    const double* eg = A.elemg + e * P.elemg_stride();
    const double* Xx = eg + nge * ncx;
    double x[ND], uq[VP_NC], s[NCU], f[NCU * ND], td[NCU];
#pragma unroll
    for (int c = 0; c < ND; ++c) x[c] = eg[g + nge * c];
#pragma unroll
    for (int c = 0; c < VP_NC; ++c)
      if (c < nc) uq[c] = A.ugpre[g + nge * (c + (long long)nc * le)];
#pragma unroll
    for (int k = 0; k < NCU; ++k) {
      s[k] = 0.0;
      td[k] = 1.0;
    }
#pragma unroll
    for (int q = 0; q < NCU * ND; ++q) f[q] = 0.0;
    if (!A.tdep || A.sourcefunc == 1)
      Mdl::source_only(0, s, x, uq, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, 1, nc, NCU, ND, ncx,
                       P.nco, P.ncw);
    Mdl::flux_only(0, f, x, uq, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, 1, nc, NCU, ND, ncx, P.nco,
                   P.ncw);
    if (A.tdep && A.tdfunc == 1)
      Mdl::tdfunc(0, td, x, uq, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, 1, nc, NCU, ND, ncx, P.nco,
                  P.ncw);
    const double J = Xx[nge * ND * ND + g];
    double* o = A.rgout + (long long)le * nge * (ND + 1) * NCU;
#pragma unroll
    for (int k = 0; k < NCU; ++k) {
      double sg = s[k];
      if (A.tdep) {
        double fv = 1.0 * A.sgpre[g + nge * (k + (long long)NCU * le)] + (-A.dtfactor) * uq[k];
        if (A.tdfunc == 1) fv = 1.0 * fv * td[k];
        sg = 1.0 * sg + 1.0 * fv;
      }
      o[g + nge * (ND + 1) * k] = sg * J;
#pragma unroll
      for (int mm = 0; mm < ND; ++mm) {
        double v = f[k] * Xx[g + nge * (ND * mm)];
#pragma unroll
        for (int j = 1; j < ND; ++j) v += f[k + NCU * j] * Xx[g + nge * (j + ND * mm)];
        o[g + nge * (1 + mm) + nge * (ND + 1) * k] = v;
      }
    }
  }
}

// Launches vol_pointwise_kernel for the model's (nd, ncu); false when that pair has no instance
template <class Mdl>
bool launch_vol_pointwise(const AsmArgs& A, int nb, cudaStream_t st) {
  const ExaDims& P = A.P;
  if (P.nc > VP_NC || !A.ugpre || !A.rgout || (A.tdep && !A.sgpre)) return false;
  const long long total = (long long)nb * P.nge;
  const int blocks = (int)std::min<long long>((total + 127) / 128, 1 << 20);
#define EXA_VP(ND, NCU)                                                   \
  if (P.nd == ND && P.ncu == NCU) {                                       \
    vol_pointwise_kernel<Mdl, ND, NCU><<<blocks, 128, 0, st>>>(A, nb);    \
    return true;                                                          \
  }
  EXA_VP(1, 1) EXA_VP(2, 1) EXA_VP(3, 1) EXA_VP(2, 2) EXA_VP(3, 2) EXA_VP(2, 3) EXA_VP(3, 3)
  EXA_VP(2, 4) EXA_VP(3, 4) EXA_VP(2, 5) EXA_VP(3, 5)
#undef EXA_VP
  return false;
}

template <class Mdl, bool JAC>
__global__ void vol_points_kernel(AsmArgs A, double* Ru, double* rgJ) {
  extern __shared__ double sm[];
  const ExaDims& P = A.P;
  const int le = blockIdx.x, e = A.e0 + le;
  const int npe = P.npe, nge = P.nge, nc = P.nc, ncu = P.ncu, nd = P.nd, ncx = P.ncx;
  double* un = sm;                       // npe*nc
  double* ug = un + npe * nc;            // nge*nc
  double* xg = ug + nge * nc;            // nge*ncx
  double* sg = xg + nge * ncx;           // nge*ncu
  double* fg = sg + nge * ncu;           // nge*ncu*nd
  double* sdgg = fg + nge * ncu * nd;    // nge*ncu
  double* td = sdgg + nge * ncu;         // nge*ncu
  double* rgR = td + nge * ncu;          // nge*(nd+1)*ncu
  double* sJ = rgR + nge * (nd + 1) * ncu;  // nge*ncu*nc      (JAC)
  double* fJ = sJ + nge * ncu * nc;         // nge*ncu*nd*nc   (JAC)

  const double* eg = A.elemg + (long long)e * P.elemg_stride();
  const double* Xx = eg + nge * ncx;
  const double* jac = Xx + nge * nd * nd;
  const double* U = A.udg + (long long)e * npe * nc;
  if (!A.ugpre)
    for (int t = threadIdx.x; t < npe * nc; t += blockDim.x) un[t] = U[t];
  for (int t = threadIdx.x; t < nge * ncx; t += blockDim.x) xg[t] = eg[t];
  for (int t = threadIdx.x; t < nge * ncu * nd; t += blockDim.x) fg[t] = 0.0;
  for (int t = threadIdx.x; t < nge * ncu; t += blockDim.x) sg[t] = 0.0;
  if (JAC) {
    for (int t = threadIdx.x; t < nge * ncu * nc; t += blockDim.x) sJ[t] = 0.0;
    for (int t = threadIdx.x; t < nge * ncu * nd * nc; t += blockDim.x) fJ[t] = 0.0;
  }
  __syncthreads();
  if (A.ugpre) {
    const double* ugp = A.ugpre + (long long)le * nge * nc;
    for (int t = threadIdx.x; t < nge * nc; t += blockDim.x) ug[t] = ugp[t];
  } else {
    for (int t = threadIdx.x; t < nge * nc; t += blockDim.x) {
      const int g = t % nge, c = t / nge;
      double s = 0.0;
#pragma unroll 8
      for (int j = 0; j < npe; ++j) s = fma(A.shapegt[g + nge * j], un[j + npe * c], s);
      ug[t] = s;
    }
  }
  if (A.tdep) {
    if (A.sgpre) {
      const double* sgp = A.sgpre + (long long)le * nge * ncu;
      for (int t = threadIdx.x; t < nge * ncu; t += blockDim.x) sdgg[t] = sgp[t];
    } else {
      const double* S = A.sdg + (long long)e * npe * ncu;
      for (int t = threadIdx.x; t < nge * ncu; t += blockDim.x) {
        const int g = t % nge, k = t / nge;
        double s = 0.0;
#pragma unroll 8
        for (int j = 0; j < npe; ++j) s = fma(A.shapegt[g + nge * j], S[j + npe * k], s);
        sdgg[t] = s;
      }
    }
  }
  __syncthreads();
  for (int g = threadIdx.x; g < nge; g += blockDim.x) {
    if (JAC) {
      Mdl::source(g, sg, sJ, nullptr, xg, ug, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, nge, nc,
                  ncu, nd, ncx, P.nco, P.ncw);
      Mdl::flux(g, fg, fJ, nullptr, xg, ug, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, nge, nc, ncu,
                nd, ncx, P.nco, P.ncw);
    } else {
      if (!A.tdep || A.sourcefunc == 1)
        Mdl::source_only(g, sg, xg, ug, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, nge, nc, ncu, nd,
                         ncx, P.nco, P.ncw);
      Mdl::flux_only(g, fg, xg, ug, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, nge, nc, ncu, nd, ncx,
                     P.nco, P.ncw);
    }
    if (A.tdep) {
      if (A.tdfunc == 1)
        Mdl::tdfunc(g, td, xg, ug, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, nge, nc, ncu, nd, ncx,
                    P.nco, P.ncw);
      else
        for (int k = 0; k < ncu; ++k) td[g + nge * k] = 1.0;
    }
  }
  __syncthreads();
  if (A.tdep) {
    // s += (sdg - dtfactor*u) * Tdfunc ; ds/du -= dtfactor * Tdfunc  (uequation.cpp:126-151)
    for (int t = threadIdx.x; t < nge * ncu; t += blockDim.x) {
      double f = 1.0 * sdgg[t] + (-A.dtfactor) * ug[t];
      if (JAC || A.tdfunc == 1) f = 1.0 * f * td[t];
      sg[t] = 1.0 * sg[t] + 1.0 * f;
      if (JAC) {
        const int g = t % nge, k = t / nge;
        sJ[g + nge * k + nge * ncu * k] += (-A.dtfactor) * td[t];
      }
    }
    __syncthreads();
  }
  // ApplyXxJac (kokkosimpl.h:2105-2159)
  for (int t = threadIdx.x; t < nge * ncu; t += blockDim.x) {
    const int g = t % nge, k = t / nge;
    rgR[g + nge * (nd + 1) * k] = sg[t] * jac[g];
    for (int mm = 0; mm < nd; ++mm) {
      double s = fg[g + nge * k] * Xx[g + nge * (nd * mm)];
      for (int j = 1; j < nd; ++j) s += fg[g + nge * (k + ncu * j)] * Xx[g + nge * (j + nd * mm)];
      rgR[g + nge * (1 + mm) + nge * (nd + 1) * k] = s;
    }
  }
  if (JAC) {
    double* R = rgJ + (long long)le * nge * (nd + 1) * ncu * nc;
    for (int t = threadIdx.x; t < nge * ncu * nc; t += blockDim.x) {
      const int g = t % nge, k = (t / nge) % ncu, c = t / (nge * ncu);
      const long long base = (long long)nge * (nd + 1) * (k + ncu * c);
      R[g + base] = sJ[t] * jac[g];
      for (int mm = 0; mm < nd; ++mm) {
        double s = fJ[g + nge * (k + ncu * nd * c)] * Xx[g + nge * (nd * mm)];
        for (int j = 1; j < nd; ++j) s += fJ[g + nge * (k + ncu * j + ncu * nd * c)] * Xx[g + nge * (j + nd * mm)];
        R[g + nge * (1 + mm) + base] = s;
      }
    }
  }
  __syncthreads();
  const int K = nge * (nd + 1);
  if (A.rgout) {
    double* o = A.rgout + (long long)le * K * ncu;
    for (int t = threadIdx.x; t < K * ncu; t += blockDim.x) o[t] = rgR[t];
    return;
  }
  // Ru(i,k) = sum_{g,d} shapegw[i,g,d] rgR[g,d,k]
  for (int t = threadIdx.x; t < npe * ncu; t += blockDim.x) {
    const int i = t % npe, k = t / npe;
    double s = 0.0;
    // unrolled so the weight loads (from L2) are in flight together; one accumulator, so the
    // sum keeps its order
#pragma unroll 8
    for (int q = 0; q < K; ++q) s = fma(A.shapegw[i + npe * q], rgR[q + K * k], s);
    Ru[(long long)le * P.n + t] = s;
  }
}

template <bool JAC>
inline size_t vol_points_smem(const ExaDims& P) {
  size_t s = (size_t)P.npe * P.nc + (size_t)P.nge * (P.nc + P.ncx + P.ncu + P.ncu * P.nd + 2 * P.ncu +
                                                      (P.nd + 1) * P.ncu);
  if (JAC) s += (size_t)P.nge * P.ncu * P.nc * (1 + P.nd);
  return s * sizeof(double);
}

// ----------------------------------------------------------------------------------
// D and B volume blocks: for each (k, c) pair,
//   M[i, j] = - sum_g ( sum_d shapegw[i,g,d] rgJ[g,d,k,c] ) shapegt[g,j]
// (the reference contracts shapegw x shapegt over (g,d) in one GEMM; summing over d
// first is the same sum with fewer products).  c < ncu goes to D[(i,k),(j,c)],
// c = ncu + nq + ncu*d goes to B[(i,k), j + npe*d + npe*nd*nq].
// Grid: (tiles, elements, ncu*nc); 64x64 tiles as exa_gemm.
// ----------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) vol_mat_kernel(ExaDims P, const double* shapegw, const double* shapegt,
                                                      const double* rgJ, double* D, double* B) {
  constexpr int TMv = 64, TNv = 64, TKv = 16;
  __shared__ double As[TKv][TMv + 1];
  __shared__ double Bs[TKv][TNv + 1];
  const int npe = P.npe, nge = P.nge, nd = P.nd, ncu = P.ncu, n = P.n;
  const int tiles = (npe + TMv - 1) / TMv;
  const int tm = blockIdx.x % tiles, tn = blockIdx.x / tiles;
  const int le = blockIdx.y, kc = blockIdx.z;
  const int k = kc % ncu, c = kc / ncu;
  const double* R = rgJ + (long long)le * nge * (nd + 1) * ncu * P.nc + (long long)nge * (nd + 1) * kc;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int r0 = tm * TMv, c0 = tn * TNv;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int g0 = 0; g0 < nge; g0 += TKv) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int t = threadIdx.x + 256 * q;
      const int r = t & 63, kk = t >> 6;
      const int gi = r0 + r, gg = g0 + kk;
      double v = 0.0;
      if (gi < npe && gg < nge)
        for (int d = 0; d <= nd; ++d) v = fma(shapegw[gi + npe * gg + npe * nge * d], R[gg + nge * d], v);
      As[kk][r] = v;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int t = threadIdx.x + 256 * q;
      const int kk = t & 15, cc = t >> 4;
      const int gg = g0 + kk, gj = c0 + cc;
      Bs[kk][cc] = (gg < nge && gj < npe) ? shapegt[gg + nge * gj] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TKv; ++kk) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = As[kk][ty + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = Bs[kk][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
    __syncthreads();
  }
  double* out;
  long long col0, ld = n;
  if (c < ncu) {
    out = D + (long long)le * n * n;
    col0 = (long long)npe * c;
  } else {
    const int qc = c - ncu, nq = qc % ncu, d = qc / ncu;
    out = B + (long long)le * n * npe * nd * ncu;
    col0 = (long long)npe * d + (long long)npe * nd * nq;
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = r0 + ty + 16 * a;
    if (i >= npe) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int j = c0 + tx + 16 * b;
      if (j >= npe) continue;
      out[(i + npe * k) + ld * (col0 + j)] = -acc[a][b];
    }
  }
}

// The left factors of the same products for elements le0 .. le0 + nbs - 1 of the chunk, for the
// FP64 DMMA GEMM: T[i, g] = -sum_d shapegw[i, g, d] rgJ[g, d, k, c], npe x nge column-major, block
// (k, c) of element le at T + ((le - le0) ncu nc + k + ncu c) npe nge.  Consecutive threads take
// consecutive i: the weight loads are coalesced and the rgJ loads shared by the warp.
__global__ void vol_t_kernel(ExaDims P, const double* __restrict__ shapegw, const double* __restrict__ rgJ, int le0,
                             int nbs, double* __restrict__ T) {
  const int npe = P.npe, nge = P.nge, nd = P.nd, nblk = P.ncu * P.nc;
  const long long blk = (long long)npe * nge;
  const long long total = blk * nblk * nbs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long bq = t / blk;  // (element, block) pair
    const int r = (int)(t - bq * blk), i = r % npe, g = r / npe;
    const double* R = rgJ + (long long)(le0 + bq / nblk) * nge * (nd + 1) * nblk + (long long)nge * (nd + 1) * (bq % nblk);
    double v = 0.0;
    for (int d = 0; d <= nd; ++d) v = fma(shapegw[i + (long long)npe * (g + (long long)nge * d)], R[g + nge * d], v);
    T[t] = -v;
  }
}

// ----------------------------------------------------------------------------------
// faces.  Per element face l (processed in order by the whole block):
//   uhat, (u, q) at the face nodes (elemcon / perm), then at the face points;
//   numerical flux fh = f(uhat, q).n + tau (u - uhat) and its derivatives
//   (FhatDriver, backend/Model/ModelDrivers.cpp:789-849), times the face jacobian;
//   interior formula into Ru, D, B, F; trace rows (Fbou on boundary faces) into
//   Rh, K, G, H (uequation.cpp:300-487, kokkosimpl.h:1650-1730).
// JAC = false computes Ru and Rh only (RuEquationElemFaceBlock, uequation.cpp:883-1077).
// F, K, G, H must be zero on entry; Ru holds the volume part.
// ----------------------------------------------------------------------------------
template <class Mdl, bool JAC>
__global__ void face_kernel(AsmArgs A, double* Ru, double* Rh, double* D, double* B, double* F, double* K,
                            double* G, double* H) {
  extern __shared__ double sm[];
  const ExaDims& P = A.P;
  const int le = blockIdx.x, e = A.e0 + le;
  const int npe = P.npe, npf = P.npf, ngf = P.ngf, nc = P.nc, ncu = P.ncu, nd = P.nd, ncx = P.ncx;
  const int nfe = P.nfe, ndf = P.ndf, n = P.n, m = P.m;
  const int nqn = npe * nd * ncu;  // columns of B and G
  double* sW = sm;                    // npf*ngf: shapfgw[:, :, 0]
  double* sT = sW + npf * ngf;        // ngf*npf: shapfgt[:, :, 0]
  double* uhn = sT + npf * ngf;       // npf*ncu
  double* un = uhn + npf * ncu;       // npf*nc
  double* uhg = un + npf * nc;        // ngf*ncu
  double* ugq = uhg + ngf * ncu;      // ngf*nc   (u, q)
  double* uqh = ugq + ngf * nc;       // ngf*nc   (uhat, q)
  double* fg = uqh + ngf * nc;        // ngf*ncu*nd
  double* fh = fg + ngf * ncu * nd;   // ngf*ncu
  double* fb = fh + ngf * ncu;        // ngf*ncu
  double* fJ = fb + ngf * ncu;        // ngf*ncu*nd*nc   (JAC)
  double* fh_uq = fJ + ngf * ncu * nd * nc;  // ngf*ncu*nc
  double* fh_uh = fh_uq + ngf * ncu * nc;    // ngf*ncu*ncu
  double* fb_uq = fh_uh + ngf * ncu * ncu;   // ngf*ncu*nc
  double* fb_uh = fb_uq + ngf * ncu * nc;    // ngf*ncu*ncu
  // JAC: index tables of the block placement, filled once per element (no divisions per entry):
  // column q = k + ncu c of the derivatives as k | c << 8 | (c - ncu) % ncu << 16 | (c - ncu) / ncu
  // << 24; the row parts of the packed offsets of B (rows of Ru) and G (trace rows), with the
  // row groups of their tiles
  int* qtab = reinterpret_cast<int*>(fb_uh + ngf * ncu * ncu);  // ncu*nc
  int* brow = qtab + ncu * nc;  // n: row part, then n: groups of the row's tile
  int* grow = brow + 2 * n;     // m, m
  // JAC in the mixed form (packed G given): the pair products in FP32, from FP32 copies of the
  // face weights (once per element) and of each face's flux derivatives
  const bool f32 = JAC && A.Gp.hi != nullptr;
  float* sW32 = reinterpret_cast<float*>(grow + 2 * m);  // npf*ngf
  float* sT32 = sW32 + npf * ngf;                        // ngf*npf
  float* fq32 = sT32 + npf * ngf;                        // ngf*ncu*nc: fh_uq
  float* fTq32 = fq32 + ngf * ncu * nc;                  // ngf*ncu*nc: trace-row u-q derivatives
  float* fh32 = fTq32 + ngf * ncu * nc;                  // ngf*ncu*ncu: fh_uh
  float* fTh32 = fh32 + ngf * ncu * ncu;                 // ngf*ncu*ncu: trace-row uhat derivatives
  __shared__ int s_ib;
  for (int t = threadIdx.x; t < npf * ngf; t += blockDim.x) {
    sW[t] = A.shapfgw[t];
    sT[t] = A.shapfgt[t];
  }
  if (f32)
    for (int t = threadIdx.x; t < npf * ngf; t += blockDim.x) {
      sW32[t] = (float)A.shapfgw[t];
      sT32[t] = (float)A.shapfgt[t];
    }
  if (JAC) {
    for (int q = threadIdx.x; q < ncu * nc; q += blockDim.x) {
      const int k = q % ncu, c = q / ncu;
      const int qc = c < ncu ? 0 : c - ncu;
      qtab[q] = k | (c << 8) | ((qc % ncu) << 16) | ((qc / ncu) << 24);
    }
    auto rowpart = [](int row, int R, int K, int TR, int& ng) {
      const int nkc = (K + exa_tc::PK - 1) / exa_tc::PK;
      const int t = row / TR, rl = row - t * TR;
      const int rows_t = (R - t * TR) < TR ? (R - t * TR) : TR;
      ng = (rows_t + 7) / 8;
      return t * (TR / 8) * nkc * 128 + (rl >> 3) * 128 + (rl & 7) * 4;
    };
    const int qg = exa_tc::qk_group(npe);
    if (A.Bp.hi)
      for (int r = threadIdx.x; r < n; r += blockDim.x) brow[r] = rowpart(r, n, qg * nd, A.Bp.TR, brow[n + r]);
    if (A.Gp.hi)
      for (int r = threadIdx.x; r < m; r += blockDim.x) grow[r] = rowpart(r, m, qg * nd, A.Gp.TR, grow[m + r]);
  }

  const double* U = A.udg + (long long)e * npe * nc;
  double* Rue = Ru + (long long)le * n;
  double* Rhe = Rh + (long long)le * m;
  const double tau0 = A.tau[0];
  for (int l = 0; l < nfe; ++l) {
    const double* fgeo = A.faceg + ((long long)e * nfe + l) * P.faceg_stride();
    const double* xg = fgeo;
    const double* nl = fgeo + ngf * ncx;
    const double* jac = nl + ngf * nd;
    const int* pl = A.perm + npf * l;
    if (threadIdx.x == 0) s_ib = A.bf[l + nfe * e];
    for (int t = threadIdx.x; t < npf * ncu; t += blockDim.x) {
      const int a = t % npf, k = t / npf;
      uhn[t] = A.uh[k + ncu * (long long)A.elemcon[a + npf * l + ndf * e]];
    }
    for (int t = threadIdx.x; t < npf * nc; t += blockDim.x) {
      const int a = t % npf, c = t / npf;
      un[t] = U[pl[a] + npe * c];
    }
    for (int t = threadIdx.x; t < ngf * ncu * nd; t += blockDim.x) fg[t] = 0.0;
    if (JAC)
      for (int t = threadIdx.x; t < ngf * ncu * nd * nc; t += blockDim.x) fJ[t] = 0.0;
    for (int t = threadIdx.x; t < ngf * ncu; t += blockDim.x) fb[t] = 0.0;
    if (JAC) {
      for (int t = threadIdx.x; t < ngf * ncu * nc; t += blockDim.x) fb_uq[t] = 0.0;
      for (int t = threadIdx.x; t < ngf * ncu * ncu; t += blockDim.x) fb_uh[t] = 0.0;
    }
    __syncthreads();
    const int ib = s_ib;
    for (int t = threadIdx.x; t < ngf * ncu; t += blockDim.x) {
      const int g = t % ngf, k = t / ngf;
      double s = 0.0;
      for (int a = 0; a < npf; ++a) s = fma(sT[g + ngf * a], uhn[a + npf * k], s);
      uhg[t] = s;
    }
    for (int t = threadIdx.x; t < ngf * nc; t += blockDim.x) {
      const int g = t % ngf, c = t / ngf;
      double s = 0.0;
      for (int a = 0; a < npf; ++a) s = fma(sT[g + ngf * a], un[a + npf * c], s);
      ugq[t] = s;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < ngf * nc; t += blockDim.x) uqh[t] = (t < ngf * ncu) ? uhg[t] : ugq[t];
    __syncthreads();
    for (int g = threadIdx.x; g < ngf; g += blockDim.x) {
      if (JAC) {
        Mdl::flux(g, fg, fJ, nullptr, xg, uqh, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, ngf, nc, ncu,
                  nd, ncx, P.nco, P.ncw);
        if (ib > 0)
          Mdl::fbou(g, fb, fb_uq, nullptr, fb_uh, xg, ugq, nullptr, nullptr, uhg, nl, A.tau, A.uinf, A.param, A.time,
                    A.modelnumber, ib, ngf, nc, ncu, nd, ncx, P.nco, P.ncw);
      } else {
        Mdl::flux_only(g, fg, xg, uqh, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, ngf, nc, ncu, nd, ncx,
                       P.nco, P.ncw);
        if (ib > 0)
          Mdl::fbou_only(g, fb, xg, ugq, nullptr, nullptr, uhg, nl, A.tau, A.uinf, A.param, A.time, A.modelnumber, ib,
                         ngf, nc, ncu, nd, ncx, P.nco, P.ncw);
      }
    }
    __syncthreads();
    // f.n, derivatives, stabilisation, face jacobian (FluxDotNormal, AddStabilization1,
    // columnwiseMultiply)
    for (int t = threadIdx.x; t < ngf * ncu; t += blockDim.x) {
      const int g = t % ngf, k = t / ngf;
      double s = fg[g + ngf * k] * nl[g];
      for (int d = 1; d < nd; ++d) s += fg[g + ngf * (k + ncu * d)] * nl[g + ngf * d];
      s += tau0 * (ugq[t] - uhg[t]);
      fh[t] = s * jac[g];
      if (ib > 0) fb[t] = fb[t] * jac[g];
      if (JAC) {
        for (int c = 0; c < nc; ++c) {
          double v = fJ[g + ngf * (k + ncu * nd * c)] * nl[g];
          for (int d = 1; d < nd; ++d) v += fJ[g + ngf * (k + ncu * d + ncu * nd * c)] * nl[g + ngf * d];
          if (c < ncu) {
            double vh = v, vu = 0.0;
            if (c == k) {
              vu += tau0;
              vh -= tau0;
            }
            fh_uh[g + ngf * (k + ncu * c)] = vh * jac[g];
            fh_uq[g + ngf * (k + ncu * c)] = vu * jac[g];
          } else {
            fh_uq[g + ngf * (k + ncu * c)] = v * jac[g];
          }
          if (ib > 0) {
            fb_uq[g + ngf * (k + ncu * c)] *= jac[g];
            if (c < ncu) fb_uh[g + ngf * (k + ncu * c)] *= jac[g];
          }
        }
      }
    }
    __syncthreads();
    const double* fT = (ib > 0) ? fb : fh;
    // Ru -= shapfgw . fh at this face's element nodes; Rh = -shapfgw . fT
    for (int t = threadIdx.x; t < npf * ncu; t += blockDim.x) {
      const int a = t % npf, k = t / npf;
      double s = 0.0, r = 0.0;
      for (int g = 0; g < ngf; ++g) {
        s = fma(sW[a + npf * g], fh[g + ngf * k], s);
        r = fma(sW[a + npf * g], fT[g + ngf * k], r);
      }
      Rue[pl[a] + npe * k] -= s;
      Rhe[k + ncu * (a + npf * l)] = -r;
    }
    if (JAC) {
      const double* fT_uq = (ib > 0) ? fb_uq : fh_uq;
      const double* fT_uh = (ib > 0) ? fb_uh : fh_uh;
      double* De = D + (long long)le * n * n;
      double* Be = B + (long long)le * n * nqn;
      double* Fe = F + (long long)le * n * m;
      double* Ke = K + (long long)le * m * n;
      double* Ge = G + (long long)le * m * nqn;
      double* He = H + (long long)le * m * m;
      // one thread per face-node pair (a, b): the weight w_g = shapfgw[a, g] shapfgt[g, b] is
      // formed once per g and shared by every column q = k + ncu c, taken QC at a time
      constexpr int QC = 4;
      const int nq = ncu * nc;
      const int qg = exa_tc::qk_group(npe);  // K group of the packed B and G
      // the pair products of the face, in TA (FP64, or FP32 in the mixed form)
      auto pairs = [&](auto zero, const auto* W, const auto* Tt, const auto* fq, const auto* fTq, const auto* fh,
                       const auto* fTh) {
        using TA = decltype(zero);
        for (int ab = threadIdx.x; ab < npf * npf; ab += blockDim.x) {
          const int a = ab % npf, b = ab / npf;
          const int pa = pl[a], pb = pl[b];
          for (int q0 = 0; q0 < nq; q0 += QC) {
            TA vq[QC], vT[QC], vh[QC], vTh[QC];
  #pragma unroll
            for (int u = 0; u < QC; ++u) vq[u] = vT[u] = vh[u] = vTh[u] = TA(0);
            for (int g = 0; g < ngf; ++g) {
              const TA w = W[a + npf * g] * Tt[g + ngf * b];
  #pragma unroll
              for (int u = 0; u < QC; ++u) {
                const int q = q0 + u;
                if (q < nq) {
                  vq[u] = fma(w, fq[g + ngf * q], vq[u]);
                  vT[u] = fma(w, fTq[g + ngf * q], vT[u]);
                  if (q < ncu * ncu) {
                    vh[u] = fma(w, fh[g + ngf * q], vh[u]);
                    vTh[u] = fma(w, fTh[g + ngf * q], vTh[u]);
                  }
                }
              }
            }
  #pragma unroll
            for (int u = 0; u < QC; ++u) {
              const int q = q0 + u;
              if (q >= nq) break;
              const int qd = qtab[q];
              const int k = qd & 255, c = (qd >> 8) & 255;
              const int row_e = pa + npe * k;             // element row (i,k)
              const int row_t = k + ncu * (a + npf * l);  // trace row (k, jf)
              if (c < ncu) {
                De[row_e + (long long)n * (pb + npe * c)] += vq[u];
                Fe[row_e + (long long)n * (c + ncu * (b + npf * l))] = vh[u];
                Ke[row_t + (long long)m * (pb + npe * c)] = vT[u];
                He[row_t + (long long)m * (c + ncu * (b + npf * l))] = vTh[u];
              } else {
                const int nqc = (qd >> 16) & 255, d = qd >> 24;
                const long long col = pb + (long long)npe * d + (long long)npe * nd * nqc;
                // packed column part of k = pb + qg d for a row of ng groups (pack_off's k terms)
                const int kk = pb + qg * d;
                auto colpart = [kk](int ng) { return (kk >> 4) * ng * 128 + ((kk >> 2) & 3) * 32 + (kk & 3); };
                if (A.Bp.hi) {
                  float* bp = A.Bp.hi + (long long)le * A.Bp.sb + (long long)nqc * A.Bp.sb2 + brow[row_e] +
                              colpart(brow[n + row_e]);
                  *bp += (float)vq[u];
                } else {
                  Be[row_e + (long long)n * col] += vq[u];
                }
                if (A.Gp.hi) {
                  const long long o = (long long)le * A.Gp.sb + (long long)nqc * A.Gp.sb2 + grow[row_t] +
                                      colpart(grow[m + row_t]);
                  if (A.Gp.lo) {
                    float h, lo;
                    exa_tc::split_tf32(vT[u], h, lo);
                    A.Gp.hi[o] = h;
                    A.Gp.lo[o] = lo;
                  } else {
                    A.Gp.hi[o] = (float)vT[u];  // FP32 operand, split by the GEMM on chip
                  }
                } else {
                  Ge[row_t + (long long)m * col] = vT[u];
                }
              }
            }
          }
        }
      };
      if (f32) {
        for (int t = threadIdx.x; t < ngf * ncu * nc; t += blockDim.x) {
          fq32[t] = (float)fh_uq[t];
          fTq32[t] = (float)fT_uq[t];
        }
        for (int t = threadIdx.x; t < ngf * ncu * ncu; t += blockDim.x) {
          fh32[t] = (float)fh_uh[t];
          fTh32[t] = (float)fT_uh[t];
        }
        __syncthreads();
        pairs(0.0f, sW32, sT32, fq32, fTq32, fh32, fTh32);
      } else {
        pairs(0.0, sW, sT, fh_uq, fT_uq, fh_uh, fT_uh);
      }
    }
    __syncthreads();
  }
}

inline size_t face_smem(const ExaDims& P, bool jac) {
  size_t s = (size_t)P.npf * (P.ncu + P.nc) + (size_t)P.ngf * (P.ncu + 2 * P.nc + P.ncu * P.nd + 2 * P.ncu);
  if (jac) s += (size_t)P.ngf * P.ncu * (P.nd * P.nc + 2 * P.nc + 2 * P.ncu);
  s += 2 * (size_t)P.npf * P.ngf;  // shapfgw, shapfgt
  // the JAC index tables (ints): derivative columns, packed row parts of B and G; then the
  // FP32 copies of the mixed form's pair products (floats)
  const size_t ti = jac ? (size_t)P.ncu * P.nc + 2 * (size_t)P.n + 2 * (size_t)P.m : 0;
  const size_t tf = jac ? 2 * (size_t)P.npf * P.ngf + 2 * (size_t)P.ngf * P.ncu * (P.nc + P.ncu) : 0;
  return s * sizeof(double) + ti * sizeof(int) + tf * sizeof(float);
}

// Binds a generated model namespace to the argument roles the kernels use
// (Exasim's DefaultModel functors, backend/Model/modeltemplate.hpp:377-457).
#define EXA_BIND_MODEL(NS)                                                                                      \
  struct ExaModel {                                                                                             \
    __device__ static void flux(size_t i, double* f, double* J1, double* J2, const double* x, const double* uq,  \
                                const double* v, const double* w, const double* eta, const double* mu,          \
                                double t, int mn, int N, int a, int b, int c, int d, int e, int h) {           \
      NS::HdgFlux_pt(i, f, J1, J2, x, uq, v, w, eta, mu, t, mn, N, a, b, c, d, e, h);                            \
    }                                                                                                           \
    __device__ static void source(size_t i, double* f, double* J1, double* J2, const double* x, const double* uq, \
                                  const double* v, const double* w, const double* eta, const double* mu,        \
                                  double t, int mn, int N, int a, int b, int c, int d, int e, int h) {         \
      NS::HdgSource_pt(i, f, J1, J2, x, uq, v, w, eta, mu, t, mn, N, a, b, c, d, e, h);                          \
    }                                                                                                           \
    __device__ static void flux_only(size_t i, double* f, const double* x, const double* uq, const double* v,    \
                                     const double* w, const double* eta, const double* mu, double t, int mn,    \
                                     int N, int a, int b, int c, int d, int e, int h) {                         \
      NS::KokkosFlux_pt(i, f, x, uq, v, w, eta, mu, t, mn, N, a, b, c, d, e, h);                                 \
    }                                                                                                           \
    __device__ static void source_only(size_t i, double* f, const double* x, const double* uq, const double* v,  \
                                       const double* w, const double* eta, const double* mu, double t, int mn,  \
                                       int N, int a, int b, int c, int d, int e, int h) {                       \
      NS::KokkosSource_pt(i, f, x, uq, v, w, eta, mu, t, mn, N, a, b, c, d, e, h);                               \
    }                                                                                                           \
    __device__ static void tdfunc(size_t i, double* f, const double* x, const double* uq, const double* v,       \
                                  const double* w, const double* eta, const double* mu, double t, int mn, int N, \
                                  int a, int b, int c, int d, int e, int h) {                                   \
      NS::KokkosTdfunc_pt(i, f, x, uq, v, w, eta, mu, t, mn, N, a, b, c, d, e, h);                               \
    }                                                                                                           \
    __device__ static void fbou(size_t i, double* f, double* J1, double* J2, double* J3, const double* x,        \
                                const double* uq, const double* v, const double* w, const double* uh,           \
                                const double* nl, const double* tau, const double* eta, const double* mu,       \
                                double t, int mn, int ib, int N, int a, int b, int c, int d, int e, int h) {   \
      NS::HdgFbou_pt(i, f, J1, J2, J3, x, uq, v, w, uh, nl, tau, eta, mu, t, mn, ib, N, a, b, c, d, e, h);       \
    }                                                                                                           \
    __device__ static void fbou_only(size_t i, double* f, const double* x, const double* uq, const double* v,    \
                                     const double* w, const double* uh, const double* nl, const double* tau,    \
                                     const double* eta, const double* mu, double t, int mn, int ib, int N,     \
                                     int a, int b, int c, int d, int e, int h) {                                \
      NS::HdgFbouonly_pt(i, f, x, uq, v, w, uh, nl, tau, eta, mu, t, mn, ib, N, a, b, c, d, e, h);               \
    }                                                                                                           \
    /* the LDG boundary functions (KokkosUbou, KokkosFbou); empty when the model has none */                    \
    static constexpr bool has_ldg_boundary = NS::has_KokkosUbou && NS::has_KokkosFbou;                          \
    __device__ static void ubou(size_t i, double* f, const double* x, const double* uq, const double* uh,        \
                                const double* nl, const double* tau, const double* eta, const double* mu,       \
                                double t, int mn, int ib, int N, int a, int b, int c, int d, int e, int h) {   \
      NS::KokkosUbou_pt(i, f, x, uq, nullptr, nullptr, uh, nl, tau, eta, mu, t, mn, ib, N, a, b, c, d, e, h);    \
    }                                                                                                           \
    __device__ static void fbou_ldg(size_t i, double* f, const double* x, const double* uq, const double* uh,    \
                                    const double* nl, const double* tau, const double* eta, const double* mu,   \
                                    double t, int mn, int ib, int N, int a, int b, int c, int d, int e,        \
                                    int h) {                                                                    \
      NS::KokkosFbou_pt(i, f, x, uq, nullptr, nullptr, uh, nl, tau, eta, mu, t, mn, ib, N, a, b, c, d, e, h);    \
    }                                                                                                           \
  };

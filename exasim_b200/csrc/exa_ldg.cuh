// LDG face residual of one generated model (included by exa_model.cu after EXA_BIND_MODEL).
//
// One block per face f.  The states of the two sides at the face nodes (ldg_fcon: side 1's
// node order) are interpolated to the face Gauss points; inside the domain the numerical flux
// is the average of the two sides' fluxes dotted with side 1's outward normal plus the
// stabilisation tau (u1 - u2) (FhatDriver without a model Fhat, backend/Model/
// KokkosDrivers.cpp:349-409: AverageFlux, AverageFluxDotNormal, AddStabilization1/2/3,
// kokkosimpl.h:68-150); on the boundary uhat comes from the model's Ubou at the face nodes,
// with the nodes' coordinates and normals (UhatBlock, getuhat.cpp:121-145), and the flux from
// its Fbou at the Gauss points (FbouDriver, KokkosDrivers.cpp:413-438).  The flux times the
// face jacobian is projected on the face basis: Rh[a, k, f] = sum_g shapfgw[a, g] jac fhat
// (ApplyJacFhat + Gauss2Node, uresidual.cpp:323-326).
#pragma once
#include "exa_common.cuh"
#include "exa_kernels.cuh"

struct LdgArgs {
  ExaDims P;
  const double *shapfgt, *shapfgw, *shapfnt;
  const int *f2e, *perm, *bf, *fcon;
  const double *xdg, *faceg, *uinf, *param, *tau;
  int ntau, modelnumber;
  double time;
  const double* u;  // element states [npe, nc, ne]
  double* Rh;       // [npf, ncu, nf]
  int f0;           // first face of the launch
};

inline size_t ldg_face_smem(const ExaDims& P) {
  const size_t npf = P.npf, ngf = P.ngf, nc = P.nc, ncu = P.ncu, nd = P.nd, ncx = P.ncx;
  return sizeof(double) * (2 * npf * nc + 2 * ngf * nc + 2 * ngf * ncu * nd + ngf * ncu +  // u, ug, f, fh
                           npf * ncx + npf * nd + 2 * npf * ncu + ngf * ncu);              // boundary
}

template <class Mdl>
__global__ void __launch_bounds__(64) ldg_face_kernel(LdgArgs A) {
  extern __shared__ double sm[];
  const ExaDims& P = A.P;
  const int f = A.f0 + blockIdx.x;
  const int npe = P.npe, npf = P.npf, ngf = P.ngf, nc = P.nc, ncu = P.ncu, nd = P.nd, ncx = P.ncx, nfe = P.nfe;
  double* u1n = sm;                    // [npf, nc]
  double* u2n = u1n + npf * nc;        // [npf, nc]
  double* ug1 = u2n + npf * nc;        // [ngf, nc]
  double* ug2 = ug1 + ngf * nc;        // [ngf, nc]
  double* f1 = ug2 + ngf * nc;         // [ngf, ncu, nd]
  double* f2 = f1 + ngf * ncu * nd;    // [ngf, ncu, nd]
  double* fh = f2 + ngf * ncu * nd;    // [ngf, ncu]
  double* xn = fh + ngf * ncu;         // [npf, ncx]   boundary: node coordinates
  double* nn = xn + npf * ncx;         // [npf, nd]    boundary: node normals
  double* uhn = nn + npf * nd;         // [npf, ncu]   boundary: Ubou at the nodes
  double* uhs = uhn + npf * ncu;       // [npf, ncu]   the uhat argument of Ubou
  double* uhg = uhs + npf * ncu;       // [ngf, ncu]   boundary: uhat at the Gauss points
  const int e1 = A.f2e[4 * f], l1 = A.f2e[4 * f + 1], e2 = A.f2e[4 * f + 2];
  const bool bnd = e2 < 0;
  const double* fgeo = A.faceg + ((long long)e1 * nfe + l1) * P.faceg_stride();
  const double* xg = fgeo;
  const double* nl = fgeo + ngf * ncx;
  const double* jac = nl + ngf * nd;
  const int* fc = A.fcon + 2LL * npf * f;
  for (int t = threadIdx.x; t < npf * nc; t += blockDim.x) {
    const int a = t % npf, c = t / npf;
    const int k1 = fc[2 * a];
    u1n[t] = A.u[(k1 % npe) + npe * c + (long long)npe * nc * (k1 / npe)];
    if (!bnd) {
      const int k2 = fc[2 * a + 1];
      u2n[t] = A.u[(k2 % npe) + npe * c + (long long)npe * nc * (k2 / npe)];
    }
  }
  if (bnd) {
    // the face nodes' coordinates, then the tangents and the normal there (FaceGeom)
    const int* pl = A.perm + npf * l1;
    const double* X = A.xdg + (long long)e1 * npe * ncx;
    for (int t = threadIdx.x; t < npf; t += blockDim.x) {
      for (int c = 0; c < ncx; ++c) {
        double s = 0.0;
        for (int b = 0; b < npf; ++b) s += A.shapfnt[t + npf * b] * X[pl[b] + npe * c];
        xn[t + npf * c] = s;
      }
      if (nd == 1) {
        nn[t] = (l1 % 2 == 0) ? -1.0 : 1.0;
        continue;
      }
      double T[3][2];
      for (int c = 0; c < nd; ++c)
        for (int r = 0; r < nd - 1; ++r) {
          double s = 0.0;
          for (int b = 0; b < npf; ++b) s += A.shapfnt[t + npf * b + npf * npf * (1 + r)] * X[pl[b] + npe * c];
          T[c][r] = s;
        }
      if (nd == 2) {
        const double Jx = T[0][0], Jy = T[1][0];
        const double j = sqrt(Jx * Jx + Jy * Jy);
        nn[t] = Jy / j;
        nn[t + npf] = -Jx / j;
      } else {
        const double a1 = T[0][0], a2 = T[1][0], a3 = T[2][0];
        const double b1 = T[0][1], b2 = T[1][1], b3 = T[2][1];
        const double n1 = a2 * b3 - a3 * b2, n2 = a3 * b1 - a1 * b3, n3 = a1 * b2 - a2 * b1;
        const double j = sqrt(n1 * n1 + n2 * n2 + n3 * n3);
        nn[t] = n1 / j;
        nn[t + npf] = n2 / j;
        nn[t + 2 * npf] = n3 / j;
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < ngf * nc; t += blockDim.x) {
    const int g = t % ngf, c = t / ngf;
    double s1 = 0.0, s2 = 0.0;
    for (int a = 0; a < npf; ++a) {
      const double w = A.shapfgt[g + ngf * a];
      s1 = fma(w, u1n[a + npf * c], s1);
      if (!bnd) s2 = fma(w, u2n[a + npf * c], s2);
    }
    ug1[t] = s1;
    ug2[t] = s2;
  }
  for (int t = threadIdx.x; t < ngf * ncu * nd; t += blockDim.x) {
    f1[t] = 0.0;
    f2[t] = 0.0;
  }
  if (bnd)
    for (int t = threadIdx.x; t < npf * ncu; t += blockDim.x) {
      uhn[t] = 0.0;
      uhs[t] = u1n[t];  // Ubou's uhat argument: the side's own state (the reference passes scratch)
    }
  __syncthreads();
  const int ib = bnd ? A.bf[l1 + nfe * e1] : 0;
  if (!bnd) {
    // both sides' fluxes at once: threads [0, ngf) side 1, [ngf, 2 ngf) side 2
    for (int t = threadIdx.x; t < 2 * ngf; t += blockDim.x) {
      const int g = t < ngf ? t : t - ngf;
      Mdl::flux_only(g, t < ngf ? f1 : f2, xg, t < ngf ? ug1 : ug2, nullptr, nullptr, A.uinf, A.param, A.time,
                     A.modelnumber, ngf, nc, ncu, nd, ncx, P.nco, P.ncw);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < ngf * ncu; t += blockDim.x) {
      const int g = t % ngf, k = t / ngf;
      double s = (0.5 * (f1[g + ngf * k] + f2[g + ngf * k])) * nl[g];
      for (int d = 1; d < nd; ++d) {
        const int o = g + ngf * (k + ncu * d);
        s += (0.5 * (f1[o] + f2[o])) * nl[g + ngf * d];
      }
      if (A.ntau <= 1) {
        s += A.tau[0] * (ug1[t] - ug2[t]);
      } else if (A.ntau == ncu) {
        s += A.tau[k] * (ug1[t] - ug2[t]);
      } else {
        for (int j = 0; j < ncu; ++j) s += A.tau[j * ncu + k] * (ug1[g + ngf * j] - ug2[g + ngf * j]);
      }
      fh[t] = s * jac[g];
    }
  } else {
    for (int a = threadIdx.x; a < npf; a += blockDim.x)
      Mdl::ubou(a, uhn, xn, u1n, uhs, nn, A.tau, A.uinf, A.param, A.time, A.modelnumber, ib, npf, nc, ncu, nd, ncx,
                P.nco, P.ncw);
    __syncthreads();
    for (int t = threadIdx.x; t < ngf * ncu; t += blockDim.x) {
      const int g = t % ngf, k = t / ngf;
      double s = 0.0;
      for (int a = 0; a < npf; ++a) s = fma(A.shapfgt[g + ngf * a], uhn[a + npf * k], s);
      uhg[t] = s;
      fh[t] = 0.0;
    }
    __syncthreads();
    for (int g = threadIdx.x; g < ngf; g += blockDim.x)
      Mdl::fbou_ldg(g, fh, xg, ug1, uhg, nl, A.tau, A.uinf, A.param, A.time, A.modelnumber, ib, ngf, nc, ncu, nd, ncx,
                    P.nco, P.ncw);
    __syncthreads();
    for (int t = threadIdx.x; t < ngf * ncu; t += blockDim.x) fh[t] = fh[t] * jac[t % ngf];
  }
  __syncthreads();
  double* R = A.Rh + (long long)npf * ncu * f;
  for (int t = threadIdx.x; t < npf * ncu; t += blockDim.x) {
    const int a = t % npf, k = t / npf;
    double s = 0.0;
    for (int g = 0; g < ngf; ++g) s = fma(A.shapfgw[a + npf * g], fh[g + ngf * k], s);
    R[t] = s;
  }
}

// Interior faces with the dimension and the number of fields fixed at compile time (nc = ncu,
// no q): FPB faces per block; each face's states at its nodes (both sides) are staged in
// shared memory, then one thread per face Gauss point interpolates them, evaluates both sides'
// fluxes with the model at that point alone (N = 1, in registers) and forms jac fhat; then the
// projection on the face basis.  The same arithmetic as ldg_face_kernel's interior branch.
__host__ __device__ inline int ldg_faces_per_block(const ExaDims& P) { return P.ngf >= 128 ? 1 : 128 / P.ngf; }
inline size_t ldg_inner_smem(const ExaDims& P) {
  return sizeof(double) * (size_t)ldg_faces_per_block(P) * (2 * P.npf * P.nc + (size_t)P.ngf * P.ncu);
}

template <class Mdl, int ND, int NCU>
__global__ void __launch_bounds__(128, 6) ldg_face_inner_kernel(LdgArgs A, int nfaces) {
  extern __shared__ double sm[];
  const ExaDims& P = A.P;
  const int npe = P.npe, npf = P.npf, ngf = P.ngf, nfe = P.nfe, ncx = P.ncx;
  const int FPB = ldg_faces_per_block(P);
  const int fb = A.f0 + blockIdx.x * FPB;
  double* un = sm;                                  // [FPB][2][npf][NCU]
  double* fh = un + (size_t)FPB * 2 * npf * NCU;   // [FPB][ngf][NCU]
  for (int t = threadIdx.x; t < FPB * 2 * npf * NCU; t += blockDim.x) {
    const int c = t % NCU, a = (t / NCU) % npf, sd = (t / (NCU * npf)) % 2, j = t / (2 * NCU * npf);
    const int f = fb + j;
    if (f < A.f0 + nfaces) {
      const int k = A.fcon[2LL * (npf * (long long)f + a) + sd];
      un[t] = A.u[(k % npe) + npe * c + (long long)npe * NCU * (k / npe)];
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < FPB * ngf; t += blockDim.x) {
    const int g = t % ngf, j = t / ngf;
    const int f = fb + j;
    if (f >= A.f0 + nfaces) continue;
    const int e1 = A.f2e[4 * f], l1 = A.f2e[4 * f + 1];
    const double* fgeo = A.faceg + ((long long)e1 * nfe + l1) * P.faceg_stride();
    const double* u1 = un + (size_t)j * 2 * npf * NCU;
    const double* u2 = u1 + npf * NCU;
    double x[ND], n[ND], ug1[NCU], ug2[NCU], f1[NCU * ND], f2[NCU * ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      x[d] = fgeo[g + ngf * d];
      n[d] = fgeo[g + ngf * (ncx + d)];
    }
    const double jac = fgeo[g + ngf * (ncx + ND)];
#pragma unroll
    for (int c = 0; c < NCU; ++c) {
      double s1 = 0.0, s2 = 0.0;
      for (int a = 0; a < npf; ++a) {
        const double w = A.shapfgt[g + ngf * a];
        s1 = fma(w, u1[a * NCU + c], s1);
        s2 = fma(w, u2[a * NCU + c], s2);
      }
      ug1[c] = s1;
      ug2[c] = s2;
    }
#pragma unroll
    for (int q = 0; q < NCU * ND; ++q) {
      f1[q] = 0.0;
      f2[q] = 0.0;
    }
    Mdl::flux_only(0, f1, x, ug1, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, 1, NCU, NCU, ND, ncx,
                   P.nco, P.ncw);
    Mdl::flux_only(0, f2, x, ug2, nullptr, nullptr, A.uinf, A.param, A.time, A.modelnumber, 1, NCU, NCU, ND, ncx,
                   P.nco, P.ncw);
    double* o = fh + (size_t)j * ngf * NCU;
#pragma unroll
    for (int k = 0; k < NCU; ++k) {
      double s = (0.5 * (f1[k] + f2[k])) * n[0];
#pragma unroll
      for (int d = 1; d < ND; ++d) s += (0.5 * (f1[k + NCU * d] + f2[k + NCU * d])) * n[d];
      if (A.ntau <= 1) {
        s += A.tau[0] * (ug1[k] - ug2[k]);
      } else if (A.ntau == NCU) {
        s += A.tau[k] * (ug1[k] - ug2[k]);
      } else {
#pragma unroll
        for (int i = 0; i < NCU; ++i) s += A.tau[i * NCU + k] * (ug1[i] - ug2[i]);
      }
      o[g + ngf * k] = s * jac;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < FPB * npf * NCU; t += blockDim.x) {
    const int a = t % npf, k = (t / npf) % NCU, j = t / (npf * NCU);
    const int f = fb + j;
    if (f >= A.f0 + nfaces) continue;
    const double* o = fh + (size_t)j * ngf * NCU;
    double s = 0.0;
    for (int g = 0; g < ngf; ++g) s = fma(A.shapfgw[a + npf * g], o[g + ngf * k], s);
    A.Rh[a + (long long)npf * (k + (long long)NCU * f)] = s;
  }
}

// Launches ldg_face_inner_kernel over `nfaces` interior faces from A.f0 for the model's
// (nd, ncu); false when that pair has no instance (the general kernel runs them then)
template <class Mdl>
bool launch_ldg_face_inner(const LdgArgs& A, int nfaces, cudaStream_t st) {
  const ExaDims& P = A.P;
  if (P.nc != P.ncu || nfaces <= 0) return false;
  const int FPB = ldg_faces_per_block(P);
  const unsigned blocks = (unsigned)((nfaces + FPB - 1) / FPB);
  const size_t smem = ldg_inner_smem(P);
#define EXA_LF(ND, NCU)                                                                               \
  if (P.nd == ND && P.ncu == NCU) {                                                                   \
    if (exa_allow_smem((const void*)ldg_face_inner_kernel<Mdl, ND, NCU>, smem) != 0) return false;    \
    ldg_face_inner_kernel<Mdl, ND, NCU><<<blocks, 128, smem, st>>>(A, nfaces);                        \
    return true;                                                                                      \
  }
  EXA_LF(1, 1) EXA_LF(2, 1) EXA_LF(3, 1) EXA_LF(2, 4) EXA_LF(3, 4) EXA_LF(2, 5) EXA_LF(3, 5)
#undef EXA_LF
  return false;
}

// Model-independent HDG kernels: geometry at quadrature points, the q-equation
// element matrices, and the trace-space operations of the Krylov solver (gather /
// scatter through the face connectivity, condensed matvec, block-Jacobi and
// elemental additive-Schwarz preconditioners, Newton update of the element unknowns).
// Every kernel maps one element (or one face) to one block, so the element-to-face
// assembly needs no atomics: the first element of a face writes, the second adds,
// as Exasim's PutElementFaceNodes pair does (backend/Common/kokkosimpl.h:1032-1065).
#include <map>
#include <mutex>
#include <tuple>

#include "exa_kernels.cuh"
#include "exa_tc.cuh"
#include "exa_umma.cuh"

namespace {

// ----------------------------------------------------------------------------------
// geometry (backend/Discretization/geometry.cpp:44-222, kokkosimpl.h:2321-2415)
// elemg per element: xg [nge, ncx] | Xx [nge, nd*nd] | jac [nge]
// faceg per element face: xg [ngf, ncx] | nl [ngf, nd] | jac [ngf]
// ----------------------------------------------------------------------------------
__global__ void elem_geom_kernel(ExaDims P, const double* shapegt, const double* xdg, double* elemg) {
  const int e = blockIdx.x;
  const int nge = P.nge, npe = P.npe, nd = P.nd, ncx = P.ncx;
  const double* x = xdg + (long long)e * npe * ncx;
  double* out = elemg + (long long)e * P.elemg_stride();
  for (int g = threadIdx.x; g < nge; g += blockDim.x) {
    double J[3][3];  // J[c][r] = d x_c / d xi_r
    for (int c = 0; c < ncx; ++c) {
      double s = 0.0;
      for (int j = 0; j < npe; ++j) s += shapegt[g + nge * j] * x[j + npe * c];
      out[g + nge * c] = s;
    }
    for (int c = 0; c < nd; ++c)
      for (int r = 0; r < nd; ++r) {
        double s = 0.0;
        for (int j = 0; j < npe; ++j) s += shapegt[g + nge * j + nge * npe * (1 + r)] * x[j + npe * c];
        J[c][r] = s;
      }
    double* Xx = out + nge * ncx;
    double* jac = Xx + nge * nd * nd;
    if (nd == 1) {
      jac[g] = J[0][0];
      Xx[g] = 1.0;
    } else if (nd == 2) {
      const double J11 = J[0][0], J12 = J[1][0], J21 = J[0][1], J22 = J[1][1];
      jac[g] = J11 * J22 - J12 * J21;
      Xx[g + nge * 0] = J22;    // Xx11
      Xx[g + nge * 1] = -J21;   // Xx21 = jac * dxi/dy
      Xx[g + nge * 2] = -J12;   // Xx12 = jac * deta/dx
      Xx[g + nge * 3] = J11;    // Xx22
    } else {
      const double J11 = J[0][0], J12 = J[1][0], J13 = J[2][0];
      const double J21 = J[0][1], J22 = J[1][1], J23 = J[2][1];
      const double J31 = J[0][2], J32 = J[1][2], J33 = J[2][2];
      jac[g] = J11 * J22 * J33 - J11 * J32 * J23 + J21 * J32 * J13 - J21 * J12 * J33 + J31 * J12 * J23 -
               J31 * J22 * J13;
      Xx[g + nge * 0] = J22 * J33 - J23 * J32;
      Xx[g + nge * 1] = J23 * J31 - J21 * J33;
      Xx[g + nge * 2] = J21 * J32 - J22 * J31;
      Xx[g + nge * 3] = J13 * J32 - J12 * J33;
      Xx[g + nge * 4] = J11 * J33 - J13 * J31;
      Xx[g + nge * 5] = J12 * J31 - J11 * J32;
      Xx[g + nge * 6] = J12 * J23 - J13 * J22;
      Xx[g + nge * 7] = J13 * J21 - J11 * J23;
      Xx[g + nge * 8] = J11 * J22 - J12 * J21;
    }
  }
}

__global__ void face_geom_kernel(ExaDims P, const double* shapfgt, const int* perm, const double* xdg,
                                 double* faceg) {
  const int e = blockIdx.x;
  const int ngf = P.ngf, npf = P.npf, npe = P.npe, nd = P.nd, ncx = P.ncx;
  const double* x = xdg + (long long)e * npe * ncx;
  for (int t = threadIdx.x; t < ngf * P.nfe; t += blockDim.x) {
    const int g = t % ngf, l = t / ngf;
    double* out = faceg + ((long long)e * P.nfe + l) * P.faceg_stride();
    double* nl = out + ngf * ncx;
    double* jac = nl + ngf * nd;
    for (int c = 0; c < ncx; ++c) {
      double s = 0.0;
      for (int a = 0; a < npf; ++a) s += shapfgt[g + ngf * a] * x[perm[a + npf * l] + npe * c];
      out[g + ngf * c] = s;
    }
    if (nd == 1) {
      jac[g] = 1.0;
      nl[g] = (l % 2 == 0) ? -1.0 : 1.0;   // FaceGeom1D + FixNormal1D
      continue;
    }
    double T[3][2];  // T[c][r] = d x_c / d s_r along the face
    for (int c = 0; c < nd; ++c)
      for (int r = 0; r < nd - 1; ++r) {
        double s = 0.0;
        for (int a = 0; a < npf; ++a) s += shapfgt[g + ngf * a + ngf * npf * (1 + r)] * x[perm[a + npf * l] + npe * c];
        T[c][r] = s;
      }
    if (nd == 2) {
      const double Jx = T[0][0], Jy = T[1][0];
      const double j = sqrt(Jx * Jx + Jy * Jy);
      jac[g] = j;
      nl[g] = Jy / j;
      nl[g + ngf] = -Jx / j;
    } else {
      const double a1 = T[0][0], a2 = T[1][0], a3 = T[2][0];
      const double b1 = T[0][1], b2 = T[1][1], b3 = T[2][1];
      const double n1 = a2 * b3 - a3 * b2, n2 = a3 * b1 - a1 * b3, n3 = a1 * b2 - a2 * b1;
      const double j = sqrt(n1 * n1 + n2 * n2 + n3 * n3);
      jac[g] = j;
      nl[g] = n1 / j;
      nl[g + ngf] = n2 / j;
      nl[g + 2 * ngf] = n3 / j;
    }
  }
}

// ----------------------------------------------------------------------------------
// q-equation element matrices before the mass inverse (qequation.cpp:66-170, 255-338):
//   mass[a,b]      = sum_g (w0[a,g] t0[g,b]) jac[g]
//   cw[a,b,d]      = sum_r sum_g (w_{1+r}[a,g] t0[g,b]) Xx[g, d + nd r]   (terms added per r)
//   ew[perm[a,l], (b,l), d] = sum_g (wf0[a,g] tf0[g,b]) (nl_d[g] jac[g])
// ----------------------------------------------------------------------------------
__global__ void qmats_kernel(ExaDims P, const double* shapegt, const double* shapegw, const double* shapfgt,
                             const double* shapfgw, const int* perm, const double* elemg, const double* faceg,
                             double* mass, double* cw, double* ew) {
  const int e = blockIdx.x;
  const int npe = P.npe, nge = P.nge, nd = P.nd, npf = P.npf, ngf = P.ngf, ndf = P.ndf;
  const double* eg = elemg + (long long)e * P.elemg_stride();
  const double* Xx = eg + nge * P.ncx;
  const double* jac = Xx + nge * nd * nd;
  double* M = mass + (long long)e * npe * npe;
  double* C = cw + (long long)e * npe * npe * nd;
  double* E = ew + (long long)e * npe * ndf * nd;
  for (int t = threadIdx.x; t < npe * npe; t += blockDim.x) {
    const int a = t % npe, b = t / npe;
    double s = 0.0;
    for (int g = 0; g < nge; ++g) s += (shapegw[a + npe * g] * shapegt[g + nge * b]) * jac[g];
    M[t] = s;
    for (int d = 0; d < nd; ++d) {
      double acc = 0.0;
      for (int r = 0; r < nd; ++r) {
        double sr = 0.0;
        for (int g = 0; g < nge; ++g)
          sr += (shapegw[a + npe * g + npe * nge * (1 + r)] * shapegt[g + nge * b]) * Xx[g + nge * (d + nd * r)];
        acc = (r == 0) ? sr : acc + sr;
      }
      C[t + npe * npe * d] = acc;
    }
  }
  for (int t = threadIdx.x; t < npe * ndf * nd; t += blockDim.x) E[t] = 0.0;
  __syncthreads();
  for (int t = threadIdx.x; t < npf * npf * P.nfe * nd; t += blockDim.x) {
    const int a = t % npf, b = (t / npf) % npf, l = (t / (npf * npf)) % P.nfe, d = t / (npf * npf * P.nfe);
    const double* fg = faceg + ((long long)e * P.nfe + l) * P.faceg_stride();
    const double* nl = fg + ngf * P.ncx;
    const double* fj = nl + ngf * nd;
    double s = 0.0;
    for (int g = 0; g < ngf; ++g) s += (shapfgw[a + npf * g] * shapfgt[g + ngf * b]) * ((1.0 * nl[g + ngf * d]) * fj[g]);
    E[perm[a + npf * l] + npe * (b + npf * l) + npe * ndf * d] = s;
  }
}

// ----------------------------------------------------------------------------------
// trace-space gather / scatter and operators
// ----------------------------------------------------------------------------------
// w (face vector [ncu, npf, nf]) from element vectors we ([ncu, npf, nfe] per element):
// the face's first element writes, the second adds (interior faces only).
__global__ void scatter_kernel(ExaDims P, const int* f2e, const int* elemcon, const double* we, double* w) {
  const int ncu = P.ncu, npf = P.npf, m = P.m;
  const long long N = (long long)ncu * npf * P.nf;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N; idx += (long long)gridDim.x * blockDim.x) {
    const int k = idx % ncu;
    const long long q = idx / ncu;
    const int a = q % npf;
    const int f = q / npf;
    const int e1 = f2e[4 * f], l1 = f2e[4 * f + 1], e2 = f2e[4 * f + 2], l2 = f2e[4 * f + 3];
    double v = we[(long long)e1 * m + k + ncu * (a + npf * l1)];
    if (f < P.nf0 && e2 >= 0) {
      const int ii = elemcon[a + npf * l2 + P.ndf * e2] - npf * f;
      v += we[(long long)e2 * m + k + ncu * (ii + npf * l2)];
    }
    w[idx] = v;
  }
}

template <typename T>
__global__ void bj_build_kernel(ExaDims P, const int* f2e, const int* elemcon, const T* H, T* BE) {
  const int ncu = P.ncu, npf = P.npf, ncf = ncu * npf, m = P.m;
  const long long N = (long long)ncf * ncf * P.nf;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N; idx += (long long)gridDim.x * blockDim.x) {
    const int r = idx % ncf;
    const long long q = idx / ncf;
    const int c = q % ncf;
    const int f = q / ncf;
    const int e1 = f2e[4 * f], l1 = f2e[4 * f + 1], e2 = f2e[4 * f + 2], l2 = f2e[4 * f + 3];
    double v = (double)H[(long long)e1 * m * m + (r + ncf * l1) + (long long)m * (c + ncf * l1)];
    if (f < P.nf0 && e2 >= 0) {
      const int dm = r % ncu + ncu * (elemcon[r / ncu + npf * l2 + P.ndf * e2] - npf * f);
      const int dn = c % ncu + ncu * (elemcon[c / ncu + npf * l2 + P.ndf * e2] - npf * f);
      v += (double)H[(long long)e2 * m * m + (dm + ncf * l2) + (long long)m * (dn + ncf * l2)];
    }
    BE[idx] = (T)v;
  }
}

// elemental additive Schwarz: both elements of an interior face get the sum of their
// face blocks (kokkosimpl.h:1113-1143); BE starts as a copy of H.
template <typename T>
__global__ void eas_build_kernel(ExaDims P, const int* f2e, const int* elemcon, const T* H, T* BE) {
  const int ncu = P.ncu, npf = P.npf, ncf = ncu * npf, m = P.m;
  const long long N = (long long)ncf * ncf * P.nf;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N; idx += (long long)gridDim.x * blockDim.x) {
    const int r = idx % ncf;
    const long long q = idx / ncf;
    const int c = q % ncf;
    const int f = q / ncf;
    const int e1 = f2e[4 * f], l1 = f2e[4 * f + 1], e2 = f2e[4 * f + 2], l2 = f2e[4 * f + 3];
    if (e2 < 0) continue;
    const int dm = r % ncu + ncu * (elemcon[r / ncu + npf * l2 + P.ndf * e2] - npf * f);
    const int dn = c % ncu + ncu * (elemcon[c / ncu + npf * l2 + P.ndf * e2] - npf * f);
    const long long i1 = (long long)e1 * m * m + (r + ncf * l1) + (long long)m * (c + ncf * l1);
    const long long i2 = (long long)e2 * m * m + (dm + ncf * l2) + (long long)m * (dn + ncf * l2);
    const T tm = (T)((double)H[i1] + (double)H[i2]);
    BE[i1] = tm;
    BE[i2] = tm;
  }
}

template <typename T>
__global__ void bj_apply_kernel(ExaDims P, const T* BE, const double* x, double* y) {
  const int ncf = P.ncu * P.npf;
  const long long N = (long long)ncf * P.nf;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N; idx += (long long)gridDim.x * blockDim.x) {
    const int r = idx % ncf;
    const long long f = idx / ncf;
    const T* A = BE + f * ncf * ncf;
    const double* xf = x + f * ncf;
    double s = 0.0;
    for (int c = 0; c < ncf; ++c) s = fma((double)A[r + ncf * c], xf[c], s);
    y[idx] = s;
  }
}

// y_e = alpha A_e x_e + beta y0_e for a batch of column-major M x K blocks A_e (leading
// dimension M, batch stride sA; y0 may alias y).  x_e is read at x + e sx, or, with elemcon,
// gathered from a trace vector: x_e[k] = x[k % ncu + ncu elemcon[k / ncu + ndf e]].  One
// CTA per block: 8 warps split the columns (warp w takes c = w, w + 8, ...), CU at a time
// with the next CU loaded ahead (CU = 2 where 4 would not fit the registers); lane l keeps
// the partial sums of rows V l + 32 V i + v (i < RI, v < V) in registers, so each column is
// one coalesced load per 32 V rows (V = 2: pairs of floats, as many bytes per load as FP64);
// the 8 partial sums of a row meet in shared memory in a fixed order.  Serves the condensed matvec w_e = H_e gather(v)
// (hdgMatVec, matvec.cpp:240-389) and the additive-Schwarz apply, du = Ru + D^-1 F x
// (hdgGetDUDG, matvec.cpp:219-238) and the mixed form's Ru <- D^-1 Ru, Rh <- Rh - K Ru.
template <typename T, int RI, int V, int CU>
__global__ void __launch_bounds__(256) bgemv_kernel(int M, int K, const T* A, long long sA, const double* x,
                                                    long long sx, const int* elemcon, int ndf, int ncu,
                                                    double alpha, double beta, const double* y0, double* y,
                                                    long long sy) {
  static_assert(V == 1 || (V == 2 && sizeof(T) == 4), "pairs of floats only");
  extern __shared__ double sm[];
  double* xe = sm;         // [K]
  double* part = sm + K;   // [8][M]
  const long long e = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const T* Ae = A + e * sA;
  // rows V (lane + 32 i) .. + V - 1 of column c0 + 8 u; with V = 2, M is even, so a pair is
  // either inside the block or past it, and 8-byte aligned
  auto loadc = [&](int c0, T (&v)[CU][RI][V]) {
#pragma unroll
    for (int u = 0; u < CU; ++u) {
      const T* a = Ae + (long long)M * (c0 + 8 * u);
#pragma unroll
      for (int i = 0; i < RI; ++i) {
        const int r = V * (lane + 32 * i);
        if constexpr (V == 2) {
          const float2 t = r < M ? *reinterpret_cast<const float2*>(a + r) : make_float2(0.f, 0.f);
          v[u][i][0] = t.x;
          v[u][i][1] = t.y;
        } else {
          v[u][i][0] = r < M ? a[r] : T(0);
        }
      }
    }
  };
  int c = warp;
  T a[CU][RI][V];
  if (c + 8 * (CU - 1) < K) loadc(c, a);
  for (int k = threadIdx.x; k < K; k += blockDim.x)
    xe[k] = elemcon ? x[k % ncu + ncu * (long long)elemcon[k / ncu + (long long)ndf * e]] : x[e * sx + k];
  __syncthreads();
  double acc[RI][V];
#pragma unroll
  for (int i = 0; i < RI; ++i)
#pragma unroll
    for (int w = 0; w < V; ++w) acc[i][w] = 0.0;
  for (; c + 8 * (CU - 1) < K; c += 8 * CU) {
    T an[CU][RI][V];
    const bool more = c + 8 * CU + 8 * (CU - 1) < K;
    if (more) loadc(c + 8 * CU, an);
#pragma unroll
    for (int u = 0; u < CU; ++u) {
      const double xv = xe[c + 8 * u];
#pragma unroll
      for (int i = 0; i < RI; ++i)
#pragma unroll
        for (int w = 0; w < V; ++w) acc[i][w] = fma((double)a[u][i][w], xv, acc[i][w]);
    }
    if (more) {
#pragma unroll
      for (int u = 0; u < CU; ++u)
#pragma unroll
        for (int i = 0; i < RI; ++i)
#pragma unroll
          for (int w = 0; w < V; ++w) a[u][i][w] = an[u][i][w];
    }
  }
  for (; c < K; c += 8) {
    const T* a0 = Ae + (long long)M * c;
    const double xv = xe[c];
#pragma unroll
    for (int i = 0; i < RI; ++i) {
      const int r = V * (lane + 32 * i);
      if (r < M) {
#pragma unroll
        for (int w = 0; w < V; ++w) acc[i][w] = fma((double)a0[r + w], xv, acc[i][w]);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < RI; ++i)
#pragma unroll
    for (int w = 0; w < V; ++w) {
      const int r = V * (lane + 32 * i) + w;
      if (r < M) part[warp * M + r] = acc[i][w];
    }
  __syncthreads();
  for (int r = threadIdx.x; r < M; r += blockDim.x) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) s += part[w * M + r];
    const double prev = beta != 0.0 ? y0[e * sy + r] : 0.0;
    y[e * sy + r] = alpha * s + beta * prev;
  }
}

// The same product, persistent (for FP64 blocks): CTA b takes blocks b, b + gridDim.x, ...
// Per block, 8 warps split the columns
// (warp w takes c = w, w + 8, ...), CU at a time with the next CU loaded ahead (CU = 2 where 4
// would not fit the registers); lane l keeps the partial sums of rows V l + 32 V i + v
// (i < RI, v < V) in registers, so each column is one coalesced load per 32 V rows (V = 2:
// pairs of floats, as many bytes per load as FP64); the 8 partial sums of a row meet in shared
// memory in a fixed order.  The first columns of the CTA's next block and its gathered x
// (the other of two buffers) are loaded before the partial sums of the current one are
// reduced, so their latency overlaps that step.  Serves the condensed matvec
// w_e = H_e gather(v) (hdgMatVec, matvec.cpp:240-389) and the additive-Schwarz apply,
// du = Ru + D^-1 F x (hdgGetDUDG, matvec.cpp:219-238) and the mixed form's Ru <- D^-1 Ru,
// Rh <- Rh - K Ru.
template <typename T, int RI, int V, int CU>
__global__ void __launch_bounds__(256) bgemv_pers_kernel(int M, int K, int batch, const T* A, long long sA,
                                                    const double* x, long long sx, const int* elemcon, int ndf,
                                                    int ncu, double alpha, double beta, const double* y0, double* y,
                                                    long long sy) {
  static_assert(V == 1 || (V == 2 && sizeof(T) == 4), "pairs of floats only");
  extern __shared__ double sm[];
  double* xb = sm;             // [2][K]
  double* part = sm + 2 * K;   // [8][M]
  long long e = blockIdx.x;
  if (e >= batch) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // rows V (lane + 32 i) .. + V - 1 of column c0 + 8 u; with V = 2, M is even, so a pair is
  // either inside the block or past it, and 8-byte aligned
  auto loadc = [&](const T* Ae, int c0, T (&v)[CU][RI][V]) {
#pragma unroll
    for (int u = 0; u < CU; ++u) {
      const T* a = Ae + (long long)M * (c0 + 8 * u);
#pragma unroll
      for (int i = 0; i < RI; ++i) {
        const int r = V * (lane + 32 * i);
        if constexpr (V == 2) {
          const float2 t = r < M ? *reinterpret_cast<const float2*>(a + r) : make_float2(0.f, 0.f);
          v[u][i][0] = t.x;
          v[u][i][1] = t.y;
        } else {
          v[u][i][0] = r < M ? a[r] : T(0);
        }
      }
    }
  };
  auto gather = [&](long long eb, double* xe) {
    for (int k = threadIdx.x; k < K; k += blockDim.x)
      xe[k] = elemcon ? x[k % ncu + ncu * (long long)elemcon[k / ncu + (long long)ndf * eb]] : x[eb * sx + k];
  };
  int buf = 0;
  T a[CU][RI][V];
  if (warp + 8 * (CU - 1) < K) loadc(A + e * sA, warp, a);
  gather(e, xb);
  __syncthreads();
  for (;;) {
    const T* Ae = A + e * sA;
    const double* xe = xb + buf * K;
    double acc[RI][V];
#pragma unroll
    for (int i = 0; i < RI; ++i)
#pragma unroll
      for (int w = 0; w < V; ++w) acc[i][w] = 0.0;
    int c = warp;
    for (; c + 8 * (CU - 1) < K; c += 8 * CU) {
      T an[CU][RI][V];
      const bool more = c + 8 * CU + 8 * (CU - 1) < K;
      if (more) loadc(Ae, c + 8 * CU, an);
#pragma unroll
      for (int u = 0; u < CU; ++u) {
        const double xv = xe[c + 8 * u];
#pragma unroll
        for (int i = 0; i < RI; ++i)
#pragma unroll
          for (int w = 0; w < V; ++w) acc[i][w] = fma((double)a[u][i][w], xv, acc[i][w]);
      }
      if (more) {
#pragma unroll
        for (int u = 0; u < CU; ++u)
#pragma unroll
          for (int i = 0; i < RI; ++i)
#pragma unroll
            for (int w = 0; w < V; ++w) a[u][i][w] = an[u][i][w];
      }
    }
    for (; c < K; c += 8) {
      const T* a0 = Ae + (long long)M * c;
      const double xv = xe[c];
#pragma unroll
      for (int i = 0; i < RI; ++i) {
        const int r = V * (lane + 32 * i);
        if (r < M) {
#pragma unroll
          for (int w = 0; w < V; ++w) acc[i][w] = fma((double)a0[r + w], xv, acc[i][w]);
        }
      }
    }
    // the next block's first columns and x, in flight while this block's sums are reduced
    const long long en = e + gridDim.x;
    const bool next = en < batch;
    if (next) {
      if (warp + 8 * (CU - 1) < K) loadc(A + en * sA, warp, a);
      gather(en, xb + (buf ^ 1) * K);
    }
#pragma unroll
    for (int i = 0; i < RI; ++i)
#pragma unroll
      for (int w = 0; w < V; ++w) {
        const int r = V * (lane + 32 * i) + w;
        if (r < M) part[warp * M + r] = acc[i][w];
      }
    __syncthreads();
    for (int r = threadIdx.x; r < M; r += blockDim.x) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < 8; ++w) s += part[w * M + r];
      const double prev = beta != 0.0 ? y0[e * sy + r] : 0.0;
      y[e * sy + r] = alpha * s + beta * prev;
    }
    __syncthreads();  // part is rewritten and the other x buffer read next
    if (!next) break;
    e = en;
    buf ^= 1;
  }
}

// The same product for FP32 blocks streamed through shared memory: one CTA per block; a
// producer warp copies chunks of CW columns (contiguous in the column-major block) into a
// ring of BG_ST stages with cp.async.bulk, each completing on its stage's mbarrier by
// transaction count; 8 consumer warps split the rows (lane l of warp w keeps rows
// w rpw + l + 32 i) and run over every column of each chunk from shared memory, so no
// partial sums cross warps and the registers hold only the sums.  Two CTAs share an SM, so
// up to six 32 KB chunks are in flight per SM.  Every wait is bounded: one that runs out sets
// *flag to EXA_UMMA_TIMEOUT, the CTA skips the rest of its work and, before it exits, waits
// (bounded) for the copies it issued.
constexpr int BG_ST = 3, BG_STAGE_BYTES = 32768, BG_CONS = 256;

size_t bgemv_bulk_smem(int K) { return (size_t)BG_ST * BG_STAGE_BYTES + 8 * (size_t)K + 16 * BG_ST + 16; }

template <int RI>
__global__ void __launch_bounds__(BG_CONS + 32, 2)
    bgemv_bulk_kernel(int M, int K, int CW, const float* A, long long sA, const double* x, long long sx,
                      const int* elemcon, int ndf, int ncu, double alpha, double beta, const double* y0, double* y,
                      long long sy, int* flag) {
  using namespace exa_tc;
  extern __shared__ __align__(128) uint8_t bsm[];
  float* stage = reinterpret_cast<float*>(bsm);
  double* xe = reinterpret_cast<double*>(bsm + (size_t)BG_ST * BG_STAGE_BYTES);  // [K]
  uint64_t* full = reinterpret_cast<uint64_t*>(xe + K);
  uint64_t* empty = full + BG_ST;
  int* abort_flag = reinterpret_cast<int*>(empty + BG_ST);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long e = blockIdx.x;
  const int nch = (K + CW - 1) / CW;
  const float* Ae = A + e * sA;
  if (tid == 0) {
    for (int s = 0; s < BG_ST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], BG_CONS / 32);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  volatile int* ab = abort_flag;
  if (warp == BG_CONS / 32) {
    if (lane == 0) {
      int issued = 0;
      for (int q = 0; q < nch; ++q) {
        const int s = q % BG_ST;
        if (q >= BG_ST && (*ab || !mbar_wait(&empty[s], (uint32_t)((q / BG_ST - 1) & 1)))) {
          *ab = 1;
          break;
        }
        const int c0 = q * CW, ncol = min(CW, K - c0);
        const uint32_t bytes = (uint32_t)M * ncol * 4;
        mbar_expect_tx(&full[s], bytes);
        bulk_g2s(stage + (size_t)s * (BG_STAGE_BYTES / 4), Ae + (long long)c0 * M, bytes, &full[s]);
        issued = q + 1;
      }
      // copies still in flight (only after an abort): their stages' latest phases
      for (int q = max(0, issued - BG_ST); q < issued; ++q) mbar_wait(&full[q % BG_ST], (uint32_t)((q / BG_ST) & 1));
    }
  } else {
    for (int k = tid; k < K; k += BG_CONS)
      xe[k] = elemcon ? x[k % ncu + ncu * (long long)elemcon[k / ncu + (long long)ndf * e]] : x[e * sx + k];
    asm volatile("bar.sync 1, %0;" ::"n"(BG_CONS) : "memory");
    const int rpw = (M + 7) / 8, r0 = warp * rpw, r1 = min(M, r0 + rpw);
    double acc[RI];
#pragma unroll
    for (int i = 0; i < RI; ++i) acc[i] = 0.0;
    for (int q = 0; q < nch; ++q) {
      const int s = q % BG_ST;
      if (!*ab && !mbar_wait(&full[s], (uint32_t)((q / BG_ST) & 1))) *ab = 1;
      if (!*ab) {
        const float* S = stage + (size_t)s * (BG_STAGE_BYTES / 4);
        const int c0 = q * CW, ncol = min(CW, K - c0);
        for (int cc = 0; cc < ncol; ++cc) {
          const double xv = xe[c0 + cc];
          const float* col = S + (size_t)cc * M;
#pragma unroll
          for (int i = 0; i < RI; ++i) {
            const int r = r0 + lane + 32 * i;
            if (r < r1) acc[i] = fma((double)col[r], xv, acc[i]);
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
    if (!*ab) {
#pragma unroll
      for (int i = 0; i < RI; ++i) {
        const int r = r0 + lane + 32 * i;
        if (r < r1) {
          const double prev = beta != 0.0 ? y0[e * sy + r] : 0.0;
          y[e * sy + r] = alpha * acc[i] + beta * prev;
        }
      }
    }
  }
  __syncthreads();
  if (tid == 0 && *ab) atomicExch(flag, EXA_UMMA_TIMEOUT);
}

// columns per chunk for the streamed kernel: at most one stage, with every chunk's bytes and
// start a multiple of 16; 0 where no such split exists (the register kernel serves those)
int bgemv_bulk_cw(int M, int K, long long sA) {
  // one CTA per block: the ring only pays where a block fills it several times.  The FP32
  // matvec of 3D Euler (480 x 480, 0.9 MB) went from 230 to 181 ms per 32^3 solve; that of
  // the 3D convection-diffusion case (150 x 150, 90 KB) from 1.96 to 2.12 ms per solve, so
  // blocks under 256 KB keep the register kernel
  if (M <= 0 || K <= 0 || M > 512 || sA % 4 != 0 || (long long)M * K < 65536) return 0;
  for (int cw = std::min(K, BG_STAGE_BYTES / (4 * M)); cw >= 1; --cw) {
    const int rem = K % cw;
    if ((M * cw) % 4 == 0 && (M * rem) % 4 == 0) return cw;
  }
  return 0;
}

int launch_bgemv_bulk(int M, int K, int cw, int batch, const float* A, long long sA, const double* x, long long sx,
                      const int* elemcon, int ndf, int ncu, double alpha, double beta, const double* y0, double* y,
                      long long sy, int* flag, cudaStream_t st) {
  const size_t smem = bgemv_bulk_smem(K);
  const int ri = ((M + 7) / 8 + 31) / 32;
  if (ri <= 1) {
    EXA_TRY(exa_allow_smem((const void*)bgemv_bulk_kernel<1>, smem));
    bgemv_bulk_kernel<1><<<batch, BG_CONS + 32, smem, st>>>(M, K, cw, A, sA, x, sx, elemcon, ndf, ncu, alpha, beta,
                                                            y0, y, sy, flag);
  } else {
    EXA_TRY(exa_allow_smem((const void*)bgemv_bulk_kernel<2>, smem));
    bgemv_bulk_kernel<2><<<batch, BG_CONS + 32, smem, st>>>(M, K, cw, A, sA, x, sx, elemcon, ndf, ncu, alpha, beta,
                                                            y0, y, sy, flag);
  }
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

// CTAs of a persistent batched-gemv launch: the blocks per SM that the instance's registers
// and shared memory allow (cached per instance, device and shared-memory size) times the SMs
int bgemv_grid(const void* kern, size_t smem, int batch) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, size_t>, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return batch;
  int per = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find({kern, dev, smem});
    if (it != cache.end()) per = it->second;
  }
  if (per == 0) {
    int sms = 0, occ = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, smem) != cudaSuccess || occ <= 0 || sms <= 0)
      return batch;  // one CTA per block
    per = occ * sms;
    std::lock_guard<std::mutex> lk(mu);
    cache[{kern, dev, smem}] = per;
  }
  return batch < per ? batch : per;
}

template <typename T>
int launch_bgemv(int M, int K, int batch, const T* A, long long sA, const double* x, long long sx,
                 const int* elemcon, int ndf, int ncu, double alpha, double beta, const double* y0, double* y,
                 long long sy, cudaStream_t st, int* flag = nullptr) {
  if (batch <= 0 || M <= 0) return EXA_OK;
  if (M > 512 || K > 512) {
    exa_set_error("batched gemv: blocks of %d x %d exceed 512 x 512", M, K);
    return EXA_ERR_UNSUPPORTED;
  }
  if constexpr (sizeof(T) == 4) {
    // FP32 blocks stream through shared memory where a flag for the bounded waits is given,
    // the blocks start on 16-byte boundaries and a chunking exists
    const int cw = flag ? bgemv_bulk_cw(M, K, sA) : 0;
    if (cw > 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0)
      return launch_bgemv_bulk(M, K, cw, batch, A, sA, x, sx, elemcon, ndf, ncu, alpha, beta, y0, y, sy, flag, st);
  }
  const size_t smem = sizeof(double) * (2 * (size_t)(K > 0 ? K : 1) + 8 * (size_t)M);
  const size_t smem1 = sizeof(double) * ((size_t)(K > 0 ? K : 1) + 8 * (size_t)M);
  // FP64 blocks persistent (bgemv_pers_kernel): as many CTAs as fit on the device at once (the
  // occupancy of the instance, taken once per instance and device).  FP32 blocks one CTA per
  // block (bgemv_kernel): their blocks are half the bytes, and the persistent form was slower
  // for them (0.104 against 0.096 ms per matvec of the benchmark workload; 0.140 against 0.145
  // ms for its FP64 blocks)
#define EXA_BGEMV(R, V)                                                                                     \
  do {                                                                                                      \
    if constexpr (sizeof(T) == 8) {                                                                         \
      auto kern = bgemv_pers_kernel<T, R, V, (R > 12) ? 2 : 4>;                                               \
      const int g = bgemv_grid((const void*)kern, smem, batch);                                             \
      kern<<<g, 256, smem, st>>>(M, K, batch, A, sA, x, sx, elemcon, ndf, ncu, alpha, beta, y0, y, sy);    \
    } else {                                                                                                \
      bgemv_kernel<T, R, V, 4><<<batch, 256, smem1, st>>>(M, K, A, sA, x, sx, elemcon, ndf, ncu, alpha, beta, \
                                                          y0, y, sy);                                         \
    }                                                                                                       \
  } while (0)
  // rows covered per warp with single rows (RI from 1-6, 8, 10, 12, 16) and with pairs (RI from
  // 1-6, 8): pairs only where they pad no more rows (m = 150: 160 single against 192 paired)
  auto inst = [](int r, bool pairs) {
    const int lim[] = {1, 2, 3, 4, 5, 6, 8, 10, 12, 16};
    for (int v : lim)
      if (v >= r && (!pairs || v <= 8)) return v;
    return pairs ? 8 : 16;
  };
  const bool pairs = sizeof(T) == 4 && M % 2 == 0 && 64 * inst((M + 63) / 64, true) <= 32 * inst((M + 31) / 32, false);
  if (pairs) {
    if constexpr (sizeof(T) == 4) {
      // pairs of rows per lane: ceil(M / 64) pairs
      const int ri = (M + 63) / 64;
      if (ri <= 1) EXA_BGEMV(1, 2);
      else if (ri <= 2) EXA_BGEMV(2, 2);
      else if (ri <= 3) EXA_BGEMV(3, 2);
      else if (ri <= 4) EXA_BGEMV(4, 2);
      else if (ri <= 5) EXA_BGEMV(5, 2);
      else if (ri <= 6) EXA_BGEMV(6, 2);
      else EXA_BGEMV(8, 2);
    }
  } else {
    const int ri = (M + 31) / 32;
    if (ri <= 1) EXA_BGEMV(1, 1);
    else if (ri <= 2) EXA_BGEMV(2, 1);
    else if (ri <= 3) EXA_BGEMV(3, 1);
    else if (ri <= 4) EXA_BGEMV(4, 1);
    else if (ri <= 5) EXA_BGEMV(5, 1);
    else if (ri <= 6) EXA_BGEMV(6, 1);
    else if (ri <= 8) EXA_BGEMV(8, 1);
    else if (ri <= 10) EXA_BGEMV(10, 1);
    else if (ri <= 12) EXA_BGEMV(12, 1);
    else EXA_BGEMV(16, 1);
  }
#undef EXA_BGEMV
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

__global__ void udg_update_kernel(ExaDims P, double* udg, const double* du, double alpha) {
  const long long N = (long long)P.n * P.ne;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N; idx += (long long)gridDim.x * blockDim.x) {
    const long long e = idx / P.n;
    const int ik = idx % P.n;  // i + npe*k
    udg[ik + (long long)P.npe * P.nc * e] += alpha * du[idx];
  }
}

// q = MinvC u - MinvE uhat per dimension (qequation.cpp:372-470)
__global__ void getq_kernel(ExaDims P, const int* elemcon, const double* MC, const double* ME, const double* uh,
                            double* udg) {
  extern __shared__ double sm[];
  const int e = blockIdx.x, npe = P.npe, ncu = P.ncu, ndf = P.ndf, nd = P.nd, nc = P.nc;
  double* u = sm;               // [npe, ncu]
  double* uhe = sm + npe * ncu; // [ndf, ncu]
  double* U = udg + (long long)e * npe * nc;
  for (int t = threadIdx.x; t < npe * ncu; t += blockDim.x) u[t] = U[t];
  for (int t = threadIdx.x; t < ndf * ncu; t += blockDim.x) {
    const int jf = t % ndf, k = t / ndf;
    uhe[t] = uh[k + ncu * (long long)elemcon[jf + ndf * e]];
  }
  __syncthreads();
  const double* C = MC + (long long)e * npe * npe * nd;
  const double* E = ME + (long long)e * npe * ndf * nd;
  for (int t = threadIdx.x; t < npe * ncu * nd; t += blockDim.x) {
    const int i = t % npe, k = (t / npe) % ncu, d = t / (npe * ncu);
    double s = 0.0;
    const double* Cd = C + i + npe * d;
    const double* Ed = E + i + npe * d;
    const int ld = npe * nd;
    for (int j = 0; j < npe; ++j) s = fma(Cd[ld * j], u[j + npe * k], s);
    double r = 0.0;
    for (int j = 0; j < ndf; ++j) r = fma(Ed[ld * j], uhe[j + ndf * k], r);
    U[i + npe * (ncu + k + ncu * d)] = s - r;
  }
}

// The same q without MinvC and MinvE: q_d = Minv (C_d u - E_d uhat), with C_d u and E_d uhat
// by quadrature (the sums that define C and E in qmats_kernel, taken over the Gauss points of
// u and uhat instead of stored as matrices), so each element reads its 125 KB Minv (p = 4 hex)
// instead of 825 KB of MinvC and MinvE.  One block per element.
//
// With wpre set, C_d u comes from there (w of element e at wpre + e npe ncu nd, computed for all
// elements by two GEMMs, exa_k_getq_gemm) and the block does the face terms and Minv only.
//
// The face terms of all faces are formed at once; each element node then subtracts the terms
// of the faces it lies on in increasing face order, the order of a face-by-face update.
__host__ __device__ inline size_t getq_mf_doubles(const ExaDims& P, bool wpre) {
  const size_t own = (size_t)P.ndf * P.ncu + (size_t)P.npe * P.ncu * P.nd + (size_t)P.ngf * P.nd * P.ncu * P.nfe +
                     (size_t)P.ndf * P.ncu * P.nd;
  return own + (wpre ? 0 : (size_t)P.npe * P.ncu + (size_t)P.nge * P.nd * P.nd * P.ncu);
}
__host__ __device__ inline size_t getq_mf_ints(const ExaDims& P) { return (size_t)P.ndf + (size_t)P.npe * (P.nfe + 1); }

__global__ void __launch_bounds__(128, 8) getq_mf_kernel(ExaDims P, const double* shapegt, const double* shapegw, const double* shapfgt,
                               const double* shapfgw, const int* perm, const int* elemcon, const double* elemg,
                               const double* faceg, const double* Minv, const double* uh, double* udg,
                               const double* wpre) {
  extern __shared__ double sm[];
  const int e = blockIdx.x, npe = P.npe, ncu = P.ncu, ndf = P.ndf, nd = P.nd, nc = P.nc;
  const int nge = P.nge, npf = P.npf, ngf = P.ngf, nfe = P.nfe;
  double* uhe = sm;                      // [ndf, ncu]
  double* w = uhe + ndf * ncu;           // [npe, ncu, nd]
  double* hg = w + npe * ncu * nd;       // [ngf, nd, ncu, nfe]: n_d fj uhat(g) on every face
  double* hs = hg + ngf * nd * ncu * nfe;  // [ndf, ncu, nd]: E_d uhat of each face node
  double* u = hs + ndf * ncu * nd;       // [npe, ncu]                      (without wpre)
  double* vg = u + npe * ncu;            // [nge, nd (ref r), nd (phys d), ncu]: Xx[g, d, r] u(g)
  int* sperm = reinterpret_cast<int*>(sm + getq_mf_doubles(P, wpre != nullptr));  // [ndf]
  int* ntab = sperm + ndf;               // [npe, 1 + nfe]: count, then face-node slots a + npf l
  double* U = udg + (long long)e * npe * nc;
  const double* eg = elemg + (long long)e * P.elemg_stride();
  const double* Xx = eg + nge * P.ncx;
  for (int t = threadIdx.x; t < ndf * ncu; t += blockDim.x) {
    const int jf = t % ndf, k = t / ndf;
    uhe[t] = uh[k + ncu * (long long)elemcon[jf + ndf * e]];
  }
  for (int t = threadIdx.x; t < ndf; t += blockDim.x) sperm[t] = perm[t];
  {
    // the element's Minv is streamed last, after the face terms: ask for it in L2 now, one
    // 128-byte line per request, so its DRAM reads overlap the face phase
    const char* mb = reinterpret_cast<const char*>(Minv + (long long)e * npe * npe);
    const long long bytes = (long long)npe * npe * (long long)sizeof(double);
    for (long long o = 128LL * threadIdx.x; o < bytes; o += 128LL * blockDim.x)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(mb + o));
  }
  if (wpre) {
    const double* we = wpre + (long long)e * npe * ncu * nd;
    for (int t = threadIdx.x; t < npe * ncu * nd; t += blockDim.x) w[t] = we[t];
  } else {
    for (int t = threadIdx.x; t < npe * ncu; t += blockDim.x) u[t] = U[t];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < npe; i += blockDim.x) {
    int n = 0;
    for (int t = 0; t < ndf; ++t)
      if (sperm[t] == i && n < nfe) ntab[i * (1 + nfe) + 1 + n++] = t;
    ntab[i * (1 + nfe)] = n;
  }
  if (!wpre) {
    for (int t = threadIdx.x; t < nge * ncu; t += blockDim.x) {
      const int g = t % nge, k = t / nge;
      double s = 0.0;
      for (int b = 0; b < npe; ++b) s = fma(shapegt[g + nge * b], u[b + npe * k], s);
      for (int d = 0; d < nd; ++d)
        for (int r = 0; r < nd; ++r) vg[g + nge * (r + nd * (d + nd * k))] = Xx[g + nge * (d + nd * r)] * s;
    }
    __syncthreads();
    // C_d u: sum over g and r of shapegw[a, g, 1 + r] vg[g, r, d]; one thread per (a, k) takes
    // every d, so each shapegw entry is loaded once for the nd products that use it
    for (int t = threadIdx.x; t < npe * ncu; t += blockDim.x) {
      const int a = t % npe, k = t / npe;
      double s[3] = {0.0, 0.0, 0.0};
      for (int r = 0; r < nd; ++r) {
        const double* W = shapegw + a + (long long)npe * nge * (1 + r);
        const double* v = vg + nge * (r + nd * nd * k);
        for (int g = 0; g < nge; ++g) {
          const double wv = W[npe * g];
#pragma unroll
          for (int d = 0; d < 3; ++d)
            if (d < nd) s[d] = fma(wv, v[g + nge * nd * d], s[d]);
        }
      }
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d < nd) w[a + npe * (k + ncu * d)] = s[d];
    }
  }
  // E_d uhat: uhat at the Gauss points of every face, then its weighted sums at the face nodes
  for (int t = threadIdx.x; t < ngf * ncu * nfe; t += blockDim.x) {
    const int g = t % ngf, k = (t / ngf) % ncu, l = t / (ngf * ncu);
    const double* fg = faceg + ((long long)e * nfe + l) * P.faceg_stride();
    const double* nl = fg + ngf * P.ncx;
    const double* fj = nl + ngf * nd;
    double s = 0.0;
    for (int b = 0; b < npf; ++b) s = fma(shapfgt[g + ngf * b], uhe[b + npf * l + ndf * k], s);
    for (int d = 0; d < nd; ++d) hg[g + ngf * (d + nd * (k + ncu * l))] = nl[g + ngf * d] * fj[g] * s;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < npf * ncu * nd * nfe; t += blockDim.x) {
    const int a = t % npf, k = (t / npf) % ncu, d = (t / (npf * ncu)) % nd, l = t / (npf * ncu * nd);
    double s = 0.0;
    for (int g = 0; g < ngf; ++g) s = fma(shapfgw[a + npf * g], hg[g + ngf * (d + nd * (k + ncu * l))], s);
    hs[a + npf * l + ndf * (k + ncu * d)] = s;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < npe * ncu * nd; t += blockDim.x) {
    const int i = t % npe, kd = t / npe;
    const int* nt = ntab + i * (1 + nfe);
    double v = w[t];
    for (int c = 1; c <= nt[0]; ++c) v -= hs[nt[c] + ndf * kd];
    w[t] = v;
  }
  __syncthreads();
  // q = Minv w: one thread per (row i, group of up to 8 of the ncu nd right-hand sides), so
  // each Minv entry is read once per 8 products; eight columns of Minv are loaded at a time
  const double* Mi = Minv + (long long)e * npe * npe;
  const int nq = ncu * nd, ngrp = (nq + 7) / 8;
  for (int t = threadIdx.x; t < npe * ngrp; t += blockDim.x) {
    const int i = t % npe, q0 = 8 * (t / npe);
    double s[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) s[q] = 0.0;
    const double* Mr = Mi + i;
    int j = 0;
    for (; j + 8 <= npe; j += 8) {
      double m[8];
#pragma unroll
      for (int x = 0; x < 8; ++x) m[x] = __ldcs(Mr + (long long)npe * (j + x));
#pragma unroll
      for (int x = 0; x < 8; ++x)
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (q0 + q < nq) s[q] = fma(m[x], w[j + x + npe * (q0 + q)], s[q]);
    }
    for (; j < npe; ++j) {
      const double m = __ldcs(Mr + (long long)npe * j);
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (q0 + q < nq) s[q] = fma(m, w[j + npe * (q0 + q)], s[q]);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if (q0 + q < nq) U[i + npe * (ncu + q0 + q)] = s[q];
  }
}

// V[g + nge r, k + ncu (d + nd e)] = Xx_e[g, d, r] UG[g + nge (e + ne k)]: the Gauss-point
// values of u_k times the geometric factors, the right operand of C_d u for all elements
__global__ void getq_v_kernel(ExaDims P, const double* elemg, const double* UG, double* V) {
  const int nge = P.nge, nd = P.nd, ncu = P.ncu;
  const long long ne = P.ne, K = (long long)nge * nd;
  const long long total = K * nd * ncu * ne;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long col = idx / K;
    const int row = (int)(idx - col * K);
    const int g = row % nge, r = row / nge;
    const int k = (int)(col % ncu);
    const long long de = col / ncu;
    const int d = (int)(de % nd);
    const long long e = de / nd;
    const double* Xx = elemg + e * P.elemg_stride() + (long long)nge * P.ncx;
    V[idx] = Xx[g + nge * (d + nd * r)] * UG[g + nge * (e + ne * k)];
  }
}

// uh from the first element of each face (kokkosimpl.h:901-915)
__global__ void face_nodes_kernel(ExaDims P, const int* f2e, const int* perm, const double* udg, double* uh) {
  const long long N = (long long)P.ncu * P.npf * P.nf;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N; idx += (long long)gridDim.x * blockDim.x) {
    const int k = idx % P.ncu;
    const long long q = idx / P.ncu;
    const int a = q % P.npf;
    const int f = q / P.npf;
    const int e1 = f2e[4 * f], l1 = f2e[4 * f + 1];
    uh[idx] = udg[perm[a + P.npf * l1] + P.npe * k + (long long)P.npe * P.nc * e1];
  }
}

int grid_for(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

}  // namespace

int exa_k_geometry(const ExaDims& P, const double* shapegt, const double* shapfgt, const int* perm,
                   const double* xdg, double* elemg, double* faceg, cudaStream_t st) {
  elem_geom_kernel<<<P.ne, 128, 0, st>>>(P, shapegt, xdg, elemg);
  EXA_LAUNCH_CHECK();
  face_geom_kernel<<<P.ne, 128, 0, st>>>(P, shapfgt, perm, xdg, faceg);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_k_qmats(const ExaDims& P, const double* shapegt, const double* shapegw, const double* shapfgt,
                const double* shapfgw, const int* perm, const double* elemg, const double* faceg, double* mass,
                double* cw, double* ew, cudaStream_t st) {
  qmats_kernel<<<P.ne, 256, 0, st>>>(P, shapegt, shapegw, shapfgt, shapfgw, perm, elemg, faceg, mass, cw, ew);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_k_scatter(const ExaDims& P, const int* f2e, const int* elemcon, const double* we, double* w, cudaStream_t st) {
  scatter_kernel<<<grid_for((long long)P.ncu * P.npf * P.nf), 256, 0, st>>>(P, f2e, elemcon, we, w);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

template <typename T>
int exa_k_elem_matvec(const ExaDims& P, const int* elemcon, const T* A, const double* v, double* we,
                      cudaStream_t st, int* flag) {
  // we_e = A_e gather(v): A_e = H (matvec) or the additive-Schwarz inverse blocks
  return launch_bgemv<T>(P.m, P.m, P.ne, A, (long long)P.m * P.m, v, 0, elemcon, P.ndf, P.ncu, 1.0, 0.0, nullptr, we,
                         P.m, st, flag);
}

template <typename T>
int exa_k_bj_build(const ExaDims& P, const int* f2e, const int* elemcon, const T* H, T* BE, cudaStream_t st) {
  const long long ncf = (long long)P.ncu * P.npf;
  bj_build_kernel<<<grid_for(ncf * ncf * P.nf), 256, 0, st>>>(P, f2e, elemcon, H, BE);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

template <typename T>
int exa_k_eas_build(const ExaDims& P, const int* f2e, const int* elemcon, const T* H, T* BE, cudaStream_t st) {
  EXA_CUDA(cudaMemcpyAsync(BE, H, sizeof(T) * (size_t)P.m * P.m * P.ne, cudaMemcpyDeviceToDevice, st));
  const long long ncf = (long long)P.ncu * P.npf;
  eas_build_kernel<<<grid_for(ncf * ncf * P.nf), 256, 0, st>>>(P, f2e, elemcon, H, BE);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

template <typename T>
int exa_k_bj_apply(const ExaDims& P, const T* BE, const double* x, double* y, cudaStream_t st) {
  bj_apply_kernel<<<grid_for((long long)P.ncu * P.npf * P.nf), 256, 0, st>>>(P, BE, x, y);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

template <typename T>
int exa_k_dudg(const ExaDims& P, const int* elemcon, const T* DinvF, const double* Ru, const double* x,
               double* du, cudaStream_t st, int* flag) {
  // du_e = Ru_e + DinvF_e gather(x)
  return launch_bgemv<T>(P.n, P.m, P.ne, DinvF, (long long)P.n * P.m, x, 0, elemcon, P.ndf, P.ncu, 1.0, 1.0, Ru, du,
                         P.n, st, flag);
}

int exa_k_udg_update(const ExaDims& P, double* udg, const double* du, double alpha, cudaStream_t st) {
  udg_update_kernel<<<grid_for((long long)P.n * P.ne), 256, 0, st>>>(P, udg, du, alpha);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_k_getq(const ExaDims& P, const int* elemcon, const double* MC, const double* ME, const double* uh,
               double* udg, cudaStream_t st) {
  size_t smem = sizeof(double) * ((size_t)P.npe * P.ncu + (size_t)P.ndf * P.ncu);
  getq_kernel<<<P.ne, 128, smem, st>>>(P, elemcon, MC, ME, uh, udg);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

size_t exa_getq_mf_smem(const ExaDims& P, bool wpre) {
  return sizeof(double) * getq_mf_doubles(P, wpre) + sizeof(int) * getq_mf_ints(P);
}

int exa_k_getq_mf(const ExaDims& P, const double* shapegt, const double* shapegw, const double* shapfgt,
                  const double* shapfgw, const int* perm, const int* elemcon, const double* elemg,
                  const double* faceg, const double* Minv, const double* uh, double* udg, cudaStream_t st,
                  const double* wpre) {
  const size_t smem = exa_getq_mf_smem(P, wpre != nullptr);
  EXA_TRY(exa_allow_smem((const void*)getq_mf_kernel, smem));
  getq_mf_kernel<<<P.ne, 128, smem, st>>>(P, shapegt, shapegw, shapfgt, shapfgw, perm, elemcon, elemg, faceg, Minv,
                                          uh, udg, wpre);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_k_getq_gemm(const ExaDims& P, const double* shapegt, const double* shapegw, const double* elemg,
                    const double* udg, double* UG, double* V, double* W, cudaStream_t st) {
  if (P.ne <= 0 || P.ncq == 0) return EXA_OK;
  GemmBatch g{};
  // UG[:, e + ne k] = shapegt (nge x npe) u_k of element e
  g.M = P.nge; g.N = P.ne; g.K = P.npe; g.alpha = 1.0; g.beta = 0.0;
  g.A = shapegt; g.lda = P.nge;
  g.B = udg; g.ldb = (long long)P.npe * P.nc; g.sB = P.npe;
  g.C = UG; g.ldc = P.nge; g.sC = (long long)P.nge * P.ne;
  g.batch = P.ncu; g.batch2 = 1;
  EXA_TRY(exa_gemm(g, st));
  const long long nv = (long long)P.nge * P.nd * P.nd * P.ncu * P.ne;
  getq_v_kernel<<<grid_for(nv), 256, 0, st>>>(P, elemg, UG, V);
  EXA_LAUNCH_CHECK();
  // W[:, k + ncu (d + nd e)] = shapegw[:, :, 1..nd] (npe x nge nd) V: C_d u of every element
  GemmBatch h{};
  h.M = P.npe; h.N = P.ncu * P.nd * P.ne; h.K = P.nge * P.nd; h.alpha = 1.0; h.beta = 0.0;
  h.A = shapegw + (long long)P.npe * P.nge; h.lda = P.npe;
  h.B = V; h.ldb = (long long)P.nge * P.nd;
  h.C = W; h.ldc = P.npe;
  h.batch = 1; h.batch2 = 1;
  return exa_gemm(h, st);
}

int exa_k_face_nodes(const ExaDims& P, const int* f2e, const int* perm, const double* udg, double* uh, cudaStream_t st) {
  face_nodes_kernel<<<grid_for((long long)P.ncu * P.npf * P.nf), 256, 0, st>>>(P, f2e, perm, udg, uh);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

namespace {
__global__ void to_f32_kernel(const double* x, float* y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}
}  // namespace

int exa_k_gemv32(int M, int K, int batch, double alpha, const float* A, long long sA, const double* x, long long sx,
                 double beta, double* y, long long sy, cudaStream_t st, int* flag) {
  return launch_bgemv<float>(M, K, batch, A, sA, x, sx, nullptr, 0, 1, alpha, beta, y, y, sy, st, flag);
}

int exa_k_to_f32(const double* x, float* y, long long n, cudaStream_t st) {
  if (n <= 0) return EXA_OK;
  to_f32_kernel<<<grid_for(n), 256, 0, st>>>(x, y, n);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

// block arrays in FP64 (plain form) and FP32 (mixed-precision form)
#define EXA_INST_BLOCK_KERNELS(T)                                                                              \
  template int exa_k_elem_matvec<T>(const ExaDims&, const int*, const T*, const double*, double*, cudaStream_t, \
                                    int*);                                                                     \
  template int exa_k_bj_build<T>(const ExaDims&, const int*, const int*, const T*, T*, cudaStream_t);           \
  template int exa_k_eas_build<T>(const ExaDims&, const int*, const int*, const T*, T*, cudaStream_t);          \
  template int exa_k_bj_apply<T>(const ExaDims&, const T*, const double*, double*, cudaStream_t);              \
  template int exa_k_dudg<T>(const ExaDims&, const int*, const T*, const double*, const double*, double*, cudaStream_t, \
                             int*);
EXA_INST_BLOCK_KERNELS(double)
EXA_INST_BLOCK_KERNELS(float)

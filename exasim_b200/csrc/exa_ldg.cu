// The model-independent kernels of the LDG residual: the face-node table of both sides, the
// sum of the face residuals into the elements, and the combination of residuals that forms a
// Jacobian-vector product by differences.
#include "exa_common.cuh"
#include "exa_kernels.cuh"

namespace {

// fcon[2 g + s] = e npe + node for face node g = f npf + i (side 1's order) on side s: the
// side of element e's local face l is 1 when (e, l) is the face's first element and face
// (the facecon of connectivity.cpp, built from f2e, perm and elemcon)
__global__ void ldg_fcon_kernel(ExaDims P, const int* f2e, const int* perm, const int* elemcon, int* fcon) {
  const long long total = (long long)P.ndf * P.ne;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int jf = (int)(t % P.ndf), e = (int)(t / P.ndf);
    const int a = jf % P.npf, l = jf / P.npf;
    const int g = elemcon[t];
    const int f = g / P.npf;
    const int side = (f2e[4 * f] == e && f2e[4 * f + 1] == l) ? 0 : 1;
    fcon[2LL * g + side] = e * P.npe + perm[a + P.npf * l];
  }
}

__global__ void ldg_fcon_boundary_kernel(ExaDims P, const int* f2e, int* fcon) {
  const long long total = (long long)P.npf * P.nf;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long f = t / P.npf;
    if (f2e[4 * f + 2] < 0) fcon[2 * t + 1] = fcon[2 * t];
  }
}

// Ru of element e: its volume residual, minus the face residuals of the faces it is the first
// element of and plus those of the others, face by face in the order of its local faces
// (PutFaceNodes, kokkosimpl.h:1575-1603); then Ru <- -Ru and, time-dependent, Ru <- Ru / dtfactor
// (Residual, residual.cpp:604-610).  One block per element.
__global__ void ldg_gather_kernel(ExaDims P, const int* f2e, const int* perm, const int* elemcon, const double* Rue,
                                  const double* Rh, double* Ru, int tdep, double dtfactor) {
  extern __shared__ double acc[];  // [npe, ncu]
  const int e = blockIdx.x, npe = P.npe, ncu = P.ncu, npf = P.npf, ndf = P.ndf;
  const long long base = (long long)e * npe * ncu;
  for (int t = threadIdx.x; t < npe * ncu; t += blockDim.x) acc[t] = Rue[base + t];
  __syncthreads();
  for (int l = 0; l < P.nfe; ++l) {
    for (int t = threadIdx.x; t < npf * ncu; t += blockDim.x) {
      const int a = t % npf, k = t / npf;
      const int g = elemcon[a + npf * l + (long long)ndf * e];
      const int f = g / npf, i = g - f * npf;
      const double r = Rh[i + (long long)npf * (k + (long long)ncu * f)];
      const int node = perm[a + npf * l];
      if (f2e[4 * f] == e && f2e[4 * f + 1] == l)
        acc[node + npe * k] -= r;
      else
        acc[node + npe * k] += r;
    }
    __syncthreads();
  }
  const double s = 1.0 / dtfactor;
  for (int t = threadIdx.x; t < npe * ncu; t += blockDim.x) {
    double v = -1.0 * acc[t];
    if (tdep) v = s * v;
    Ru[base + t] = v;
  }
}

// The element mass matrices M[a, b] = sum_g shapegw[a, g] shapegt[g, b] jac[g] (the sums of
// qmats_kernel), for the LDG preconditioner's mass inverse
__global__ void ldg_mass_kernel(ExaDims P, const double* shapegt, const double* shapegw, const double* elemg,
                                double* mass) {
  const int e = blockIdx.x, npe = P.npe, nge = P.nge;
  const double* jac = elemg + (long long)e * P.elemg_stride() + nge * (P.ncx + P.nd * P.nd);
  double* M = mass + (long long)e * npe * npe;
  for (int t = threadIdx.x; t < npe * npe; t += blockDim.x) {
    const int a = t % npe, b = t / npe;
    double s = 0.0;
    for (int g = 0; g < nge; ++g) s += (shapegw[a + npe * g] * shapegt[g + nge * b]) * jac[g];
    M[t] = s;
  }
}

__global__ void lincomb_kernel(double* out, double a, const double* x, double b, const double* y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = a * x[i] + b * y[i];
}

int blocks_for(long long n) {
  const long long b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 4096 ? 4096 : b));
}

}  // namespace

int exa_k_ldg_fcon(const ExaDims& P, const int* f2e, const int* perm, const int* elemcon, int* fcon, cudaStream_t st) {
  ldg_fcon_kernel<<<blocks_for((long long)P.ndf * P.ne), 256, 0, st>>>(P, f2e, perm, elemcon, fcon);
  EXA_LAUNCH_CHECK();
  ldg_fcon_boundary_kernel<<<blocks_for((long long)P.npf * P.nf), 256, 0, st>>>(P, f2e, fcon);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_k_ldg_gather(const ExaDims& P, const int* f2e, const int* perm, const int* elemcon, const double* Rue,
                     const double* Rh, double* Ru, int tdep, double dtfactor, cudaStream_t st) {
  if (P.ne <= 0) return EXA_OK;
  const size_t smem = sizeof(double) * (size_t)P.npe * P.ncu;
  EXA_TRY(exa_allow_smem((const void*)ldg_gather_kernel, smem));
  ldg_gather_kernel<<<P.ne, 128, smem, st>>>(P, f2e, perm, elemcon, Rue, Rh, Ru, tdep, dtfactor);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_k_ldg_mass(const ExaDims& P, const double* shapegt, const double* shapegw, const double* elemg, double* mass,
                   cudaStream_t st) {
  if (P.ne <= 0) return EXA_OK;
  ldg_mass_kernel<<<P.ne, 128, 0, st>>>(P, shapegt, shapegw, elemg, mass);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_lincomb(double* out, double a, const double* x, double b, const double* y, long long n, cudaStream_t st) {
  if (n <= 0) return EXA_OK;
  lincomb_kernel<<<blocks_for(n), 256, 0, st>>>(out, a, x, b, y, n);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

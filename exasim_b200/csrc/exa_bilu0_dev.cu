// Device side of the super-element additive Schwarz preconditioner with block ILU(0)
// (Exasim preconditioner = 2): assembly of the sub-domain face blocks from the condensed
// element matrices, the block ILU(0) factorization and its application.
//
// Blocks are ncf x ncf (ncf = ncu npf), column-major; block (r, t) of sub-domain r and CRS
// position t lies at BE + ncf^2 (r + nse t), as in the reference (kokkosimpl.h:1264-1341).
// The factorization (matvec.cpp:119-166) and the sweeps (preconditioner.cpp:184-271) are
// sequential over the faces of a sub-domain and parallel over the sub-domains: one CTA per
// sub-domain walks the schedule built on the host (exa_bilu0.cpp) with dense block work
// spread over its threads in shared memory.  The sub-domain results are summed back onto the
// global faces in a fixed order (preconditioner.cpp:296-325 sums them atomically).
#include "exa_kernels.cuh"

namespace {

template <typename T>
__global__ void bilu_assemble_kernel(ExaDims P, const int* f2e, const int* elemcon, const int* face,
                                     const int* row_ptr, const int* col_ind, const int* row_of, int nse, int nnz,
                                     const T* H, T* BE) {
  const int ncu = P.ncu, npf = P.npf, ncf = ncu * npf, ndf = P.ndf, m = P.m;
  const long long N = (long long)ncf * ncf * nse * nnz;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
       idx += (long long)gridDim.x * blockDim.x) {
    const int mm = (int)(idx % ncf);
    long long q = idx / ncf;
    const int nn = (int)(q % ncf);
    q /= ncf;
    const int r = (int)(q % nse);
    const int t = (int)(q / nse);
    const int i = row_of[t];
    const int am = mm % ncu, bm = mm / ncu, an = nn % ncu, bn = nn / ncu;
    const int fi = face[r + nse * i];
    const int e1 = f2e[4 * fi], l1 = f2e[4 * fi + 1], e2 = f2e[4 * fi + 2], l2 = f2e[4 * fi + 3];
    double v;
    if (t == row_ptr[i]) {
      const int m1 = am + ncu * (elemcon[bm + npf * l1 + ndf * e1] - npf * fi);
      const int n1 = an + ncu * (elemcon[bn + npf * l1 + ndf * e1] - npf * fi);
      v = (double)H[(long long)e1 * m * m + (m1 + ncf * l1) + (long long)m * (n1 + ncf * l1)];
      if (e2 >= 0) {
        const int m2 = am + ncu * (elemcon[bm + npf * l2 + ndf * e2] - npf * fi);
        const int n2 = an + ncu * (elemcon[bn + npf * l2 + ndf * e2] - npf * fi);
        v += (double)H[(long long)e2 * m * m + (m2 + ncf * l2) + (long long)m * (n2 + ncf * l2)];
      }
    } else {
      // the element shared by face fi and its neighbour fj, and their local numbers in it
      const int fj = face[r + nse * col_ind[t]];
      const int je1 = f2e[4 * fj], jl1 = f2e[4 * fj + 1], je2 = f2e[4 * fj + 2], jl2 = f2e[4 * fj + 3];
      int e, k1, k2;
      if (je1 == e1) e = e1, k1 = l1, k2 = jl1;
      else if (je1 == e2) e = e2, k1 = l2, k2 = jl1;
      else if (je2 == e1) e = e1, k1 = l1, k2 = jl2;
      else e = e2, k1 = l2, k2 = jl2;
      if (e < 0 || (je2 != e && je1 != e)) {
        v = 0.0;  // the pattern of sub-domain 0 does not hold here (cartgridpart does not fit the mesh)
      } else {
        const int m1 = am + ncu * (elemcon[bm + npf * k1 + ndf * e] - npf * fi);
        const int n2 = an + ncu * (elemcon[bn + npf * k2 + ndf * e] - npf * fj);
        v = (double)H[(long long)e * m * m + (m1 + ncf * k1) + (long long)m * (n2 + ncf * k2)];
      }
    }
    BE[idx] = (T)v;
  }
}

// In-place inverse of the ncf x ncf block at `g` through the augmented matrix [A | I] in
// shared memory: Gauss-Jordan with partial pivoting (largest magnitude, first on ties).
template <typename T>
__device__ void block_inverse(T* g, T* aug, int ncf, int* flag) {
  const int w = 2 * ncf;
  __shared__ int s_piv;
  for (int x = threadIdx.x; x < ncf * w; x += blockDim.x) {
    const int rr = x % ncf, cc = x / ncf;
    aug[x] = cc < ncf ? g[rr + ncf * cc] : T(rr == cc - ncf ? 1 : 0);
  }
  __syncthreads();
  for (int k = 0; k < ncf; ++k) {
    if (threadIdx.x < 32) {
      T best = T(-1);
      int bi = ncf;
      for (int rr = k + (int)threadIdx.x; rr < ncf; rr += 32) {
        const T v = aug[rr + ncf * k] < T(0) ? -aug[rr + ncf * k] : aug[rr + ncf * k];
        if (v > best) best = v, bi = rr;
      }
      for (int off = 16; off > 0; off >>= 1) {
        const T ob = __shfl_xor_sync(0xffffffffu, best, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi < bi)) best = ob, bi = oi;
      }
      if (threadIdx.x == 0) {
        if (!(best > T(0)) || bi >= ncf) {
          atomicExch(flag, 1);
          bi = k;
        }
        s_piv = bi;
      }
    }
    __syncthreads();
    const int p = s_piv;
    if (p != k)
      for (int cc = threadIdx.x; cc < w; cc += blockDim.x) {
        const T tmp = aug[k + ncf * cc];
        aug[k + ncf * cc] = aug[p + ncf * cc];
        aug[p + ncf * cc] = tmp;
      }
    __syncthreads();
    const T d = T(1) / aug[k + ncf * k];
    __syncthreads();
    for (int cc = threadIdx.x; cc < w; cc += blockDim.x) aug[k + ncf * cc] *= d;
    __syncthreads();
    // eliminate column k from every other row: multipliers first, then the update
    for (int x = threadIdx.x; x < ncf * (w - k); x += blockDim.x) {
      const int rr = x % ncf, cc = k + x / ncf;
      if (rr == k || cc == k) continue;
      aug[rr + ncf * cc] -= aug[rr + ncf * k] * aug[k + ncf * cc];
    }
    __syncthreads();
    for (int rr = threadIdx.x; rr < ncf; rr += blockDim.x)
      if (rr != k) aug[rr + ncf * k] = T(0);
    __syncthreads();
  }
  for (int x = threadIdx.x; x < ncf * ncf; x += blockDim.x) g[x] = aug[x + ncf * ncf];
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(256) bilu_factor_kernel(int ncf, int nse, int nfse, const int* row_ptr,
                                                          const int* fac_ptr, const int* fac_ji, const int* upd_ptr,
                                                          const int* upd_jl, const int* upd_il, T* BE, int* flag) {
  extern __shared__ __align__(16) unsigned char fsm[];
  T* aug = reinterpret_cast<T*>(fsm);   // [ncf, 2 ncf]
  T* A = aug + 2 * ncf * ncf;            // (j, i) block times the inverse diagonal
  T* B = A + ncf * ncf;                  // (i, l) block
  const int r = blockIdx.x, nn = ncf * ncf;
  auto blk = [&](int t) { return BE + (long long)nn * (r + (long long)nse * t); };
  for (int i = 0; i < nfse; ++i) {
    T* D = blk(row_ptr[i]);
    block_inverse(D, aug, ncf, flag);
    // aug's right half keeps D^-1
    const T* Di = aug + nn;
    for (int q = fac_ptr[i]; q < fac_ptr[i + 1]; ++q) {
      T* Lji = blk(fac_ji[q]);
      for (int x = threadIdx.x; x < nn; x += blockDim.x) B[x] = Lji[x];
      __syncthreads();
      for (int x = threadIdx.x; x < nn; x += blockDim.x) {
        const int rr = x % ncf, cc = x / ncf;
        double s = 0.0;
        for (int k = 0; k < ncf; ++k) s += (double)B[rr + ncf * k] * (double)Di[k + ncf * cc];
        A[x] = (T)s;
        Lji[x] = (T)s;
      }
      __syncthreads();
      for (int u = upd_ptr[q]; u < upd_ptr[q + 1]; ++u) {
        const T* Uil = blk(upd_il[u]);
        for (int x = threadIdx.x; x < nn; x += blockDim.x) B[x] = Uil[x];
        __syncthreads();
        T* Cjl = blk(upd_jl[u]);
        for (int x = threadIdx.x; x < nn; x += blockDim.x) {
          const int rr = x % ncf, cc = x / ncf;
          double s = 0.0;
          for (int k = 0; k < ncf; ++k) s += (double)A[rr + ncf * k] * (double)B[k + ncf * cc];
          Cjl[x] = (T)((double)Cjl[x] - s);
        }
        __syncthreads();
      }
    }
  }
}

// y = L^-1 (gathered x), z = U^-1 y per sub-domain; out[(r + nse i) ncf + a] = z_i[a]
template <typename T>
__global__ void __launch_bounds__(256) bilu_apply_kernel(int ncf, int nse, int nfse, const int* row_ptr,
                                                         const int* col_ind, const int* face, const T* BE,
                                                         const double* x, double* out) {
  extern __shared__ double asm_[];
  double* y = asm_;                  // [nfse, ncf]
  double* z = y + nfse * ncf;        // [nfse, ncf]
  const int G = blockDim.x / ncf;    // groups of ncf threads share the blocks of a row
  double* part = z + nfse * ncf;     // [G, ncf]
  double* v = part + G * ncf;        // [ncf]
  const int r = blockIdx.x, nn = ncf * ncf;
  const int a = threadIdx.x % ncf, g = threadIdx.x / ncf;
  auto blk = [&](int t) { return BE + (long long)nn * (r + (long long)nse * t); };
  for (int t = threadIdx.x; t < nfse * ncf; t += blockDim.x) {
    const int i = t / ncf, c = t % ncf;
    y[t] = x[(long long)ncf * face[r + nse * i] + c];
  }
  __syncthreads();
  for (int i = 0; i < nfse; ++i) {
    double s = 0.0;
    if (g < G)
      for (int t = row_ptr[i] + 1 + g; t < row_ptr[i + 1]; t += G) {
        const int j = col_ind[t];
        if (j >= i) continue;
        const T* L = blk(t);
        for (int k = 0; k < ncf; ++k) s += (double)L[a + ncf * k] * y[j * ncf + k];
      }
    if (g < G) part[g * ncf + a] = s;
    __syncthreads();
    if (threadIdx.x < ncf) {
      double acc = 0.0;
      for (int q = 0; q < G; ++q) acc += part[q * ncf + threadIdx.x];
      y[i * ncf + threadIdx.x] -= acc;
    }
    __syncthreads();
  }
  for (int i = nfse - 1; i >= 0; --i) {
    double s = 0.0;
    if (g < G)
      for (int t = row_ptr[i] + 1 + g; t < row_ptr[i + 1]; t += G) {
        const int l = col_ind[t];
        if (l <= i) continue;
        const T* U = blk(t);
        for (int k = 0; k < ncf; ++k) s += (double)U[a + ncf * k] * z[l * ncf + k];
      }
    if (g < G) part[g * ncf + a] = s;
    __syncthreads();
    if (threadIdx.x < ncf) {
      double acc = 0.0;
      for (int q = 0; q < G; ++q) acc += part[q * ncf + threadIdx.x];
      v[threadIdx.x] = y[i * ncf + threadIdx.x] - acc;
    }
    __syncthreads();
    if (threadIdx.x < ncf) {
      const T* Di = blk(row_ptr[i]);
      double acc = 0.0;
      for (int k = 0; k < ncf; ++k) acc += (double)Di[threadIdx.x + ncf * k] * v[k];
      z[i * ncf + threadIdx.x] = acc;
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < nfse * ncf; t += blockDim.x) {
    const int i = t / ncf, c = t % ncf;
    out[((long long)r + (long long)nse * i) * ncf + c] = z[t];
  }
}

// w[f] = sum of the sub-domain copies of face f, in the order of gf_pos
__global__ void bilu_sum_kernel(int ncf, int nf, const int* gf_ptr, const int* gf_pos, const double* out,
                                double* w) {
  const long long N = (long long)ncf * nf;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
       idx += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(idx % ncf);
    const int f = (int)(idx / ncf);
    double s = 0.0;
    for (int p = gf_ptr[f]; p < gf_ptr[f + 1]; ++p) s += out[(long long)gf_pos[p] * ncf + c];
    w[idx] = s;
  }
}

int grid_of(long long n) {
  const long long b = (n + 255) / 256;
  return (int)(b < 148LL * 16 ? (b > 0 ? b : 1) : 148LL * 16);
}

}  // namespace

size_t exa_bilu_apply_smem(int ncf, int nfse) {
  const int G = 256 / ncf;
  return sizeof(double) * ((size_t)2 * nfse * ncf + (size_t)G * ncf + ncf);
}

template <typename T>
int exa_k_bilu_build(const ExaDims& P, const ExaBiluDev& b, const int* f2e, const int* elemcon, const T* H, T* BE,
                     int* flag, cudaStream_t st) {
  const int ncf = P.ncu * P.npf;
  if (ncf > 64) {
    exa_set_error("block ILU(0): face blocks of %d rows exceed 64", ncf);
    return EXA_ERR_UNSUPPORTED;
  }
  const long long N = (long long)ncf * ncf * b.nse * b.nnz;
  bilu_assemble_kernel<T><<<grid_of(N), 256, 0, st>>>(P, f2e, elemcon, b.face, b.row_ptr, b.col_ind, b.row_of, b.nse,
                                                       b.nnz, H, BE);
  EXA_LAUNCH_CHECK();
  const size_t smem = sizeof(T) * 4 * (size_t)ncf * ncf;
  EXA_TRY(exa_allow_smem((const void*)bilu_factor_kernel<T>, smem));
  bilu_factor_kernel<T><<<b.nse, 256, smem, st>>>(ncf, b.nse, b.nfse, b.row_ptr, b.fac_ptr, b.fac_ji, b.upd_ptr,
                                                   b.upd_jl, b.upd_il, BE, flag);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

template <typename T>
int exa_k_bilu_apply(const ExaDims& P, const ExaBiluDev& b, const T* BE, const double* x, double* w,
                     cudaStream_t st) {
  const int ncf = P.ncu * P.npf;
  const size_t smem = exa_bilu_apply_smem(ncf, b.nfse);
  EXA_TRY(exa_allow_smem((const void*)bilu_apply_kernel<T>, smem));
  bilu_apply_kernel<T><<<b.nse, 256, smem, st>>>(ncf, b.nse, b.nfse, b.row_ptr, b.col_ind, b.face, BE, x, b.out);
  EXA_LAUNCH_CHECK();
  bilu_sum_kernel<<<grid_of((long long)ncf * P.nf), 256, 0, st>>>(ncf, P.nf, b.gf_ptr, b.gf_pos, b.out, w);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

template int exa_k_bilu_build<double>(const ExaDims&, const ExaBiluDev&, const int*, const int*, const double*,
                                      double*, int*, cudaStream_t);
template int exa_k_bilu_build<float>(const ExaDims&, const ExaBiluDev&, const int*, const int*, const float*, float*,
                                     int*, cudaStream_t);
template int exa_k_bilu_apply<double>(const ExaDims&, const ExaBiluDev&, const double*, const double*, double*,
                                      cudaStream_t);
template int exa_k_bilu_apply<float>(const ExaDims&, const ExaBiluDev&, const float*, const double*, double*,
                                     cudaStream_t);

// Volume blocks D and B of the element Jacobian on the tcgen05 tensor cores (3xTF32,
// FP32 accumulation), for the mixed-precision form.
//
// For every element e and every (trace component k, field c) pair (uequation.cpp:45-203):
//   M[i, j] = - sum_g T[i, g] S[g, j],   T[i, g] = sum_d shapegw[i, g, d] rgJ[g, d, k, c],
// with S = shapegt[:, :, 0] the basis at the Gauss points.  S is the same for every element:
// it is packed once (hi and lo TF32 parts, B operand) and stays in shared memory for the
// whole CTA.  Each CTA walks a strided list of (element, pair) items; for each it forms T
// chunk by chunk (16 Gauss points) directly in the packed A layout in a double-buffered
// stage while one thread issues the MMAs of the previous chunk, then four warps per column
// half read the accumulator from tensor memory and write the FP64 block where the FP64
// vol_mat_kernel writes it (columns of D for c < ncu, of B otherwise).
//
// Shapes: npe <= 128 and nge <= 128 (one 128 x 128 tile).  Every mbarrier wait is bounded;
// a wait that runs out sets *flag (2), stops the CTA's loop and frees the tensor memory.
#include <cstdint>

#include "exa_kernels.cuh"
#include "exa_tc.cuh"
#include "exa_umma.cuh"

using namespace exa_tc;

namespace {

constexpr int VTN = 256;  // threads: 8 warps form T; warps w and w + 4 read TMEM lanes 32 (w % 4)

__global__ void __launch_bounds__(VTN, 1) vol_mat_tc_kernel(ExaDims P, const double* __restrict__ W, UPacked Sp,
                                                            const double* __restrict__ rgJ, double* D, double* B,
                                                            int nitems, int* flag) {
  const int npe = P.npe, nge = P.nge, nd = P.nd, ncu = P.ncu, nc = P.nc, n = P.n;
  const int nblk = ncu * nc;
  const int nkc = (nge + PK - 1) / PK, ngS = (npe + 7) / 8;
  const uint32_t sbytes = (uint32_t)nkc * ngS * 512;      // one part of S
  constexpr uint32_t ABYTES = 16 * 512;                    // one part of a T chunk (128 rows x 16)
  constexpr uint32_t IDESC = idesc_tf32(128, 128);
  extern __shared__ __align__(1024) uint8_t vsm[];
  uint8_t* s_hi = vsm;
  uint8_t* s_lo = vsm + sbytes;
  uint8_t* abuf = vsm + 2 * sbytes;                        // [2][hi, lo]
  double* Rs = reinterpret_cast<double*>(abuf + 4 * ABYTES);  // [nge * (nd + 1)]
  uint64_t* bars = reinterpret_cast<uint64_t*>(Rs + nge * (nd + 1) + 1);  // sload, abar[2], done
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 4);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < 4; ++i) mbar_init(&bars[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    // S in copies of one K chunk each (ngS groups, 512 bytes per group and part)
    const uint32_t cb = (uint32_t)ngS * 512;
    mbar_expect_tx(&bars[0], 2 * sbytes);
    for (int q = 0; q < nkc; ++q) {
      bulk_g2s(s_hi + q * cb, reinterpret_cast<const uint8_t*>(Sp.hi) + (size_t)q * cb, cb, &bars[0]);
      bulk_g2s(s_lo + q * cb, reinterpret_cast<const uint8_t*>(Sp.lo) + (size_t)q * cb, cb, &bars[0]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  bool ok = __syncthreads_and(mbar_wait(&bars[0], 0));

  long long chunk = 0;  // chunks issued by this CTA: buffer chunk & 1, its mbarrier phase chunk >> 1
  int items = 0;
  for (int it = blockIdx.x; ok && it < nitems; it += gridDim.x, ++items) {
    const int e = it / nblk, kc = it - e * nblk;
    const int k = kc % ncu, c = kc / ncu;
    const double* R = rgJ + (long long)e * nge * (nd + 1) * nblk + (long long)nge * (nd + 1) * kc;
    for (int t = tid; t < nge * (nd + 1); t += VTN) Rs[t] = R[t];
    __syncthreads();
    for (int q = 0; q < nkc; ++q, ++chunk) {
      const int bsel = (int)(chunk & 1);
      if (chunk >= 2) {
        const bool w = mbar_wait(&bars[1 + bsel], (uint32_t)(((chunk >> 1) - 1) & 1));
        if (!__syncthreads_and(w)) {
          ok = false;
          break;
        }
      }
      uint8_t* ah = abuf + bsel * 2 * ABYTES;
      uint8_t* al = ah + ABYTES;
      // a warp fills one core matrix (8 rows x 4 Gauss points) per pass: 64 cores per chunk
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const int ci = warp + 8 * p, i8 = ci & 15, ki = ci >> 4;
        const int i = 8 * i8 + (lane >> 2), g = PK * q + 4 * ki + (lane & 3);
        double x = 0.0;
        if (i < npe && g < nge) {
          const double* w0 = W + i + (long long)npe * g;
#pragma unroll 4
          for (int d = 0; d <= nd; ++d) x = fma(w0[(long long)npe * nge * d], Rs[g + nge * d], x);
        }
        float h, l;
        split_tf32(x, h, l);
        const int off = i8 * 512 + ki * 128 + lane * 4;
        *reinterpret_cast<float*>(ah + off) = h;
        *reinterpret_cast<float*>(al + off) = l;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a_hi = smem_addr(ah), a_lo = smem_addr(al);
        const uint32_t b_hi = smem_addr(s_hi) + (uint32_t)q * ngS * 512, b_lo = smem_addr(s_lo) + (uint32_t)q * ngS * 512;
#pragma unroll
        for (int kk = 0; kk < PK / 8; ++kk) {
          const uint32_t o = kk * 256;
          umma_tf32(tmem, sdesc(a_hi + o, 128, 512), sdesc(b_hi + o, 128, 512), IDESC, (q > 0 || kk > 0) ? 1u : 0u);
          umma_tf32(tmem, sdesc(a_hi + o, 128, 512), sdesc(b_lo + o, 128, 512), IDESC, 1u);
          umma_tf32(tmem, sdesc(a_lo + o, 128, 512), sdesc(b_hi + o, 128, 512), IDESC, 1u);
        }
        umma_commit(&bars[1 + bsel]);
      }
    }
    if (!ok) break;
    if (tid == 0) umma_commit(&bars[3]);
    if (!__syncthreads_and(mbar_wait(&bars[3], (uint32_t)(items & 1)))) {
      ok = false;
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // epilogue: warp w reads lanes 32 (w % 4) .. +31, columns [64 (w / 4), 64 (w / 4) + 64)
    double* out;
    long long col0;
    if (c < ncu) {
      out = D + (long long)e * n * n;
      col0 = (long long)npe * c;
    } else {
      const int qc = c - ncu, nq = qc % ncu, d = qc / ncu;
      out = B + (long long)e * n * npe * nd * ncu;
      col0 = (long long)npe * d + (long long)npe * nd * nq;
    }
    const int i = 32 * (warp & 3) + lane, h0 = 64 * (warp >> 2);
#pragma unroll 1
    for (int j0 = h0; j0 < h0 + 64; j0 += 16) {
      uint32_t v[16];
      const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)j0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (i < npe) {
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
          const int j = j0 + jj;
          if (j < npe) out[(i + (long long)npe * k) + (long long)n * (col0 + j)] = -(double)__uint_as_float(v[jj]);
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // TMEM read and Rs used before the next item overwrites them
  }
  if (!ok) {
    // let the MMAs already issued finish (bounded) before the tensor memory is freed
    if (tid == 0) {
      atomicExch(flag, EXA_UMMA_TIMEOUT);
      umma_commit(&bars[3]);
    }
    mbar_wait(&bars[3], (uint32_t)(items & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
}

}  // namespace

size_t exa_vol_mat_tc_smem(const ExaDims& P) {
  const size_t nkc = (P.nge + PK - 1) / PK, ngS = (P.npe + 7) / 8;
  return 2 * nkc * ngS * 512 + 4 * 16 * 512 + sizeof(double) * ((size_t)P.nge * (P.nd + 1) + 1) + 4 * 8 + 16;
}

bool exa_vol_mat_tc_fits(const ExaDims& P) {
  return P.npe <= 128 && P.nge <= 128 && exa_vol_mat_tc_smem(P) <= 227 * 1024;
}

int exa_k_vol_mat_tc(const ExaDims& P, const double* shapegw, const UPacked& Sp, const double* rgJ, double* D,
                     double* B, int nb, int* flag, cudaStream_t st) {
  if (!exa_vol_mat_tc_fits(P) || Sp.R != P.npe || Sp.K != P.nge) {
    exa_set_error("tensor-core volume kernel: npe %d, nge %d outside one 128 x 128 tile", P.npe, P.nge);
    return EXA_ERR_UNSUPPORTED;
  }
  const size_t smem = exa_vol_mat_tc_smem(P);
  EXA_CUDA(cudaFuncSetAttribute((const void*)vol_mat_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
  const int nitems = nb * P.ncu * P.nc;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = nitems < sms ? nitems : sms;
  vol_mat_tc_kernel<<<grid, VTN, smem, st>>>(P, shapegw, Sp, rgJ, D, B, nitems, flag);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

// Volume blocks D and B of the element Jacobian on the tcgen05 tensor cores (3xTF32,
// FP32 accumulation), for the mixed-precision form.
//
// For every element e and every (trace component k, field c) pair (uequation.cpp:45-203):
//   M[i, j] = - sum_g T[i, g] S[g, j],   T[i, g] = sum_d shapegw[i, g, d] rgJ[g, d, k, c],
// with S = shapegt[:, :, 0] the basis at the Gauss points.  S is the same for every element:
// it is packed once (hi and lo TF32 parts, B operand) and stays in shared memory for the
// whole CTA.  Each CTA walks a strided list of items, an item being up to four (k, c)
// pairs of one element: chunk by chunk (16 Gauss points) it loads each weight shapegw[i, g, d]
// once, forms the four T tiles directly in the packed A layout and issues their MMAs into
// four 128-column accumulators (all 512 columns of tensor memory); then the eight warps read
// the accumulators back and write the blocks where the FP64 vol_mat_kernel writes them
// (columns of D for c < ncu, of B otherwise; B packed in FP32 when the q elimination takes it
// so).
//
// T is formed in FP32 from an FP32 copy of shapegw and the FP32-rounded rgJ: its rounding
// (4 products of FP32 operands) is of the order of the 22-bit hi + lo split that the 3xTF32
// product applies to it anyway.  The four tiles are formed and multiplied in two halves (pairs
// 0-1 and 2-3), each with its own A buffers and completion barrier, so the MMAs of one half
// run while the threads form the other's tiles.
//
// Shapes: npe <= 128, nge <= 128 (one 128 x 128 tile per pair) and nd <= 3.  Every mbarrier wait is bounded;
// a wait that runs out sets *flag (2), stops the CTA's loop and frees the tensor memory.
#include <cstdint>

#include "exa_kernels.cuh"
#include "exa_tc.cuh"
#include "exa_umma.cuh"

using namespace exa_tc;

namespace {

constexpr int VTN = 256;   // threads: 8 warps form T; warps w and w + 4 read TMEM lanes 32 (w % 4)
constexpr int VGRP = 4;    // (k, c) blocks per item: 4 accumulators of 128 columns fill TMEM

__global__ void __launch_bounds__(VTN, 1) vol_mat_tc_kernel(ExaDims P, const float* __restrict__ W, UPacked Sp,
                                                            const double* __restrict__ rgJ, double* D, double* B,
                                                            UPacked Bp, int nb, int* flag) {
  const int npe = P.npe, nge = P.nge, nd = P.nd, ncu = P.ncu, nc = P.nc, n = P.n;
  const int nblk = ncu * nc, ngrp = (nblk + VGRP - 1) / VGRP;
  const int nkc = (nge + PK - 1) / PK, ngS = (npe + 7) / 8;
  const int rlen = nge * (nd + 1);
  const uint32_t sbytes = (uint32_t)nkc * ngS * 512;      // one part of S
  constexpr uint32_t ABYTES = 16 * 512;                    // one part of one T chunk (128 rows x 16)
  constexpr uint32_t IDESC = idesc_tf32(128, 128);
  extern __shared__ __align__(1024) uint8_t vsm[];
  uint8_t* s_hi = vsm;
  uint8_t* s_lo = vsm + sbytes;
  uint8_t* abuf = vsm + 2 * sbytes;                        // [VGRP][hi, lo]
  float* Rs = reinterpret_cast<float*>(abuf + 2 * VGRP * ABYTES);  // [VGRP][nge * (nd + 1)]
  uint64_t* bars = reinterpret_cast<uint64_t*>(Rs + ((VGRP * rlen + 1) & ~1));  // S load, MMAs of half 0, of half 1
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 3);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_init(&bars[2], 1);
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

  // commits to the barrier of each half so far (the same count in every thread): a half's A
  // buffers are rewritten only after its latest commit has completed
  int commits[2] = {0, 0};
  bool pending[2] = {false, false};
  const int nitems = nb * ngrp;
  for (int it = blockIdx.x; ok && it < nitems; it += gridDim.x) {
    const int e = it / ngrp, b0 = (it - e * ngrp) * VGRP;
    const int nbg = min(VGRP, nblk - b0);
    const double* R = rgJ + (long long)e * rlen * nblk + (long long)rlen * b0;
    for (int t = tid; t < nbg * rlen; t += VTN) Rs[t] = (float)R[t];
    __syncthreads();
    for (int q = 0; ok && q < nkc; ++q) {
      // every weight W[i, g, d] is loaded once per chunk and serves the item's nbg blocks; the
      // loads of all eight passes are issued before any is used (one L2 round trip per chunk)
      float w[8][4];
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const int ci = warp + 8 * p, i8 = ci & 15, ki = ci >> 4;
        const int i = 8 * i8 + (lane >> 2), g = PK * q + 4 * ki + (lane & 3);
        const bool in = i < npe && g < nge;
        const float* w0 = W + i + (long long)npe * g;
#pragma unroll
        for (int d = 0; d < 4; ++d) w[p][d] = (in && d <= nd) ? w0[(long long)npe * nge * d] : 0.0f;
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (2 * h >= nbg) break;
        if (pending[h] && !__syncthreads_and(mbar_wait(&bars[1 + h], (uint32_t)((commits[h] - 1) & 1)))) {
          ok = false;
          break;
        }
        pending[h] = false;
#pragma unroll
        for (int p = 0; p < 8; ++p) {
          const int ci = warp + 8 * p, i8 = ci & 15, ki = ci >> 4;
          const int g = PK * q + 4 * ki + (lane & 3);
          const int gg = g < nge ? g : 0;
          const int off = i8 * 512 + ki * 128 + lane * 4;
#pragma unroll
          for (int bb = 0; bb < 2; ++bb) {
            const int b = 2 * h + bb;
            if (b >= nbg) break;
            const float* rb = Rs + b * rlen + gg;
            float x = 0.0f;
#pragma unroll
            for (int d = 0; d < 4; ++d)
              if (d <= nd) x = fmaf(w[p][d], rb[nge * d], x);
            float hi, lo;
            split_tf32f(x, hi, lo);
            *reinterpret_cast<float*>(abuf + (2 * b) * ABYTES + off) = hi;
            *reinterpret_cast<float*>(abuf + (2 * b + 1) * ABYTES + off) = lo;
          }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t b_hi = smem_addr(s_hi) + (uint32_t)q * ngS * 512, b_lo = smem_addr(s_lo) + (uint32_t)q * ngS * 512;
          for (int b = 2 * h; b < 2 * h + 2 && b < nbg; ++b) {
            const uint32_t a_hi = smem_addr(abuf + (2 * b) * ABYTES), a_lo = a_hi + ABYTES;
            const uint32_t acc = tmem + (uint32_t)(128 * b);
#pragma unroll
            for (int kk = 0; kk < PK / 8; ++kk) {
              const uint32_t o = kk * 256;
              umma_tf32(acc, sdesc(a_hi + o, 128, 512), sdesc(b_hi + o, 128, 512), IDESC, (q > 0 || kk > 0) ? 1u : 0u);
              umma_tf32(acc, sdesc(a_hi + o, 128, 512), sdesc(b_lo + o, 128, 512), IDESC, 1u);
              umma_tf32(acc, sdesc(a_lo + o, 128, 512), sdesc(b_hi + o, 128, 512), IDESC, 1u);
            }
          }
          umma_commit(&bars[1 + h]);
        }
        ++commits[h];
        pending[h] = true;
      }
    }
    if (!ok) break;
    // every MMA of the item has completed before the accumulators are read
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (pending[h] && !__syncthreads_and(mbar_wait(&bars[1 + h], (uint32_t)((commits[h] - 1) & 1)))) ok = false;
      pending[h] = false;
    }
    if (!ok) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // epilogue: warp w reads lanes 32 (w % 4) .. +31 of blocks 2 (w / 4) and 2 (w / 4) + 1
    const int i = 32 * (warp & 3) + lane;
    for (int bb = 0; bb < 2; ++bb) {
      const int b = 2 * (warp >> 2) + bb;
      if (b >= nbg) break;  // warp-uniform
      const int kc = b0 + b, k = kc % ncu, c = kc / ncu;
      double* out = nullptr;
      float* outp = nullptr;  // B as the packed FP32 operand of the q elimination (part nq)
      long long col0;
      int kk0 = 0;
      if (c < ncu) {
        out = D + (long long)e * n * n;
        col0 = (long long)npe * c;
      } else {
        const int qc = c - ncu, nq = qc % ncu, d = qc / ncu;
        col0 = (long long)npe * d + (long long)npe * nd * nq;
        if (Bp.hi) {
          outp = Bp.hi + (long long)e * Bp.sb + (long long)nq * Bp.sb2;
          kk0 = qk_group(npe) * d;
        } else {
          out = B + (long long)e * n * npe * nd * ncu;
        }
      }
#pragma unroll 1
      for (int j0 = 0; j0 < 128; j0 += 16) {
        uint32_t v[16];
        const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(128 * b + j0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (i < npe) {
          if (outp) {
            // whole quads of k: the group starts on a quad and the accumulator's columns from
            // npe to the group's end are zeros (S is zero-padded there)
            const int row = i + npe * k, t = row / Bp.TR;
            const int ng = (min(Bp.TR, n - t * Bp.TR) + 7) / 8;
            float* rp = outp + pack_off(row, 0, n, Bp.K, Bp.TR);
#pragma unroll
            for (int jj = 0; jj < 16; jj += 4) {
              const int j = j0 + jj, kq = kk0 + j;
              if (j >= qk_group(npe)) break;
              *reinterpret_cast<float4*>(rp + (long long)(kq >> 4) * ng * 128 + ((kq >> 2) & 3) * 32) =
                  make_float4(-__uint_as_float(v[jj]), -__uint_as_float(v[jj + 1]), -__uint_as_float(v[jj + 2]),
                              -__uint_as_float(v[jj + 3]));
            }
          } else {
#pragma unroll
            for (int jj = 0; jj < 16; ++jj) {
              const int j = j0 + jj;
              if (j < npe) out[(i + (long long)npe * k) + (long long)n * (col0 + j)] = -(double)__uint_as_float(v[jj]);
            }
          }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // TMEM read and Rs used before the next item overwrites them
  }
  if (!ok && tid == 0) atomicExch(flag, EXA_UMMA_TIMEOUT);
  // an abort leaves the loop after a bounded wait on MMAs it issued; wait once more (bounded)
  // on each half's latest commit so none is in flight when the tensor memory is freed
  if (!ok)
    for (int h = 0; h < 2; ++h)
      if (commits[h] > 0) mbar_wait(&bars[1 + h], (uint32_t)((commits[h] - 1) & 1));
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
}

}  // namespace

size_t exa_vol_mat_tc_smem(const ExaDims& P) {
  const size_t nkc = (P.nge + PK - 1) / PK, ngS = (P.npe + 7) / 8;
  const size_t rs = ((size_t)VGRP * P.nge * (P.nd + 1) + 1) & ~(size_t)1;  // floats, even: the barriers follow
  return 2 * nkc * ngS * 512 + 2 * VGRP * 16 * 512 + sizeof(float) * rs + 3 * 8 + 16;
}

bool exa_vol_mat_tc_fits(const ExaDims& P) {
  return P.npe <= 128 && P.nge <= 128 && P.nd <= 3 && exa_vol_mat_tc_smem(P) <= 227 * 1024;
}

int exa_k_vol_mat_tc(const ExaDims& P, const float* shapegw32, const UPacked& Sp, const double* rgJ, double* D,
                     double* B, const UPacked& Bp, int nb, int* flag, cudaStream_t st) {
  if (Bp.hi && (Bp.lo || Bp.R != P.n || Bp.K != qk_group(P.npe) * P.nd || Bp.TR % 8 != 0)) {
    exa_set_error("tensor-core volume kernel: packed B must be FP32 single with %d rows and %d k", P.n,
                  qk_group(P.npe) * P.nd);
    return EXA_ERR_ARG;
  }
  if (!exa_vol_mat_tc_fits(P) || Sp.R != P.npe || Sp.K != P.nge) {
    exa_set_error("tensor-core volume kernel: npe %d, nge %d outside one 128 x 128 tile", P.npe, P.nge);
    return EXA_ERR_UNSUPPORTED;
  }
  const size_t smem = exa_vol_mat_tc_smem(P);
  EXA_TRY(exa_allow_smem((const void*)vol_mat_tc_kernel, smem));
  const int nitems = nb * ((P.ncu * P.nc + VGRP - 1) / VGRP);
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = nitems < sms ? nitems : sms;
  vol_mat_tc_kernel<<<grid, VTN, smem, st>>>(P, shapegw32, Sp, rgJ, D, B, Bp, nb, flag);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

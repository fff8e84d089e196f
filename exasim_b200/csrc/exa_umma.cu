// Batched GEMM on the 5th-generation tensor cores (tcgen05, kind::tf32) with FP32
// accumulation in tensor memory, for the mixed-precision element elimination.
//
// One CTA computes a 128-row tile of one batch entry's C = alpha A B + beta Cin over all
// of its (at most NP) columns.  The operands are column-major in HBM, FP64 or FP32 (the
// element blocks come from FP64 assembly).  256 threads load them, round them to TF32 and
// store them in shared memory in the canonical K-major, non-swizzled tcgen05 layout: core
// matrices of 8 rows x 16 bytes, 128 contiguous bytes each, the K-adjacent cores 128 bytes
// apart (LBO) and the 8-row groups 1024 bytes apart (SBO).  A stage holds 32 K values of A
// (128 x 32) and B (NP x 32); three stages form a ring.  One thread issues four
// tcgen05.mma (K = 8 each) per stage and commits them to that stage's mbarrier, which
// frees the stage for the loads three chunks later, so the loads of the next chunk
// overlap the MMAs of the current one.  The accumulator tile (128 lanes x NP columns of
// FP32) lives in tensor memory; the epilogue reads it back with tcgen05.ld (warp w reads
// lanes 32 (w % 4) .. +31, half of the columns each) and writes Cout column by column.
//
// Every wait on an mbarrier is bounded.  A wait that runs out sets *flag (EXA_UMMA_TIMEOUT),
// waits (bounded again) for the MMAs already issued, frees the tensor memory and returns.
#include <algorithm>
#include <atomic>
#include <cstdint>

#include "exa_common.cuh"
#include "exa_umma.cuh"
#include "exa_tc.cuh"

using namespace exa_tc;

namespace {

constexpr int UM = 128;      // tile rows (tcgen05 M)
constexpr int UBK = 32;      // K values per stage
constexpr int UST = 3;       // stages
constexpr int UNT = 256;     // threads
template <typename T>
__device__ __forceinline__ float ldf(const T* p) { return (float)*p; }

template <typename TA, typename TB, typename TCI, typename TCO, int NP>
__global__ void __launch_bounds__(UNT, 2) umma_gemm_kernel(UGemm g, int* flag) {
  static_assert(NP % 16 == 0 && NP >= 16 && NP <= 256, "tcgen05 M=128 needs N a multiple of 16 up to 256");
  constexpr int A_BYTES = UM * UBK * 4, B_BYTES = NP * UBK * 4, STAGE = A_BYTES + B_BYTES;
  constexpr int TCOLS = NP <= 32 ? 32 : (NP <= 64 ? 64 : (NP <= 128 ? 128 : 256));
  constexpr int LA = UM * UBK / UNT, LB = NP * UBK / UNT;
  constexpr uint32_t IDESC = idesc_tf32(UM, NP);
  extern __shared__ __align__(1024) uint8_t usm[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(usm + UST * STAGE);  // [UST] + final
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + UST + 1);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long b1 = blockIdx.y, b2 = blockIdx.z;
  const int m0 = blockIdx.x * UM;
  const TA* A = reinterpret_cast<const TA*>(g.A) + b1 * g.sA + b2 * g.sA2;
  const TB* B = reinterpret_cast<const TB*>(g.B) + b1 * g.sB + b2 * g.sB2;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s <= UST; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;

  // register prefetch of one K chunk: each warp fills whole core matrices (8 rows x 4 K),
  // lane -> (row lane / 4, k lane % 4), so a warp stores 128 contiguous bytes
  float ra[LA], rb[LB];
  const int nk = (g.K + UBK - 1) / UBK;
  auto fetch = [&](int kc) {
    const int k0 = kc * UBK;
#pragma unroll
    for (int p = 0; p < LA; ++p) {
      const int ci = warp + 8 * p, mi = ci & 15, ki = ci >> 4;
      const int m = m0 + 8 * mi + (lane >> 2), k = k0 + 4 * ki + (lane & 3);
      ra[p] = (m < g.M && k < g.K) ? ldf(A + m + g.lda * k) : 0.0f;
    }
#pragma unroll
    for (int p = 0; p < LB; ++p) {
      const int ci = warp + 8 * p, ni = ci % (NP / 8), ki = ci / (NP / 8);
      const int n = 8 * ni + (lane >> 2), k = k0 + 4 * ki + (lane & 3);
      rb[p] = (n < g.N && k < g.K) ? ldf(B + k + g.ldb * n) : 0.0f;
    }
  };
  auto stash = [&](int s) {
    uint8_t* st = usm + s * STAGE;
#pragma unroll
    for (int p = 0; p < LA; ++p) {
      const int ci = warp + 8 * p, mi = ci & 15, ki = ci >> 4;
      *reinterpret_cast<uint32_t*>(st + mi * 1024 + ki * 128 + lane * 4) = to_tf32(ra[p]);
    }
#pragma unroll
    for (int p = 0; p < LB; ++p) {
      const int ci = warp + 8 * p, ni = ci % (NP / 8), ki = ci / (NP / 8);
      *reinterpret_cast<uint32_t*>(st + A_BYTES + ni * 1024 + ki * 128 + lane * 4) = to_tf32(rb[p]);
    }
  };

  bool ok = true;
  if (nk > 0) fetch(0);
  for (int kc = 0; kc < nk; ++kc) {
    const int s = kc % UST;
    if (kc >= UST) {
      // every thread polls; the CTA leaves the loop together if any poll ran out
      const bool w = mbar_wait(&bars[s], (uint32_t)((kc / UST - 1) & 1));
      if (!__syncthreads_and(w)) {
        ok = false;
        break;
      }
    }
    stash(s);
    if (kc + 1 < nk) fetch(kc + 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t abase = smem_addr(usm + s * STAGE), bbase = abase + A_BYTES;
#pragma unroll
      for (int kk = 0; kk < UBK / 8; ++kk) {
        const uint64_t ad = sdesc(abase + kk * 256, 128, 1024);
        const uint64_t bd = sdesc(bbase + kk * 256, 128, 1024);
        umma_tf32(tmem, ad, bd, IDESC, (kc > 0 || kk > 0) ? 1u : 0u);
      }
      umma_commit(&bars[s]);
    }
  }
  // the last commit covers every MMA issued before it
  if (tid == 0) umma_commit(&bars[UST]);
  const bool fin = __syncthreads_and(mbar_wait(&bars[UST], 0));
  if ((!ok || !fin) && tid == 0) atomicExch(flag, EXA_UMMA_TIMEOUT);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok && fin) {
    // epilogue: warp w reads lanes 32 (w % 4) .. +31 (tile rows) and half of the columns
    const int q = warp & 3, h = warp >> 2;
    const int m = m0 + 32 * q + lane;
    TCO* C = reinterpret_cast<TCO*>(g.C) + b1 * g.sC + b2 * g.sC2;
    const TCI* Ci = reinterpret_cast<const TCI*>(g.Cin) + b1 * g.sCi + b2 * g.sCi2;
    constexpr int HC = NP / 2;
#pragma unroll
    for (int c0 = 0; c0 < HC; c0 += 16) {
      const int col = h * HC + c0;
      uint32_t v[16];
      const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)col;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < g.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = col + j;
          if (n < g.N) {
            double r = g.alpha * (double)__uint_as_float(v[j]);
            if (g.beta != 0.0) r += g.beta * (double)Ci[m + g.ldci * n];
            C[m + g.ldc * n] = (TCO)r;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
}

template <typename TA, typename TB, typename TCI, typename TCO, int NP>
int launch_umma(const UGemm& g, int* flag, cudaStream_t st) {
  constexpr size_t smem = (size_t)UST * (UM * UBK * 4 + NP * UBK * 4) + (UST + 1) * 8 + 16;
  static_assert(smem <= 227 * 1024, "tile exceeds shared memory");
  auto kern = umma_gemm_kernel<TA, TB, TCI, TCO, NP>;
  EXA_TRY(exa_allow_smem((const void*)kern, smem));
  EXA_CUDA(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared));
  dim3 grid((unsigned)exa_ceil_div(g.M, UM), (unsigned)g.batch, (unsigned)g.batch2);
  kern<<<grid, UNT, smem, st>>>(g, flag);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

template <typename TA, typename TB, typename TCI, typename TCO>
int dispatch_np(const UGemm& g, int* flag, cudaStream_t st) {
  if (g.N <= 128) return launch_umma<TA, TB, TCI, TCO, 128>(g, flag, st);
  if (g.N <= 160) return launch_umma<TA, TB, TCI, TCO, 160>(g, flag, st);
  if (g.N <= 192) return launch_umma<TA, TB, TCI, TCO, 192>(g, flag, st);
  return launch_umma<TA, TB, TCI, TCO, 256>(g, flag, st);
}

}  // namespace

int exa_gemm_tf32(const UGemm& g, int* flag, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0 || g.batch2 <= 0) return EXA_OK;
  if (g.K <= 0) {
    exa_set_error("tf32 gemm: K = %d", g.K);
    return EXA_ERR_ARG;
  }
  if (g.N > 256) {
    exa_set_error("tf32 gemm: N = %d exceeds one 256-column tile", g.N);
    return EXA_ERR_ARG;
  }
  if (g.batch > 65535 || g.batch2 > 65535) {
    exa_set_error("tf32 gemm: batch dimensions %d x %d exceed the grid", g.batch, g.batch2);
    return EXA_ERR_ARG;
  }
  if (g.beta != 0.0 && g.Cin == nullptr) {
    exa_set_error("tf32 gemm: beta != 0 needs Cin");
    return EXA_ERR_ARG;
  }
  const int key = (g.ta == EXA_T_F64 ? 1 : 0) | (g.tb == EXA_T_F64 ? 2 : 0) | (g.tci == EXA_T_F64 ? 4 : 0) |
                  (g.tco == EXA_T_F64 ? 8 : 0);
  switch (key) {
    case 0: return dispatch_np<float, float, float, float>(g, flag, st);
    case 1 | 4: return dispatch_np<double, float, double, float>(g, flag, st);
    case 1: return dispatch_np<double, float, float, float>(g, flag, st);
    default:
      exa_set_error("tf32 gemm: operand type combination %d is not instantiated", key);
      return EXA_ERR_UNSUPPORTED;
  }
}

// ==================================================================================
// Packed operands and the 3xTF32 GEMM with bulk-copy staging.
//
// The register-staged kernel above spends about six instructions per operand element
// (load, two conversions, address, store) and is bound by instruction issue, not by the
// tensor cores.  Here the operands arrive pre-packed in the tcgen05 layout (hi and lo
// TF32 parts), so one thread moves each K chunk into shared memory with cp.async.bulk
// (completing on the stage's mbarrier through its transaction count), one thread issues
// the MMAs, and four warps run the epilogue: no per-element staging instructions.
// ==================================================================================
namespace {

// shared-memory ring: 3 stages for N tiles up to 160 (two CTAs per SM); 2 stages for 256,
// so that two CTAs still share an SM and one's epilogue overlaps the other's main loop
constexpr int PNT = 128;  // threads (4 warps: epilogue lanes 0..127)

// one CTA per (batch entry, row tile): lane l of a warp takes row 32 rb + l of the tile and
// four consecutive k, so a warp's loads of one k are 32 consecutive rows of a column-major
// source and its float4 stores fill whole 128-byte rows of four core matrices.  Offsets
// within the tile follow pack_off with the tile's group count fixed once, without
// divisions in the loop.
template <typename TS>
__global__ void __launch_bounds__(256) pack_kernel(const TS* src, long long rs, long long ks, long long sb,
                                                   long long sb2, int batch2, int ntiles, UPacked d, int kgp,
                                                   int kgs) {
  const int t = blockIdx.x % ntiles;
  const long long e = blockIdx.x / ntiles;
  const long long b2 = e % batch2, b1 = e / batch2;
  const TS* X = src + b1 * sb + b2 * sb2;
  const int nkc = (d.K + PK - 1) / PK;
  const long long tbase = b1 * d.sb + b2 * d.sb2 + (long long)t * (d.TR / 8) * nkc * 128;
  float* hi = d.hi + tbase;
  float* lo = d.lo ? d.lo + tbase : nullptr;
  const int r0 = t * d.TR;
  const int rows_t = min(d.TR, d.R - r0), ng = (rows_t + 7) / 8;
  const int nrb = (ng * 8 + 31) / 32, nkq = nkc * 4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int kq = warp; kq < nkq; kq += blockDim.x >> 5) {
    const int k0 = 4 * kq;
    const long long ocol = (long long)(kq >> 2) * ng * 128 + (kq & 3) * 32;
    for (int rb = 0; rb < nrb; ++rb) {
      const int lr = 32 * rb + lane;
      if (lr >= ng * 8) break;
      const int row = r0 + lr;
      double x[4];
#pragma unroll
      for (int k4 = 0; k4 < 4; ++k4) {
        const int k = k0 + k4;
        // grouped K: packed k = g kgp + j holds source k = g kgs + j (j < kgs), else zero
        const int g = kgp ? k / kgp : 0, j = k - g * kgp;
        const bool kin = k < d.K && (kgp == 0 || j < kgs);
        const int sk = kgp ? g * kgs + j : k;
        x[k4] = (row < d.R && kin) ? (double)X[row * rs + (long long)sk * ks] : 0.0;
      }
      const long long o = ocol + (lr >> 3) * 128 + (lr & 7) * 4;
      if (!lo) {
        // FP32 operand (the GEMM splits it on chip)
        *reinterpret_cast<float4*>(hi + o) = make_float4((float)x[0], (float)x[1], (float)x[2], (float)x[3]);
        continue;
      }
      float4 h, l;
      split_tf32(x[0], h.x, l.x);
      split_tf32(x[1], h.y, l.y);
      split_tf32(x[2], h.z, l.z);
      split_tf32(x[3], h.w, l.w);
      *reinterpret_cast<float4*>(hi + o) = h;
      *reinterpret_cast<float4*>(lo + o) = l;
    }
  }
}

// Epilogue helpers shared by the 3xTF32 kernels.  epi_rowbase: the row-dependent parts of the
// packed outputs' offsets for row r of batch entry b1.  epi_write16: the 16 results x of row r,
// columns c0 .. c0 + 15 of the product, into the plain output C (already offset to the batch
// entry) and the packed outputs.
__device__ __forceinline__ void epi_rowbase(const UGemmP& g, long long b1, int r, long long (&pbase)[2],
                                            int (&png)[2]) {
#pragma unroll
  for (int o = 0; o < 2; ++o) {
    pbase[o] = 0;
    png[o] = 0;
    if (o >= g.nout) break;
    const UPackOut& po = g.out[o];
    if (po.as_b) {
      // row = global column, k = r: one tile of ng groups
      png[o] = (po.p.R + 7) / 8;
      pbase[o] = b1 * po.p.sb + (long long)(r >> 4) * png[o] * 128 + ((r >> 2) & 3) * 32 + (r & 3);
    } else {
      // row = r in tile t, k = global column
      const int t = r / po.p.TR, rl = r - t * po.p.TR;
      const int rows_t = min(po.p.TR, po.p.R - t * po.p.TR);
      const int nkc = (po.p.K + PK - 1) / PK;
      png[o] = (rows_t + 7) / 8;
      pbase[o] = b1 * po.p.sb + (long long)t * (po.p.TR / 8) * nkc * 128 + (rl >> 3) * 128 + (rl & 7) * 4;
    }
  }
}

template <typename TCO>
__device__ __forceinline__ void epi_write16(const UGemmP& g, TCO* C, long long b2, int r, int c0, const double (&x)[16],
                                            const long long (&pbase)[2], const int (&png)[2]) {
  if (C) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (c0 + j < g.N) C[r + g.ldc * (c0 + j)] = (TCO)x[j];
  }
#pragma unroll
  for (int o = 0; o < 2; ++o) {
    if (o >= g.nout) break;
    const UPackOut& po = g.out[o];
    if (!po.as_b && po.cmul == 1 && (po.cadd & 3) == 0) {
      // A operand, consecutive columns are consecutive k: 4 k of a core-matrix row are one
      // float4 (the packed K is zero-padded, so whole quads are written)
#pragma unroll
      for (int j = 0; j < 16; j += 4) {
        const int gc = c0 + j + g.n0 + (int)b2 * po.cadd;
        if (c0 + j >= g.N) break;
        const long long off = pbase[o] + (long long)(gc >> 4) * png[o] * 128 + ((gc >> 2) & 3) * 32;
        if (!po.p.lo) {
          // FP32 operand, split by the consumer on chip
          const float4 v = make_float4(c0 + j + 0 < g.N ? (float)x[j + 0] : 0.0f,
                                       c0 + j + 1 < g.N ? (float)x[j + 1] : 0.0f,
                                       c0 + j + 2 < g.N ? (float)x[j + 2] : 0.0f,
                                       c0 + j + 3 < g.N ? (float)x[j + 3] : 0.0f);
          *reinterpret_cast<float4*>(po.p.hi + off) = v;
          continue;
        }
        float4 h, l;
        split_tf32(c0 + j + 0 < g.N ? x[j + 0] : 0.0, h.x, l.x);
        split_tf32(c0 + j + 1 < g.N ? x[j + 1] : 0.0, h.y, l.y);
        split_tf32(c0 + j + 2 < g.N ? x[j + 2] : 0.0, h.z, l.z);
        split_tf32(c0 + j + 3 < g.N ? x[j + 3] : 0.0, h.w, l.w);
        *reinterpret_cast<float4*>(po.p.hi + off) = h;
        *reinterpret_cast<float4*>(po.p.lo + off) = l;
      }
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int c = c0 + j;
        if (c >= g.N) break;
        const int gc = (c + g.n0) * po.cmul + (int)b2 * po.cadd;
        const long long off = po.as_b ? pbase[o] + (gc >> 3) * 128 + (gc & 7) * 4
                                       : pbase[o] + (long long)(gc >> 4) * png[o] * 128 + ((gc >> 2) & 3) * 32 + (gc & 3);
        if (!po.p.lo) {
          po.p.hi[off] = (float)x[j];
          continue;
        }
        float h, l;
        split_tf32(x[j], h, l);
        po.p.hi[off] = h;
        po.p.lo[off] = l;
      }
    }
  }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

// SPLIT: both operands are stored as plain FP32 in the packed layout (lo == nullptr); the bulk
// copies land them in the hi slots, and warps 2..7 split each landed chunk in shared memory
// into hi = tf32(x) (in place) and lo = tf32(x - hi) before the MMAs read it.  Otherwise both
// operands arrive already split (hi and lo parts in HBM) and the CTA has 4 warps.
//
// RT = 2 (SPLIT only, 128 < M <= 256, NP <= 128): one CTA takes both 128-row tiles of A, so each
// K chunk of B is loaded and split once for both; tile t accumulates in tensor-memory columns
// t NP.  The second tile's slot holds only its row groups; its MMA reads 128 rows from there,
// and the rows past M, which come from the following bytes of the stage, are never read back.
//
// A stage holds [A tile 0 | A tile 1 | B] hi, then the same lo.  Warp 0 lane 0 issues the bulk
// copies, warp 1 lane 0 the MMAs.  In the epilogue warp w reads tensor-memory lanes 32 (w % 4)
// .. +31 (rows of a tile) and, with 8 warps, the column half w / 4.
template <int NP, int PST, typename TCI, typename TCO, bool SPLIT, int RT>
__global__ void __launch_bounds__(SPLIT ? 2 * PNT : PNT, 1) umma3_kernel(UGemmP g, int* flag) {
  static_assert(NP % 32 == 0 && NP >= 32 && NP <= 256, "N tile");
  static_assert(RT == 1 || (RT == 2 && SPLIT && NP <= 128), "row tiles per CTA");
  constexpr int NT = SPLIT ? 2 * PNT : PNT;
  constexpr int A_B = 16 * 512, B_B = (NP / 8) * 512;     // one part (hi or lo) of a full A tile, of B
  constexpr int TCOLS = RT * NP <= 32 ? 32 : (RT * NP <= 64 ? 64 : (RT * NP <= 128 ? 128 : (RT * NP <= 256 ? 256 : 512)));
  constexpr int NCONV = NT - 64;                           // converter threads (warps 2..7)
  constexpr int CA = (RT * A_B / 16 + NCONV - 1) / NCONV;  // float4 of A per converter thread
  constexpr int CB = (B_B / 16 + NCONV - 1) / NCONV;       // float4 of B per converter thread
  constexpr int NCOL = NP / (NT / 128);                    // epilogue columns per warp
  static_assert(NCOL % 16 == 0, "epilogue column split");
  constexpr uint32_t IDESC = idesc_tf32(UM, NP);
  extern __shared__ __align__(1024) uint8_t psm[];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long b1 = blockIdx.y, b2 = blockIdx.z;
  const int tA = blockIdx.x, m0 = tA * UM * RT;
  const int nkc = (g.K + PK - 1) / PK;
  // rows of each tile, their 8-row groups, and the stage layout (bytes)
  const int rows0 = min(UM, g.M - m0), rows1 = RT == 2 ? g.M - m0 - UM : 0;
  const int ngA0 = (rows0 + 7) / 8, ngA1 = (rows1 + 7) / 8;
  const int ngB = (g.N + 7) / 8;
  const int ngBt = (g.B.R + 7) / 8;  // groups of all of B's rows: the stride between K chunks
  const uint32_t bytesA0 = (uint32_t)ngA0 * 512, bytesA1 = (uint32_t)ngA1 * 512, bytesB = (uint32_t)ngB * 512;
  const uint32_t boff = RT == 2 ? A_B + bytesA1 : A_B;    // B's offset in a part
  const uint32_t HALF = boff + B_B, STAGE = 2 * HALF;
  uint64_t* full = reinterpret_cast<uint64_t*>(psm + PST * STAGE);
  uint64_t* empty = full + PST;
  uint64_t* conv = empty + PST;                            // SPLIT: chunk split into hi and lo
  uint64_t* done = conv + PST;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  int* abort_flag = reinterpret_cast<int*>(tslot + 1);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < PST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
      mbar_init(&conv[s], NCONV);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;

  // A tile t of this CTA starts (tA RT + t) tiles into the batch entry's A
  const long long abase = b1 * g.A.sb + b2 * g.A.sb2 + (long long)tA * RT * 16 * nkc * 128;
  const float* Ahi = g.A.hi + abase;
  const float* Bhi = g.B.hi + b1 * g.B.sb + b2 * g.B.sb2 + (long long)(g.n0 >> 3) * 128;
  const float* Alo = SPLIT ? nullptr : g.A.lo + abase;
  const float* Blo = SPLIT ? nullptr : g.B.lo + b1 * g.B.sb + b2 * g.B.sb2 + (long long)(g.n0 >> 3) * 128;

  const long long polls = g.main_wait_polls >= 0 ? g.main_wait_polls : WAIT_LIMIT;
  volatile int* ab = abort_flag;
  if (warp == 0 && lane == 0) {
    // producer: chunk kc into stage kc % PST once the MMAs of chunk kc - PST are done
    int issued = 0;
    for (int kc = 0; kc < nkc; ++kc) {
      const int s = kc % PST;
      if (kc >= PST && (*ab || !mbar_wait(&empty[s], (uint32_t)((kc / PST - 1) & 1), polls))) {
        atomicExch(abort_flag, 1);
        break;
      }
      uint8_t* st = psm + s * STAGE;
      if (SPLIT) {
        mbar_expect_tx(&full[s], bytesA0 + bytesA1 + bytesB);
        bulk_g2s(st, Ahi + (long long)kc * ngA0 * 128, bytesA0, &full[s]);
        if (RT == 2) bulk_g2s(st + A_B, Ahi + (long long)16 * nkc * 128 + (long long)kc * ngA1 * 128, bytesA1, &full[s]);
        bulk_g2s(st + boff, Bhi + (long long)kc * ngBt * 128, bytesB, &full[s]);
      } else {
        mbar_expect_tx(&full[s], 2 * (bytesA0 + bytesB));
        bulk_g2s(st, Ahi + (long long)kc * ngA0 * 128, bytesA0, &full[s]);
        bulk_g2s(st + HALF, Alo + (long long)kc * ngA0 * 128, bytesA0, &full[s]);
        bulk_g2s(st + boff, Bhi + (long long)kc * ngBt * 128, bytesB, &full[s]);
        bulk_g2s(st + HALF + boff, Blo + (long long)kc * ngBt * 128, bytesB, &full[s]);
      }
      issued = kc + 1;
    }
    // after an abort, copies may still be in flight into stages nobody consumes: wait (at the
    // normal limit) for the latest phase of every stage this loop armed, so that no copy lands
    // in shared memory after the CTA has left.  Those are the stages' newest phases (nothing
    // re-arms them later), so a completed one reads as complete.
    if (*ab)
      for (int q = max(0, issued - PST); q < issued; ++q) mbar_wait(&full[q % PST], (uint32_t)((q / PST) & 1));
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: hi*hi + hi*lo + lo*hi per K step of 8 and row tile
    for (int kc = 0; kc < nkc; ++kc) {
      const int s = kc % PST;
      if (*ab || !mbar_wait(SPLIT ? &conv[s] : &full[s], (uint32_t)((kc / PST) & 1), polls)) {
        atomicExch(abort_flag, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_hi = smem_addr(psm + s * STAGE), b_hi = a_hi + boff;
      const uint32_t a_lo = a_hi + HALF, b_lo = b_hi + HALF;
#pragma unroll
      for (int kk = 0; kk < PK / 8; ++kk) {
        const uint32_t o = kk * 256;
        const uint32_t acc_in = (kc > 0 || kk > 0) ? 1u : 0u;
#pragma unroll
        for (int t = 0; t < RT; ++t) {
          // tile 1's groups are ngA1 long per chunk: its k-step offset is the same 256 bytes
          const uint32_t ta = (uint32_t)(t * A_B);
          const uint32_t acc = tmem + (uint32_t)(t * NP);
          umma_tf32(acc, sdesc(a_hi + ta + o, 128, 512), sdesc(b_hi + o, 128, 512), IDESC, acc_in);
          umma_tf32(acc, sdesc(a_hi + ta + o, 128, 512), sdesc(b_lo + o, 128, 512), IDESC, 1u);
          umma_tf32(acc, sdesc(a_lo + ta + o, 128, 512), sdesc(b_hi + o, 128, 512), IDESC, 1u);
        }
      }
      umma_commit(&empty[s]);
    }
    umma_commit(done);  // tracks every MMA issued above
  } else if (SPLIT && warp >= 2) {
    // converters: once chunk kc has landed, split it in place (hi) and into the lo slots, make
    // the writes visible to the tensor cores' (async) proxy, then arrive on conv[s].  Each
    // thread loads all its float4 of the chunk before converting any (one shared-memory round
    // trip per chunk)
    const int ct = tid - 64;
    const int na = (int)((bytesA0 + bytesA1) >> 4), nbq = (int)(bytesB >> 4);  // A tiles are adjacent
    for (int kc = 0; kc < nkc; ++kc) {
      const int s = kc % PST;
      if (*ab || !mbar_wait(&full[s], (uint32_t)((kc / PST) & 1), polls)) {
        atomicExch(abort_flag, 1);
        break;
      }
      float4* hp = reinterpret_cast<float4*>(psm + s * STAGE);   // A hi, then B hi at boff
      float4 x[CA + CB];
#pragma unroll
      for (int u = 0; u < CA; ++u)
        if (ct + NCONV * u < na) x[u] = hp[ct + NCONV * u];
#pragma unroll
      for (int u = 0; u < CB; ++u)
        if (ct + NCONV * u < nbq) x[CA + u] = hp[boff / 16 + ct + NCONV * u];
#pragma unroll
      for (int u = 0; u < CA + CB; ++u) {
        const int i = u < CA ? ct + NCONV * u : ct + NCONV * (u - CA);
        if (i >= (u < CA ? na : nbq)) continue;
        const int o = u < CA ? i : (int)(boff / 16) + i;
        float4 h, l;
        split_tf32f(x[u].x, h.x, l.x);
        split_tf32f(x[u].y, h.y, l.y);
        split_tf32f(x[u].z, h.z, l.z);
        split_tf32f(x[u].w, h.w, l.w);
        hp[o] = h;
        hp[o + HALF / 16] = l;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&conv[s]);
    }
  }
  __syncwarp();
  const bool fin = mbar_wait(done, 0);
  const bool ok = __syncthreads_and(fin && *abort_flag == 0);
  if (!ok && tid == 0) atomicExch(flag, EXA_UMMA_TIMEOUT);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const int wq = warp & 3, cpart = warp >> 2;
#pragma unroll 1
  for (int t = 0; ok && t < RT; ++t) {
    if (m0 + UM * t + 32 * wq >= g.M) continue;  // no row of this warp in tile t (warp-uniform)
    const int r = m0 + UM * t + 32 * wq + lane;
    const bool rv = r < g.M;
    TCO* C = reinterpret_cast<TCO*>(g.C);
    const TCI* Ci = reinterpret_cast<const TCI*>(g.Cin);
    if (C) C += b1 * g.sC + b2 * g.sC2;
    if (Ci) Ci += b1 * g.sCi + b2 * g.sCi2;
    const bool use_cin = g.beta != 0.0;
    long long pbase[2];
    int png[2];
    epi_rowbase(g, b1, r, pbase, png);
#pragma unroll 1
    for (int c0 = cpart * NCOL; c0 < (cpart + 1) * NCOL; c0 += 16) {
      if (c0 >= g.N) break;  // warp-uniform
      uint32_t v[16];
      tmem_ld16(tmem + ((uint32_t)(32 * wq) << 16) + (uint32_t)(t * NP + c0), v);
      // Cin of the 16 columns first: independent loads in flight together
      double x[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int c = c0 + j;
        x[j] = (use_cin && rv && c < g.N) ? (double)Ci[r + g.ldci * c] : 0.0;
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 16; ++j) x[j] = g.alpha * (double)__uint_as_float(v[j]) + g.beta * x[j];
      if (rv) epi_write16<TCO>(g, C, b2, r, c0, x, pbase, png);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
}

template <int NP, int PST, typename TCI, typename TCO, bool SPLIT, int RT = 1>
int launch_umma3(const UGemmP& g, int* flag, cudaStream_t st) {
  // a stage: full A tile(s) (the second of RT = 2 only as many row groups as it has) and B,
  // hi and lo parts
  constexpr size_t smax = (size_t)PST * 2 * (RT * 16 * 512 + (NP / 8) * 512) + (3 * PST + 1) * 8 + 16;
  static_assert(smax <= 227 * 1024, "tile exceeds shared memory");
  const size_t a1 = RT == 2 ? (size_t)((g.M - UM + 7) / 8) * 512 : 0;
  const size_t smem = (size_t)PST * 2 * (16 * 512 + a1 + (NP / 8) * 512) + (3 * PST + 1) * 8 + 16;
  constexpr int NT = SPLIT ? 2 * PNT : PNT;
  auto kern = umma3_kernel<NP, PST, TCI, TCO, SPLIT, RT>;
  EXA_TRY(exa_allow_smem((const void*)kern, smem));
  EXA_CUDA(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared));
  dim3 grid((unsigned)exa_ceil_div(g.M, UM * RT), (unsigned)g.batch, (unsigned)g.batch2);
  kern<<<grid, NT, smem, st>>>(g, flag);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

template <typename TCI, typename TCO, bool SPLIT>
int umma3_np(const UGemmP& g, int* flag, cudaStream_t st) {
  // two row tiles of up to 256 rows in one CTA, so B is loaded and split once for both
  if constexpr (SPLIT)
    if (g.N <= 128 && g.M > UM && g.M <= 2 * UM) return launch_umma3<128, 3, TCI, TCO, SPLIT, 2>(g, flag, st);
  if (g.N <= 128) return launch_umma3<128, 3, TCI, TCO, SPLIT>(g, flag, st);
  if (g.N <= 160) return launch_umma3<160, 3, TCI, TCO, SPLIT>(g, flag, st);
  return launch_umma3<256, 2, TCI, TCO, SPLIT>(g, flag, st);
}

}  // namespace

namespace {
std::atomic<long long> g_umma_wait_polls{-1};
}

void exa_umma_set_wait_polls(long long polls) { g_umma_wait_polls.store(polls); }
long long exa_umma_wait_polls() { return g_umma_wait_polls.load(); }

long long exa_pack_size(int R, int K) { return (long long)((R + 7) / 8) * ((K + PK - 1) / PK) * 128; }

int exa_pack(const void* src, int src_f64, long long rs, long long ks, long long sb, long long sb2, int batch,
             int batch2, const UPacked& d, cudaStream_t st, int kgp, int kgs) {
  if (batch <= 0 || batch2 <= 0 || d.R <= 0 || d.K <= 0) return EXA_OK;
  if (kgp < 0 || kgs < 0 || kgs > kgp || (kgp > 0 && kgs == 0)) {
    exa_set_error("pack: K groups of %d holding %d source entries", kgp, kgs);
    return EXA_ERR_ARG;
  }
  if (d.TR % 8 != 0) {
    exa_set_error("pack: tile height %d is not a multiple of 8", d.TR);
    return EXA_ERR_ARG;
  }
  const int ntiles = (d.R + d.TR - 1) / d.TR;
  if ((long long)batch * batch2 * ntiles > 0x7fffffffLL) {
    exa_set_error("pack: %d x %d batch entries exceed the grid", batch, batch2);
    return EXA_ERR_ARG;
  }
  const unsigned grid = (unsigned)((long long)batch * batch2 * ntiles);
  if (src_f64)
    pack_kernel<double><<<grid, 256, 0, st>>>((const double*)src, rs, ks, sb, sb2, batch2, ntiles, d, kgp, kgs);
  else
    pack_kernel<float><<<grid, 256, 0, st>>>((const float*)src, rs, ks, sb, sb2, batch2, ntiles, d, kgp, kgs);
  EXA_LAUNCH_CHECK();
  return EXA_OK;
}

int exa_gemm_3xtf32(const UGemmP& g, int* flag, cudaStream_t st) {
  if (g.N > 256) {
    // column chunks of 256: B rows, C and Cin columns and packed-output indices shift by n0
    for (int c0 = 0; c0 < g.N; c0 += 256) {
      UGemmP h = g;
      h.N = (g.N - c0) < 256 ? (g.N - c0) : 256;
      h.n0 = g.n0 + c0;
      if (h.C) h.C = (char*)h.C + (long long)(h.tco == EXA_T_F64 ? 8 : 4) * h.ldc * c0;
      if (h.Cin) h.Cin = (const char*)h.Cin + (long long)(h.tci == EXA_T_F64 ? 8 : 4) * h.ldci * c0;
      EXA_TRY(exa_gemm_3xtf32(h, flag, st));
    }
    return EXA_OK;
  }
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0 || g.batch2 <= 0) return EXA_OK;
  // the kernel locates chunks from M and N, so the packed operands must have exactly those
  // rows; batch strides keep every chunk on a 16-byte boundary for the bulk copies
  // B's rows n0 .. n0 + N - 1 are read from one tile of all its rows; chunks start on a group
  if (g.K <= 0 || g.N > 256 || g.A.K != g.K || g.B.K != g.K || g.A.TR != UM || g.B.TR < g.B.R || g.A.R != g.M ||
      g.n0 < 0 || (g.n0 & 7) != 0 || g.B.R < g.n0 + g.N ||
      (!g.A.lo) != (!g.B.lo) || g.nout < 0 || g.nout > 2 || (g.beta != 0.0 && !g.Cin) ||
      (g.A.sb | g.A.sb2 | g.B.sb | g.B.sb2) % 4 != 0) {
    exa_set_error("3xtf32 gemm: inconsistent operand description (M %d N %d K %d)", g.M, g.N, g.K);
    return EXA_ERR_ARG;
  }
  if (g.batch > 65535 || g.batch2 > 65535) {
    exa_set_error("3xtf32 gemm: batch dimensions %d x %d exceed the grid", g.batch, g.batch2);
    return EXA_ERR_ARG;
  }
  for (int o = 0; o < g.nout; ++o) {
    const UPackOut& po = g.out[o];
    // B-operand outputs hold all their rows in one tile; A-operand outputs with unit column
    // step are written in aligned quads of k
    const bool bad = po.as_b ? (po.p.TR < po.p.R || po.p.K < g.M)
                             : (po.p.TR != UM || po.p.R < g.M);
    if (bad || po.p.sb % 4 != 0 || !po.p.hi) {
      exa_set_error("3xtf32 gemm: packed output %d does not fit the product", o);
      return EXA_ERR_ARG;
    }
  }
  UGemmP h = g;
  h.main_wait_polls = exa_umma_wait_polls();
  const bool ci64 = g.tci == EXA_T_F64, co64 = g.tco == EXA_T_F64, split = !g.A.lo;
  if (ci64 && !co64) return split ? umma3_np<double, float, true>(h, flag, st) : umma3_np<double, float, false>(h, flag, st);
  if (!ci64 && !co64) return split ? umma3_np<float, float, true>(h, flag, st) : umma3_np<float, float, false>(h, flag, st);
  exa_set_error("3xtf32 gemm: FP64 output is not instantiated");
  return EXA_ERR_UNSUPPORTED;
}

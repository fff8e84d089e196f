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
#include <cstdint>

#include "exa_common.cuh"
#include "exa_umma.cuh"

namespace {

constexpr int UM = 128;      // tile rows (tcgen05 M)
constexpr int UBK = 32;      // K values per stage
constexpr int UST = 3;       // stages
constexpr int UNT = 256;     // threads
constexpr long long WAIT_LIMIT = 1ll << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: K-major, no swizzle (layout type 0), version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor, kind::tf32: D FP32, A and B TF32, both K-major, N >> 3, M >> 4
__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

// true once the phase with the given parity has completed; false after WAIT_LIMIT polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_addr(bar);
  for (long long i = 0; i < WAIT_LIMIT; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

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
  EXA_CUDA(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
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

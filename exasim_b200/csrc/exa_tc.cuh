// Device helpers for the tcgen05 kernels (5th-generation tensor cores): shared-memory
// matrix and instruction descriptors, TF32 rounding and hi/lo splitting, bounded mbarrier
// waits, MMA issue and commit, bulk copies, and the packed operand layout.
#pragma once
#include <cstdint>

namespace exa_tc {

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

// true once the phase with the given parity has completed; false after `limit` polls
// (WAIT_LIMIT unless a caller passes another; 0 polls gives false at once)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit = WAIT_LIMIT) {
  const uint32_t a = smem_addr(bar);
  for (long long i = 0; i < limit; ++i) {
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

constexpr int PK = 16;  // K per chunk of a packed operand

// K index of the q elimination's packed operands (B, G, Minv C, Minv E): node j of gradient
// component d sits at k = j + qk_group(npe) d.  Groups are rounded up to whole quads of k, so
// each starts on a 16-byte boundary of a core-matrix row and a writer can store float4s; the
// padding holds zeros in both operands of a product.
__host__ __device__ inline int qk_group(int npe) { return (npe + 3) & ~3; }

__host__ __device__ inline long long pack_off(int row, int k, int R, int K, int TR) {
  const int nkc = (K + PK - 1) / PK;
  const int t = row / TR, rl = row - t * TR;
  const int rows_t = (R - t * TR) < TR ? (R - t * TR) : TR;
  const int ng = (rows_t + 7) / 8;
  const int kc = k / PK, kl = k - kc * PK;
  return (long long)t * (TR / 8) * nkc * 128 + (long long)kc * ng * 128 + (rl >> 3) * 128 + (kl >> 2) * 32 +
         (rl & 7) * 4 + (kl & 3);
}

__device__ __forceinline__ void split_tf32(double x, float& hi, float& lo) {
  const uint32_t h = to_tf32((float)x);
  hi = __uint_as_float(h);
  lo = __uint_as_float(to_tf32((float)(x - (double)hi)));
}

// hi = tf32(x), lo = tf32(x - hi) for an FP32 x: x - hi is exact in FP32
__device__ __forceinline__ void split_tf32f(float x, float& hi, float& lo) {
  hi = __uint_as_float(to_tf32(x));
  lo = __uint_as_float(to_tf32(x - hi));
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}


}  // namespace exa_tc

// Batched TF32 tensor-core GEMM (tcgen05) for the mixed-precision element elimination.
#pragma once
#include <cuda_runtime.h>

enum { EXA_T_F32 = 0, EXA_T_F64 = 1 };
// value written to the kernel's flag when an mbarrier wait ran out
enum { EXA_UMMA_TIMEOUT = 2 };

// Cout(r, c) = alpha * sum_k A(r, k) B(k, c) + beta * Cin(r, c) for every batch entry
// (b1, b2), column-major with the strides of GemmBatch; operands rounded to TF32, products
// accumulated in FP32.  Element types: A, B, Cin, Cout each FP32 or FP64 (EXA_T_*).
// N <= 256 (one tile of columns); M is tiled by 128.  Cin may alias Cout when both have
// the same type; Cin is not read when beta == 0.
struct UGemm {
  int M, N, K;
  double alpha, beta;
  const void* A; int ta; long long lda, sA, sA2;
  const void* B; int tb; long long ldb, sB, sB2;
  const void* Cin; int tci; long long ldci, sCi, sCi2;
  void* C; int tco; long long ldc, sC, sC2;
  int batch, batch2;
};

// *flag (device int) is set to EXA_UMMA_TIMEOUT if a wait inside the kernel ran out.
int exa_gemm_tf32(const UGemm& g, int* flag, cudaStream_t st);

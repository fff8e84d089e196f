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

// ---- packed operands (3xTF32) -------------------------------------------------------
// An operand X(row, k) with R rows and K reduction values is stored pre-packed in the
// canonical K-major layout of tcgen05, split into hi = tf32(x) and lo = tf32(x - hi):
//   tiles of TR rows (128 for A operands; one tile of all N rows for B operands), each
//   tile as K chunks of 16, each chunk as ceil(rows/8) groups of 8 rows x 16 k, each
//   group as 4 core matrices of 8 rows x 4 k (128 bytes).  Rows past R and k past K are
//   zero.  Floats per batch entry: ceil(R/8) * ceil(K/16) * 128 when TR is a multiple of 8.
// With lo == nullptr the operand is stored once, as FP32 values in hi, and the 3xTF32 GEMM
// splits each chunk into hi and lo parts in shared memory (half the bytes in HBM).
struct UPacked {
  float* hi;
  float* lo;
  long long sb, sb2;  // batch strides in floats
  int R, K, TR;
};
long long exa_pack_size(int R, int K);  // floats per batch entry

// Pack X(r, k) = src[b1 sb + b2 sb2 + r rs + k ks] (FP64 or FP32) for b1 < batch, b2 < batch2.
// With kgp > 0 the packed K comes in groups of kgp: packed k = g kgp + j holds source
// k = g kgs + j for j < kgs and zero for kgs <= j < kgp.
int exa_pack(const void* src, int src_f64, long long rs, long long ks, long long sb, long long sb2, int batch,
             int batch2, const UPacked& dst, cudaStream_t st, int kgp = 0, int kgs = 0);

// Packed-output description for a GEMM epilogue: C(r, c) is also stored as a packed
// operand of a later GEMM, either as an A operand (row r, k = global column) or as a B
// operand (row = global column, k = r).  global column = c * cmul + b2 * cadd; the packed
// batch index is b1.
struct UPackOut {
  UPacked p;
  int as_b;  // 0: A operand (row r, k col); 1: B operand (row col, k r)
  int cmul, cadd;
};

// Cout = alpha A B + beta Cin with A (R = M, tiles of 128) and B (R = N, one tile) packed, both
// split (hi and lo given) or both FP32 (lo null; split on chip); packed outputs in either form;
// the products hi*hi + hi*lo + lo*hi on the TF32 tensor cores, accumulated in FP32.
// Plain output C (FP32 or FP64, column-major) and up to two packed outputs, each optional.
struct UGemmP {
  int M, N, K;
  double alpha, beta;
  UPacked A, B;       // batch strides per b1 and b2
  const void* Cin; int tci; long long ldci, sCi, sCi2;
  void* C; int tco; long long ldc, sC, sC2;
  UPackOut out[2]; int nout;
  int batch, batch2;
  int n0;  // first column: the product covers columns n0 .. n0 + N - 1 of B, C and Cin (set by the host for N > 256)
  long long main_wait_polls;  // polls per main-loop wait; set by exa_gemm_3xtf32 from exa_umma_wait_polls()
};
// Polls per wait in the main loops of the 3xTF32 GEMM (negative: the normal limit).  Tests of the
// timeout path set 0, so every main-loop wait gives up at once; the waits that drain copies and
// MMAs already in flight keep the normal limit.
void exa_umma_set_wait_polls(long long polls);
long long exa_umma_wait_polls();
// N above 256 runs as column chunks of at most 256 (one launch each).
int exa_gemm_3xtf32(const UGemmP& g, int* flag, cudaStream_t st);

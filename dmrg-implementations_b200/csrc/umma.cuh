// Split-precision GEMM on the 5th-generation tensor cores (tcgen05, kind::f16).
//
// C = alpha op(A) op(B) + beta C for FP64 (or complex128) operands, computed as
// a three-term BF16 split of each operand, X = X1 + X2 + X3 with
// X1 = bf16(X), X2 = bf16(X - X1), X3 = bf16(X - X1 - X2), and the six
// products A_i B_j with i + j <= 4 accumulated in FP32 in tensor memory. The
// relative error per product term is ~2^-24 (FP32 level); the result is
// written back in FP64. Complex operands use the real embedding
// [Cr; Ci] = [[Ar, -Ai], [Ai, Ar]] [Br; Bi].
#pragma once

#include "common.cuh"

namespace dmrg2 {

// Device scratch for the BF16 pieces of one GEMM (grown on demand, owned by the caller).
struct SplitScratch {
  void* p = nullptr;
  size_t bytes = 0;
  int* err = nullptr;  // device flag: set when a tensor-core wait timed out
  void reserve(size_t b, cudaStream_t s);  // s: the stream the pieces are used on
  void release();
};

// op(A): trans 0 = N, 1 = T, 2 = C (conjugate transpose), 3 = conjugate. Row-major
// storage, leading dimensions in elements, nbatch strided batches (sA, sB, sC); an
// operand with batch stride 0 is split once and shared by all batches. Every kernel
// returns at once when *skip is nonzero (device flag, may be null).
template <typename T>
void gemm_bf16x3(int ta, int tb, int M, int N, int K, T alpha, const T* A, ll lda, ll sA, const T* B,
                 ll ldb, ll sB, T beta, T* C, ll ldc, ll sC, int nbatch, SplitScratch& ws, cudaStream_t s,
                 const int* skip = nullptr);

}  // namespace dmrg2

// Kernel argument blocks and launchers of the radiation surrogate (internal to
// librrtmg_b200.so).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace rrtmg {

enum GemmEpilogue { kEpiF32 = 0, kEpiGelu = 1, kEpiDgelu = 2 };

// C[M x N] = A[M x K] * B[N x K]^T; M, N multiples of 128, K a multiple of
// 64 * ksplit, leading dimensions multiples of 8 elements.
struct GemmArgs {
  const __nv_bfloat16 *A;
  int lda;
  const __nv_bfloat16 *B;
  int ldb;
  int M, N, K, ksplit;
  int epi;
  const float *bias;  // [N] or null
  float *C;           // kEpiF32: slab z at C + z * split_stride, row stride ldc
  int ldc;
  size_t split_stride;
  __nv_bfloat16 *H;   // kEpiGelu / kEpiDgelu: row-major [M][ldh]
  int ldh;
  __nv_bfloat16 *Ht;  // transposed [N][ldht]
  int ldht;
  const float *aux;   // kEpiDgelu: pre-activation Z [M][ldaux]
  int ldaux;
  float *Z;           // kEpiGelu: pre-activation output [M][ldz]
  int ldz;
};

cudaError_t launch_umma_gemm(const GemmArgs &g, cudaStream_t stream);
// Reads (and optionally clears) the sticky flag set when a GEMM CTA gave up
// waiting for its tensor-core work.
cudaError_t gemm_error_flag(unsigned *out, bool reset);

}  // namespace rrtmg

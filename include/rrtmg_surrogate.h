/*
 * rrtmg_surrogate: C-ABI of the learned radiation surrogate's GPU kernels
 * (hand-written tcgen05 BF16 GEMMs with fused MLP epilogues, loss, Adam, and
 * the per-column gate).  No counterpart in the reference: WRF-JAX has no
 * surrogate.  All pointers are device pointers; calls are asynchronous on the
 * given cudaStream_t (void*), and return rrtmg_status codes of rrtmg_b200.h.
 */
#ifndef RRTMG_SURROGATE_H
#define RRTMG_SURROGATE_H

#include <stddef.h>
#include <stdint.h>

#include "rrtmg_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { RRTMG_EPI_F32 = 0, RRTMG_EPI_GELU = 1, RRTMG_EPI_DGELU = 2 };

/* C[M x N] = A[M x K] * B[N x K]^T with A, B row-major BF16 and FP32
 * accumulation in tensor memory.  M and N multiples of 128; K a multiple of
 * 64 * ksplit; lda, ldb multiples of 8; 16-byte aligned A and B.
 *   RRTMG_EPI_F32:   C + z * split_stride [M][ldc] = partial sum of K split z
 *                    (+ bias[N] on split 0).
 *   RRTMG_EPI_GELU:  Z[M][ldz] = acc + bias (FP32, optional), H[M][ldh] and
 *                    Ht[N][ldht] = BF16 GELU(Z) (each optional).
 *   RRTMG_EPI_DGELU: H and Ht = BF16 acc * GELU'(aux[M][ldaux]).  */
typedef struct {
    const void *A; int lda;
    const void *B; int ldb;
    int M, N, K, ksplit, epilogue;
    const float *bias;
    float *C; int ldc; size_t split_stride;
    void *H; int ldh;
    void *Ht; int ldht;
    const float *aux; int ldaux;
    float *Z; int ldz;
} rrtmg_gemm_args;

rrtmg_status rrtmg_gemm_bf16(const rrtmg_gemm_args *args, void *stream);

/* Synchronous: reads the sticky flag that a GEMM CTA sets when it gives up
 * waiting (2 s) for its tensor-core work; clears it when reset != 0. */
rrtmg_status rrtmg_gemm_error(int reset, unsigned *flag);

#ifdef __cplusplus
}
#endif
#endif /* RRTMG_SURROGATE_H */

// Kernel argument blocks and launchers of the radiation surrogate (internal to
// librrtmg_b200.so).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/rrtmg_surrogate.h"

namespace rrtmg {

#ifdef __CUDACC__
// Decode arithmetic shared by rrtmg_sur_decode and the fused inference
// kernel, so both give the same bits.  The surrogate's outputs are
// approximations, so these use multiplications by constant reciprocals and
// one fast division instead of correctly rounded divisions (whose slow path
// every zero night-time SW rate takes).
// heatfac = g * 86400 / (cp * 100): K/day per (W/m2 per hPa)  (lw:5706, sw:2289)
constexpr float kSurHeatfac = (9.8066f * 8.6400e4f) / (1004.5f * 1.0e2f);
constexpr float kSurInvHeatfac = 1.0f / kSurHeatfac;
constexpr float kSurInvDay = 1.0f / 86400.0f;
// theta tendency [K/s] of a heating rate hr [K/day] at Exner function pi
__device__ __forceinline__ float sur_tendency(float hr, float pi) { return __fdividef(hr * kSurInvDay, pi); }
// flux divergence [W/m2] of heating rate hr over a layer of dp [hPa]
__device__ __forceinline__ float sur_flux_term(float hr, float dp) { return hr * dp * kSurInvHeatfac; }
#endif

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
  unsigned long long wait_ns;  // limit of each bounded mbarrier wait
  int withhold_commit0;        // failure-detection test: skip the commit of K block 0
  float *Z;           // kEpiGelu: pre-activation output [M][ldz]
  int ldz;
};

cudaError_t launch_umma_gemm(const GemmArgs &g, cudaStream_t stream);
// pipeline stages of the GEMM tile an N selects (the test hook's K bound)
int gemm_stages(int n);

using SurFeatureArgs = rrtmg_sur_features_args;
using SurTargetArgs = rrtmg_sur_targets_args;
using SurAdamArgs = rrtmg_sur_adam_args;
using SurDecodeArgs = rrtmg_sur_decode_args;
using SurMlpArgs = rrtmg_sur_mlp_args;
cudaError_t launch_sur_features(const SurFeatureArgs &a, cudaStream_t s);
cudaError_t launch_sur_targets(const SurTargetArgs &a, cudaStream_t s);
cudaError_t launch_sur_column_stats(const float *F, int n, int ld, int nf, float *mean, float *rstd, float *lo,
                                    float *hi, cudaStream_t s);
cudaError_t launch_sur_normalize(const float *in, int ldi, int n, int nf, const float *mean, const float *rstd,
                                 void *out, int ldo, int out_bf16, cudaStream_t s);
cudaError_t launch_sur_gather(const __nv_bfloat16 *X, int ldx, const float *T, int ldt, const int *idx, int B,
                              __nv_bfloat16 *Xb, __nv_bfloat16 *Xbt, int ldxbt, float *Tb, cudaStream_t s);
cudaError_t launch_sur_loss_grad(const float *Y, const float *T, const float *w, int B, int ld, float scale,
                                 __nv_bfloat16 *dY, __nv_bfloat16 *dYt, int lddyt, float *loss, cudaStream_t s);
cudaError_t launch_sur_row_sum(const __nv_bfloat16 *Gt, int ld, int rows, int B, float *db, cudaStream_t s);
cudaError_t launch_sur_reduce_splits(const float *P, int splits, size_t n, float *G, cudaStream_t s);
cudaError_t launch_sur_adam(const SurAdamArgs &a, cudaStream_t s);
cudaError_t launch_sur_decode(const SurDecodeArgs &a, cudaStream_t s);
cudaError_t launch_sur_compact(const unsigned *flags, int ncol, int *list, int *count, cudaStream_t s);
cudaError_t launch_sur_move_columns(const int *list, const int *count, int max_n, int nz, int ny, const float *src,
                                    float *dst, int to_compact, int stride, int offset, cudaStream_t s);
cudaError_t launch_sur_move_fields(const int *list, const int *count, int max_n, int ny, const rrtmg_sur_fields &f,
                                   int to_compact, int stride, int offset, cudaStream_t s);
void set_gemm_tile(int bn);
cudaError_t launch_timestamp(unsigned long long *slot, cudaStream_t s);
// Reads (and optionally clears) the sticky flag set when a GEMM CTA gave up
// waiting for its tensor-core work.
cudaError_t gemm_error_flag(unsigned *out, bool reset);
// Fused inference (surrogate_mlp.cu) and its weight packing and error flag.
size_t sur_weight_image_bytes();
cudaError_t launch_sur_pack_weights(const void *const W[4], void *image, cudaStream_t s);
cudaError_t launch_sur_mlp(const SurMlpArgs &a, cudaStream_t s);
cudaError_t mlp_error_flag(unsigned *out, bool reset);

}  // namespace rrtmg

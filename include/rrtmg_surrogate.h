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
 * 64 * ksplit; lda, ldb, ldh multiples of 8 and ldc, ldz, ldaux, split_stride
 * multiples of 4; every pointer 16-byte aligned.
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

/* Features of the columns of one WRF-layout domain (nx * ny = ncol columns,
 * nk levels) into rows row_offset .. row_offset + ncol - 1.  Per level k, at
 * f * nk + k: f = 0 t3d, 1 ln p3d, 2 qv, 3 qc, 4 qi, 5 qs, 6 cldfra, 7 o3,
 * 8 layer thickness p8w[k] - p8w[k+1]; then tsk, albedo, coszr, emiss
 * (9 nk + 4 features).  raw: FP32 values; X: BF16 (v - mean) * rstd, zero-
 * padded to ldx; Xt: X transposed; flags[c] = 1 when a value lies outside
 * [lo, hi] (the training range), else 0.  Every output is optional.
 * x_layout 0: X row-major [rows][ldx].  x_layout 1 (ldx = 512, X 16-byte
 * aligned, no raw or Xt): X as the feature tiles of rrtmg_sur_mlp: row
 * r = row_offset + c lies in tile r / 128 (128 KB per tile), whose eight
 * 16 KB blocks hold K = 64 b .. 64 b + 63 of its 128 rows, row r mod 128 at
 * (r mod 128) * 128 bytes with 16-byte chunk q (8 features) stored at chunk
 * position q XOR (r mod 8). */
typedef struct {
    int ncol, nk, ny;
    const float *p3d, *p8w, *t3d, *qv, *qc, *qi, *qs, *cldfra, *o3, *tsk, *albedo, *coszr, *emiss;
    int row_offset;
    float *raw; int ldf;
    const float *mean, *rstd;
    void *X; int ldx;
    void *Xt; int ldxt;
    const float *lo, *hi;
    unsigned *flags;
    int x_layout;
} rrtmg_sur_features_args;
rrtmg_status rrtmg_sur_features(const rrtmg_sur_features_args *args, void *stream);

/* Training targets from plain RRTMG outputs into rows row_offset..: LW and SW
 * heating [K/day] = rthraten * 86400 * pi3d per level, glw, lwupb, swdnb,
 * swupb, then the LW (up - down) and SW (down - up) net fluxes at the model
 * top implied by the heating profiles (2 nk + 6 values, zero-padded to ldt). */
typedef struct {
    int ncol, nk, ny;
    const float *rthratenlw, *rthratensw, *pi3d, *p8w, *glw, *lwupb, *swdnb, *swupb;
    int row_offset;
    float *T; int ldt;
} rrtmg_sur_targets_args;
rrtmg_status rrtmg_sur_targets(const rrtmg_sur_targets_args *args, void *stream);

/* Per-column statistics of F[n][ld] for columns 0..nf-1: mean, 1/std (0 for a
 * constant column), and optionally min and max. */
rrtmg_status rrtmg_sur_column_stats(const float *F, int n, int ld, int nf, float *mean, float *rstd, float *lo,
                                    float *hi, void *stream);

/* out[r][f] = (in[r][f] - mean[f]) * rstd[f] for f < nf, zero for nf <= f <
 * ldo; out is BF16 when out_bf16 != 0, else FP32. */
rrtmg_status rrtmg_sur_normalize(const float *in, int ldi, int n, int nf, const float *mean, const float *rstd,
                                 void *out, int ldo, int out_bf16, void *stream);

/* Batch gather: Xb[b] = X[idx[b]] (BF16 [B][ldx]), Xbt = Xb transposed
 * ([ldx][ldxbt]), Tb[b] = T[idx[b]] (FP32 [B][ldt], optional). */
rrtmg_status rrtmg_sur_gather(const void *X, int ldx, const float *T, int ldt, const int *idx, int B, void *Xb,
                              void *Xbt, int ldxbt, float *Tb, void *stream);

/* Weighted MSE gradient: dY = w[f] * 2 (Y - T) * scale as BF16 [B][ld] and
 * transposed [ld][lddyt]; adds sum w (Y - T)^2 to loss[0] (optional). */
rrtmg_status rrtmg_sur_loss_grad(const float *Y, const float *T, const float *w, int B, int ld, float scale,
                                 void *dY, void *dYt, int lddyt, float *loss, void *stream);

/* Bias gradient: db[r] = sum_b Gt[r][b] over a BF16 [rows][ld] matrix. */
rrtmg_status rrtmg_sur_row_sum(const void *Gt, int ld, int rows, int B, float *db, void *stream);

/* G[i] = sum_z P[z * n + i] (split-K partial sums). */
rrtmg_status rrtmg_sur_reduce_splits(const float *P, int splits, size_t n, float *G, void *stream);

/* One Adam step on an FP32 master w[rows][cols] with moments m, v:
 * w -= lr (mhat / (sqrt(vhat) + eps) + weight_decay w), mhat = m / bc1,
 * vhat = v / bc2; writes the BF16 copy wb [rows][ldwb] and its transpose
 * wbt [cols][ldwbt] when given. */
typedef struct {
    int rows, cols;
    float *w, *m, *v;
    const float *grad;
    float lr, beta1, beta2, eps, bc1, bc2, weight_decay;
    void *wb; int ldwb;
    void *wbt; int ldwbt;
} rrtmg_sur_adam_args;
rrtmg_status rrtmg_sur_adam(const rrtmg_sur_adam_args *args, void *stream);

/* Network outputs Y[ncol][ldy] (normalized) to WRF fields: rthratenlw/sw
 * (nx, nk, ny) = hr / 86400 / pi3d (a multiplication by 1/86400 and a fast
 * division), glw, lwupb, swdnb, swupb (nx, ny); SW is
 * exactly zero where coszr <= 0.  Energy gate: flags[c] |= 2 when the column-
 * integrated LW or SW heating differs from the predicted net surface minus
 * model-top flux by more than energy_tol W/m2. */
typedef struct {
    int ncol, nk, ny;
    const float *Y; int ldy;
    const float *out_mean, *out_std;
    const float *coszr, *pi3d, *p8w;
    float energy_tol;
    float *rthratenlw, *rthratensw, *glw, *lwupb, *swdnb, *swupb;
    unsigned *flags;
} rrtmg_sur_decode_args;
rrtmg_status rrtmg_sur_decode(const rrtmg_sur_decode_args *args, void *stream);

/* Bytes of the packed weight image read by rrtmg_sur_mlp. */
#define RRTMG_SUR_WEIGHT_IMAGE_BYTES 1703936

/* Packs the network's BF16 weights (W[0..2]: 512 x 512, W[3]: 128 x 512,
 * row-major [out][in], 16-byte aligned) into the image rrtmg_sur_mlp streams
 * through shared memory: 48 blocks of 32 KB (layer L < 3, rows 256 h ..
 * 256 h + 255, K = 64 b .. 64 b + 63 for block 16 L + 8 h + b) then 8 blocks
 * of 16 KB (layer 3, all 128 rows, K block b), each in the 128-byte swizzled
 * K-major layout of the feature tiles.  Repack after the weights change. */
rrtmg_status rrtmg_sur_pack_weights(const void *const W[4], void *image, void *stream);

/* Fused inference for 50-level columns: the four layers and the decode with
 * the energy gate of rrtmg_sur_decode in one kernel, giving the same bits as
 * rrtmg_gemm_bf16 (GELU, GELU, GELU, F32 epilogues) followed by
 * rrtmg_sur_decode.  X: the features of the ncol columns in x_layout 1
 * (ceil(ncol / 128) tiles, 16-byte aligned; rows past ncol are computed and
 * discarded); W: the packed weight image; bias[l]: FP32 biases (512, 512,
 * 512, 128).  flags: the range bits of rrtmg_sur_features on entry, | 2 for
 * the energy gate on exit.  Outputs as rrtmg_sur_decode.  One CTA per SM;
 * a CTA that gives up waiting for its copies or tensor-core work sets the
 * flag rrtmg_gemm_error reports. */
typedef struct {
    int ncol, nk, ny;
    const void *X;
    const void *W;
    const float *bias[4];
    const float *out_mean, *out_std;
    const float *coszr, *pi3d, *p8w;
    float energy_tol;
    float *rthratenlw, *rthratensw, *glw, *lwupb, *swdnb, *swupb;
    unsigned *flags;
} rrtmg_sur_mlp_args;
rrtmg_status rrtmg_sur_mlp(const rrtmg_sur_mlp_args *args, void *stream);

/* Writes the GPU global timer (ns) to *slot when the stream reaches this point
 * (stream-ordered, capturable in CUDA graphs; used for per-domain latencies). */
rrtmg_status rrtmg_sur_timestamp(unsigned long long *slot, void *stream);

/* Appends the columns with flags[c] != 0 to list; count must be zeroed first. */
rrtmg_status rrtmg_sur_compact(const unsigned *flags, int ncol, int *list, int *count, void *stream);

/* Gathers (to_compact = 1) or scatters (0) a field of nz levels between a
 * domain with south_north size ny and columns offset .. offset + count - 1 of
 * a compact (1, nz, stride) domain holding the listed columns; only the first
 * min(count, max_n) listed columns move (count is read on the device). */
rrtmg_status rrtmg_sur_move_columns(const int *list, const int *count, int max_n, int nz, int ny, const float *src,
                                    float *dst, int to_compact, int stride, int offset, void *stream);

/* Gathers (to_compact = 1) or scatters (0) up to RRTMG_SUR_MAX_FIELDS fields
 * in one launch, each as rrtmg_sur_move_columns does with src[i], dst[i] and
 * nz[i] levels; every compact field has level stride `stride` and column
 * offset `offset`.  Each pointer is device memory or page-locked host memory
 * mapped at the same address (read or written over the bus in place);
 * anything else is rejected with RRTMG_BAD_ARG. */
#define RRTMG_SUR_MAX_FIELDS 32
typedef struct {
    int nfields;
    const float *src[RRTMG_SUR_MAX_FIELDS];
    float *dst[RRTMG_SUR_MAX_FIELDS];
    int nz[RRTMG_SUR_MAX_FIELDS];
} rrtmg_sur_fields;
rrtmg_status rrtmg_sur_move_fields(const int *list, const int *count, int max_n, int ny, const rrtmg_sur_fields *f,
                                   int to_compact, int stride, int offset, void *stream);

/* GEMM tile width: 0 = automatic (256 columns when N allows, else 128), or
 * 128 / 256 (256 needs N % 256 == 0; narrower N falls back to 128).  Process-
 * wide; set by the ensemble autotuner. */
rrtmg_status rrtmg_gemm_set_tile(int bn);

/* Synchronous: reads the sticky flag that a CTA of rrtmg_gemm_bf16 or
 * rrtmg_sur_mlp sets when it gives up waiting for its copies or tensor-core
 * work (it then drains what it started, frees its tensor memory and writes no
 * output); clears it when reset != 0.  Returns RRTMG_TIMEOUT while the flag is
 * set, RRTMG_OK otherwise. */
rrtmg_status rrtmg_gemm_error(int reset, unsigned *flag);

/* Limit of each bounded mbarrier wait of rrtmg_gemm_bf16, in nanoseconds,
 * passed to the kernel with every call; 0 restores the default of 2 s.
 * Process-wide. */
rrtmg_status rrtmg_gemm_set_wait_ns(unsigned long long wait_ns);

/* Failure-detection test hook, off by default.  While enable != 0, every CTA
 * of later rrtmg_gemm_bf16 calls withholds the tensor-core commit of its first
 * K block: its wait for that block runs out after the wait limit, it waits for
 * the commit of its second block (which covers the first block's MMAs), frees
 * its tensor memory, writes no output and sets the flag rrtmg_gemm_error
 * reports.  While it is on, calls with K / (64 * ksplit) no larger than the
 * tile's pipeline stages (3 when N % 256 == 0 with the automatic tile, else
 * 4) are rejected with RRTMG_BAD_ARG.  Process-wide. */
rrtmg_status rrtmg_gemm_test_withhold_commit(int enable);

#ifdef __cplusplus
}
#endif
#endif /* RRTMG_SURROGATE_H */

// C-ABI of the surrogate kernels.  See include/rrtmg_surrogate.h.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "../../include/rrtmg_surrogate.h"
#include "surrogate_kernels.h"

using namespace rrtmg;

namespace {
bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

constexpr unsigned long long kDefaultWaitNs = 2000000000ull;  // 2 s
std::atomic<unsigned long long> g_wait_ns{kDefaultWaitNs};
std::atomic<int> g_withhold_commit{0};
}  // namespace

extern "C" rrtmg_status rrtmg_gemm_bf16(const rrtmg_gemm_args *a, void *stream) {
  if (!a || !a->A || !a->B) return RRTMG_BAD_ARG;
  if (a->M <= 0 || a->N <= 0 || a->K <= 0 || a->ksplit <= 0) return RRTMG_BAD_ARG;
  if (a->M % 128 || a->N % 128 || a->K % (64 * a->ksplit)) return RRTMG_BAD_ARG;
  if (a->lda % 8 || a->ldb % 8 || a->lda < a->K || a->ldb < a->K) return RRTMG_BAD_ARG;
  if (!aligned16(a->A) || !aligned16(a->B)) return RRTMG_BAD_ARG;
  // the epilogue stores 16-byte vectors along rows
  if ((a->C && (!aligned16(a->C) || a->ldc % 4 || a->split_stride % 4)) || (a->Z && (!aligned16(a->Z) || a->ldz % 4)) ||
      (a->aux && (!aligned16(a->aux) || a->ldaux % 4)) || (a->H && (!aligned16(a->H) || a->ldh % 8)))
    return RRTMG_BAD_ARG;
  switch (a->epilogue) {
    case RRTMG_EPI_F32:
      if (!a->C || a->ldc < a->N) return RRTMG_BAD_ARG;
      if (a->ksplit > 1 && a->split_stride < static_cast<size_t>(a->M) * a->ldc) return RRTMG_BAD_ARG;
      break;
    case RRTMG_EPI_GELU:
      if (a->ksplit != 1) return RRTMG_BAD_ARG;
      if ((a->Z && a->ldz < a->N) || (a->H && a->ldh < a->N) || (a->Ht && a->ldht < a->M)) return RRTMG_BAD_ARG;
      break;
    case RRTMG_EPI_DGELU:
      if (a->ksplit != 1 || !a->aux || a->ldaux < a->N) return RRTMG_BAD_ARG;
      if ((a->H && a->ldh < a->N) || (a->Ht && a->ldht < a->M)) return RRTMG_BAD_ARG;
      break;
    default:
      return RRTMG_BAD_ARG;
  }
  GemmArgs g{};
  g.A = static_cast<const __nv_bfloat16 *>(a->A);
  g.lda = a->lda;
  g.B = static_cast<const __nv_bfloat16 *>(a->B);
  g.ldb = a->ldb;
  g.M = a->M; g.N = a->N; g.K = a->K; g.ksplit = a->ksplit; g.epi = a->epilogue;
  g.bias = a->bias;
  g.C = a->C; g.ldc = a->ldc; g.split_stride = a->split_stride;
  g.H = static_cast<__nv_bfloat16 *>(a->H); g.ldh = a->ldh;
  g.Ht = static_cast<__nv_bfloat16 *>(a->Ht); g.ldht = a->ldht;
  g.aux = a->aux; g.ldaux = a->ldaux;
  g.Z = a->Z; g.ldz = a->ldz;
  g.wait_ns = g_wait_ns.load();
  g.withhold_commit0 = g_withhold_commit.load();
  // the hook needs a later commit to drain behind the withheld one and a wait
  // on the withheld one inside the K loop: more K blocks than stages
  if (g.withhold_commit0 && a->K / (64 * a->ksplit) <= gemm_stages(a->N)) return RRTMG_BAD_ARG;
  return launch_umma_gemm(g, static_cast<cudaStream_t>(stream)) == cudaSuccess ? RRTMG_OK : RRTMG_CUDA;
}

extern "C" rrtmg_status rrtmg_gemm_error(int reset, unsigned *flag) {
  if (!flag) return RRTMG_BAD_ARG;
  unsigned g = 0, m = 0;
  if (gemm_error_flag(&g, reset != 0) != cudaSuccess || mlp_error_flag(&m, reset != 0) != cudaSuccess)
    return RRTMG_CUDA;
  *flag = g | m;
  return *flag ? RRTMG_TIMEOUT : RRTMG_OK;
}

extern "C" rrtmg_status rrtmg_gemm_set_wait_ns(unsigned long long wait_ns) {
  g_wait_ns.store(wait_ns ? wait_ns : kDefaultWaitNs);
  return RRTMG_OK;
}

extern "C" rrtmg_status rrtmg_gemm_test_withhold_commit(int enable) {
  g_withhold_commit.store(enable != 0);
  return RRTMG_OK;
}

namespace {
rrtmg_status cuda_status(cudaError_t e) { return e == cudaSuccess ? RRTMG_OK : RRTMG_CUDA; }

// A pointer the kernels may dereference: device memory, managed memory, or
// page-locked host memory mapped at the same address (unified addressing).
bool device_reachable(const void *p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();  // clear the sticky error of an unknown pointer
    return false;
  }
  if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) return true;
  return at.type == cudaMemoryTypeHost && at.devicePointer == p;
}
cudaStream_t as_stream(void *s) { return static_cast<cudaStream_t>(s); }
}  // namespace

extern "C" rrtmg_status rrtmg_sur_features(const rrtmg_sur_features_args *a, void *stream) {
  if (!a || a->ncol < 0 || a->nk <= 0 || a->ny <= 0 || a->row_offset < 0) return RRTMG_BAD_ARG;
  if (!a->p3d || !a->p8w || !a->t3d || !a->qv || !a->qc || !a->qi || !a->qs || !a->cldfra || !a->o3 || !a->tsk ||
      !a->albedo || !a->coszr || !a->emiss)
    return RRTMG_BAD_ARG;
  const int nf = 9 * a->nk + 4;
  if (a->raw && a->ldf < nf) return RRTMG_BAD_ARG;
  if (a->X && (a->ldx < nf || !a->mean || !a->rstd)) return RRTMG_BAD_ARG;
  if (a->Xt && (!a->X || a->ldxt < a->row_offset + a->ncol)) return RRTMG_BAD_ARG;
  if (a->x_layout != 0 && (a->x_layout != 1 || !a->X || a->ldx != 512 || !aligned16(a->X) || a->raw || a->Xt ||
                           9 * a->nk + 4 > 512))
    return RRTMG_BAD_ARG;
  if ((a->lo == nullptr) != (a->hi == nullptr)) return RRTMG_BAD_ARG;
  if (a->ncol == 0) return RRTMG_OK;
  return cuda_status(launch_sur_features(*a, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_targets(const rrtmg_sur_targets_args *a, void *stream) {
  if (!a || a->ncol < 0 || a->nk <= 0 || a->ny <= 0 || a->row_offset < 0 || !a->T || a->ldt < 2 * a->nk + 6)
    return RRTMG_BAD_ARG;
  if (!a->rthratenlw || !a->rthratensw || !a->pi3d || !a->p8w || !a->glw || !a->lwupb || !a->swdnb || !a->swupb)
    return RRTMG_BAD_ARG;
  if (a->ncol == 0) return RRTMG_OK;
  return cuda_status(launch_sur_targets(*a, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_column_stats(const float *F, int n, int ld, int nf, float *mean, float *rstd,
                                               float *lo, float *hi, void *stream) {
  if (!F || n <= 0 || nf <= 0 || ld < nf || !mean || !rstd) return RRTMG_BAD_ARG;
  return cuda_status(launch_sur_column_stats(F, n, ld, nf, mean, rstd, lo, hi, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_gather(const void *X, int ldx, const float *T, int ldt, const int *idx, int B,
                                         void *Xb, void *Xbt, int ldxbt, float *Tb, void *stream) {
  if (!X || !idx || B <= 0 || ldx <= 0 || !Xb || !Xbt || ldxbt < B || (Tb && (!T || ldt <= 0))) return RRTMG_BAD_ARG;
  return cuda_status(launch_sur_gather(static_cast<const __nv_bfloat16 *>(X), ldx, T, ldt, idx, B,
                                       static_cast<__nv_bfloat16 *>(Xb), static_cast<__nv_bfloat16 *>(Xbt), ldxbt,
                                       Tb, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_loss_grad(const float *Y, const float *T, const float *w, int B, int ld,
                                            float scale, void *dY, void *dYt, int lddyt, float *loss, void *stream) {
  if (!Y || !T || !w || B <= 0 || ld <= 0 || !dY || !dYt || lddyt < B) return RRTMG_BAD_ARG;
  return cuda_status(launch_sur_loss_grad(Y, T, w, B, ld, scale, static_cast<__nv_bfloat16 *>(dY),
                                          static_cast<__nv_bfloat16 *>(dYt), lddyt, loss, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_row_sum(const void *Gt, int ld, int rows, int B, float *db, void *stream) {
  if (!Gt || !db || rows <= 0 || B <= 0 || ld < B) return RRTMG_BAD_ARG;
  return cuda_status(launch_sur_row_sum(static_cast<const __nv_bfloat16 *>(Gt), ld, rows, B, db, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_reduce_splits(const float *P, int splits, size_t n, float *G, void *stream) {
  if (!P || !G || splits <= 0 || n == 0) return RRTMG_BAD_ARG;
  return cuda_status(launch_sur_reduce_splits(P, splits, n, G, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_adam(const rrtmg_sur_adam_args *a, void *stream) {
  if (!a || a->rows <= 0 || a->cols <= 0 || !a->w || !a->m || !a->v || !a->grad) return RRTMG_BAD_ARG;
  if ((a->wb && a->ldwb < a->cols) || (a->wbt && a->ldwbt < a->rows)) return RRTMG_BAD_ARG;
  return cuda_status(launch_sur_adam(*a, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_decode(const rrtmg_sur_decode_args *a, void *stream) {
  if (!a || a->ncol < 0 || a->nk <= 0 || a->ny <= 0 || !a->Y || a->ldy < 2 * a->nk + 6 || 2 * a->nk + 6 > 128 ||
      !a->out_mean ||
      !a->out_std || !a->coszr || !a->pi3d || !a->p8w || !a->rthratenlw || !a->rthratensw || !a->glw || !a->lwupb ||
      !a->swdnb || !a->swupb || !a->flags)
    return RRTMG_BAD_ARG;
  if (a->ncol == 0) return RRTMG_OK;
  return cuda_status(launch_sur_decode(*a, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_compact(const unsigned *flags, int ncol, int *list, int *count, void *stream) {
  if (!flags || ncol < 0 || !list || !count) return RRTMG_BAD_ARG;
  if (ncol == 0) return RRTMG_OK;
  return cuda_status(launch_sur_compact(flags, ncol, list, count, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_move_columns(const int *list, const int *count, int max_n, int nz, int ny,
                                               const float *src, float *dst, int to_compact, int stride, int offset,
                                               void *stream) {
  if (!list || !count || max_n < 0 || nz <= 0 || ny <= 0 || !src || !dst || offset < 0 || stride < offset + max_n)
    return RRTMG_BAD_ARG;
  return cuda_status(launch_sur_move_columns(list, count, max_n, nz, ny, src, dst, to_compact, stride, offset,
                                             as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_gemm_set_tile(int bn) {
  if (bn != 0 && bn != 128 && bn != 256) return RRTMG_BAD_ARG;
  set_gemm_tile(bn);
  return RRTMG_OK;
}

extern "C" rrtmg_status rrtmg_sur_normalize(const float *in, int ldi, int n, int nf, const float *mean,
                                            const float *rstd, void *out, int ldo, int out_bf16, void *stream) {
  if (!in || !mean || !rstd || !out || n <= 0 || nf <= 0 || ldi < nf || ldo < nf) return RRTMG_BAD_ARG;
  return cuda_status(launch_sur_normalize(in, ldi, n, nf, mean, rstd, out, ldo, out_bf16, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_timestamp(unsigned long long *slot, void *stream) {
  if (!slot) return RRTMG_BAD_ARG;
  return cuda_status(launch_timestamp(slot, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_pack_weights(const void *const W[4], void *image, void *stream) {
  if (!W || !image || !aligned16(image)) return RRTMG_BAD_ARG;
  for (int l = 0; l < 4; ++l)
    if (!W[l] || !aligned16(W[l])) return RRTMG_BAD_ARG;
  return cuda_status(launch_sur_pack_weights(W, image, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_mlp(const rrtmg_sur_mlp_args *a, void *stream) {
  if (!a || a->ncol < 0 || a->nk != 50 || a->ny <= 0 || !a->X || !a->W || !aligned16(a->X) || !aligned16(a->W))
    return RRTMG_BAD_ARG;
  for (int l = 0; l < 4; ++l)
    if (!a->bias[l]) return RRTMG_BAD_ARG;
  if (!a->out_mean || !a->out_std || !a->coszr || !a->pi3d || !a->p8w || !a->rthratenlw || !a->rthratensw ||
      !a->glw || !a->lwupb || !a->swdnb || !a->swupb || !a->flags)
    return RRTMG_BAD_ARG;
  if (a->ncol == 0) return RRTMG_OK;
  return cuda_status(launch_sur_mlp(*a, as_stream(stream)));
}

extern "C" rrtmg_status rrtmg_sur_move_fields(const int *list, const int *count, int max_n, int ny,
                                              const rrtmg_sur_fields *f, int to_compact, int stride, int offset,
                                              void *stream) {
  if (!list || !count || !f || max_n < 0 || ny <= 0 || offset < 0 || stride < offset + max_n || f->nfields < 0 ||
      f->nfields > RRTMG_SUR_MAX_FIELDS)
    return RRTMG_BAD_ARG;
  for (int i = 0; i < f->nfields; ++i) {
    if (!f->src[i] || !f->dst[i] || f->nz[i] <= 0) return RRTMG_BAD_ARG;
    if (!device_reachable(f->src[i]) || !device_reachable(f->dst[i])) return RRTMG_BAD_ARG;
  }
  return cuda_status(launch_sur_move_fields(list, count, max_n, ny, *f, to_compact, stride, offset,
                                            as_stream(stream)));
}

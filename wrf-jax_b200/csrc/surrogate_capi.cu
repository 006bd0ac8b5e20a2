// C-ABI of the surrogate kernels.  See include/rrtmg_surrogate.h.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rrtmg_surrogate.h"
#include "surrogate_kernels.h"

using namespace rrtmg;

namespace {
bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
}  // namespace

extern "C" rrtmg_status rrtmg_gemm_bf16(const rrtmg_gemm_args *a, void *stream) {
  if (!a || !a->A || !a->B) return RRTMG_BAD_ARG;
  if (a->M <= 0 || a->N <= 0 || a->K <= 0 || a->ksplit <= 0) return RRTMG_BAD_ARG;
  if (a->M % 128 || a->N % 128 || a->K % (64 * a->ksplit)) return RRTMG_BAD_ARG;
  if (a->lda % 8 || a->ldb % 8 || a->lda < a->K || a->ldb < a->K) return RRTMG_BAD_ARG;
  if (!aligned16(a->A) || !aligned16(a->B)) return RRTMG_BAD_ARG;
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
  return launch_umma_gemm(g, static_cast<cudaStream_t>(stream)) == cudaSuccess ? RRTMG_OK : RRTMG_CUDA;
}

extern "C" rrtmg_status rrtmg_gemm_error(int reset, unsigned *flag) {
  if (!flag) return RRTMG_BAD_ARG;
  return gemm_error_flag(flag, reset != 0) == cudaSuccess ? RRTMG_OK : RRTMG_CUDA;
}

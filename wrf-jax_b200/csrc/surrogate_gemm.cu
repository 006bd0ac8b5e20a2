// BF16 GEMM on the 5th-generation tensor cores (tcgen05) with fused MLP
// epilogues, for the radiation surrogate's training and inference.
//
//   C[M x N] = A[M x K] * B[N x K]^T      (A, B row-major BF16, FP32 accumulate)
//
// One CTA of 128 threads owns a 128 x BN output tile (BN = 256 when N allows,
// else 128).  Its accumulator lives in tensor memory (128 lanes x BN FP32
// columns).  K advances in blocks of 64: all threads copy the A and B blocks
// into shared memory (cp.async, 3-4 stages in flight) in the 128-byte swizzled
// K-major layout, and one thread issues four tcgen05.mma (K = 16 each)
// whose completion is committed to the stage's mbarrier before the stage is
// refilled.  The epilogue reads the accumulator back with tcgen05.ld (warp w
// owns lanes 32w..32w+31, i.e. tile rows) and applies one of:
//   kEpiF32    C (+ bias) as FP32, one slab per K split (split-K partials)
//   kEpiGelu   Z = acc + bias (FP32), H = GELU(Z) as BF16 row-major and
//              transposed (the transposed copy feeds the weight gradient)
//   kEpiDgelu  dZ = acc * GELU'(aux) as BF16 row-major and transposed
//
// Shared-memory layout of an operand block (R rows x 64 K, BF16): the
// canonical K-major SWIZZLE_128B layout, row r at r * 128 bytes with its eight
// 16-byte chunks permuted by XOR with r mod 8, 8-row groups 1024 bytes apart;
// each block stage starts on a 1024-byte boundary.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "surrogate_kernels.h"
#include "umma_common.cuh"

namespace rrtmg {
namespace {

using umma::gelu;
using umma::gelu_grad;
using umma::mbar_wait;
using umma::smem_desc;
using umma::smem_u32;
using umma::swz;

constexpr int kBM = 128, kBK = 64;
constexpr int kThreads = 128;

template <int BN>
struct Tile {
  static constexpr int kStages = BN == 256 ? 3 : 4;
  static constexpr int kBytesA = kBM * kBK * 2;
  static constexpr int kBytesB = BN * kBK * 2;
  static constexpr int kStageBytes = kBytesA + kBytesB;
  // one extra KB so the stages can start on a 1024-byte boundary
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024;
  static constexpr uint32_t kIdesc = umma::idesc_bf16(kBM, BN);
};

__device__ unsigned g_gemm_error;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}

// Tile (m-tile = blockIdx.y, n-tile = blockIdx.x, K split = blockIdx.z): the
// n-tiles of one m-tile are neighbouring CTAs, so they share the A rows in L2.
// K blocks stream through kStages shared-memory stages: the copies of block
// kb + kStages - 1 are in flight while the tensor cores work on block kb.
template <int BN>
__global__ void __launch_bounds__(kThreads, 1) umma_gemm_kernel(GemmArgs g) {
  using TL = Tile<BN>;
  constexpr int S = TL::kStages;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t mbar[S];
  __shared__ uint32_t tmem_sh;
  __shared__ int fail_sh;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n0 = blockIdx.x * BN, m0 = blockIdx.y * kBM;
  const int kper = g.K / g.ksplit;
  const int kbeg = blockIdx.z * kper;
  const int nkb = kper / kBK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[s])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fail_sh = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_sh;

  uint8_t *tiles = smem + ((1024u - (smem_u32(smem) & 1023u)) & 1023u);
  auto stage_a = [&](int s) { return tiles + s * TL::kStageBytes; };
  auto stage_b = [&](int s) { return tiles + s * TL::kStageBytes + TL::kBytesA; };
  auto load = [&](int kb, int s) {
    const int k0 = kbeg + kb * kBK;
    uint8_t *a = stage_a(s), *b = stage_b(s);
    // 8 consecutive threads copy one 128-byte row: coalesced global reads and
    // conflict-free swizzled shared-memory writes
#pragma unroll
    for (int i = 0; i < (kBM * kBK / 8) / kThreads; ++i) {
      const int q = tid + i * kThreads;
      const int r = q >> 3, kc = q & 7;
      cp_async16(a + swz(r, kc), g.A + static_cast<size_t>(m0 + r) * g.lda + k0 + kc * 8);
    }
#pragma unroll
    for (int i = 0; i < (BN * kBK / 8) / kThreads; ++i) {
      const int q = tid + i * kThreads;
      const int r = q >> 3, kc = q & 7;
      cp_async16(b + swz(r, kc), g.B + static_cast<size_t>(n0 + r) * g.ldb + k0 + kc * 8);
    }
  };

  // prologue: blocks 0 .. S-2, one commit group each (empty groups keep the count)
#pragma unroll
  for (int s = 0; s < S - 1; ++s) {
    if (s < nkb) load(s, s);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  bool ok = true;
  int issued = 0;
  for (int kb = 0; kb < nkb; ++kb) {
    const int s = kb % S;
    asm volatile("cp.async.wait_group %0;" ::"n"(S - 2) : "memory");
    // make the generic-proxy shared-memory writes visible to the tensor cores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t abase = smem_u32(stage_a(s)), bbase = smem_u32(stage_b(s));
#pragma unroll
      for (int kk = 0; kk < kBK / 16; ++kk) {
        const uint64_t adesc = smem_desc(abase + kk * 32);
        const uint64_t bdesc = smem_desc(bbase + kk * 32);
        const uint32_t accumulate = (kb > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            :
            : "r"(tmem), "l"(adesc), "l"(bdesc), "r"(TL::kIdesc), "r"(accumulate)
            : "memory");
      }
      // (the failure-detection test withholds block 0's commit: the wait for it
      // below runs out, and block 1's commit, which covers every earlier MMA,
      // still lets the CTA drain before it frees its tensor memory)
      if (!(g.withhold_commit0 && kb == 0))
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&mbar[s]))
                     : "memory");
    }
    issued = kb + 1;
    const int next = kb + S - 1;
    if (next < nkb) {
      // stage next % S was last read by the MMAs of block kb - 1
      if (kb >= 1 && !mbar_wait(smem_u32(&mbar[(kb - 1) % S]), static_cast<uint32_t>((kb - 1) / S) & 1u, g.wait_ns))
        ok = false;
      if (__syncthreads_or(!ok)) {
        if (tid == 0) fail_sh = 1;
        break;
      }
      load(next, next % S);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  // wait for the last committed group (it covers every earlier MMA) before
  // the tensor memory is freed; this drain keeps the default limit even when
  // the pipeline waits above run with a shorter one
  if (issued > 0) {
    const int last = issued - 1;
    if (tid == 0 && !mbar_wait(smem_u32(&mbar[last % S]), static_cast<uint32_t>(last / S) & 1u)) fail_sh = 1;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const bool failed = fail_sh != 0 || issued != nkb;
  if (failed) {
    if (tid == 0) atomicOr(&g_gemm_error, 1u);
  } else {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      // each thread holds 16 consecutive columns of its row: row-major outputs
      // are written as 16-byte vectors, transposed ones as 2-byte elements
      // that are contiguous across the warp's 32 rows
      float acc[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) acc[j] = __uint_as_float(v[j]);
      const int nc = n0 + c;
      if (g.epi == kEpiF32) {
        if (g.bias && blockIdx.z == 0) {
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[j] += g.bias[nc + j];
        }
        float4 *dst = reinterpret_cast<float4 *>(g.C + static_cast<size_t>(blockIdx.z) * g.split_stride +
                                                 static_cast<size_t>(row) * g.ldc + nc);
#pragma unroll
        for (int q = 0; q < 4; ++q) dst[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
      } else {
        __align__(16) __nv_bfloat16 h[16];
        if (g.epi == kEpiGelu) {
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[j] += g.bias ? g.bias[nc + j] : 0.0f;
          if (g.Z) {
            float4 *dz = reinterpret_cast<float4 *>(g.Z + static_cast<size_t>(row) * g.ldz + nc);
#pragma unroll
            for (int q = 0; q < 4; ++q) dz[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
          }
#pragma unroll
          for (int j = 0; j < 16; ++j) h[j] = __float2bfloat16_rn(gelu(acc[j]));
        } else {  // kEpiDgelu
          const float4 *za = reinterpret_cast<const float4 *>(g.aux + static_cast<size_t>(row) * g.ldaux + nc);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const float4 z = za[q];
            h[4 * q + 0] = __float2bfloat16_rn(acc[4 * q + 0] * gelu_grad(z.x));
            h[4 * q + 1] = __float2bfloat16_rn(acc[4 * q + 1] * gelu_grad(z.y));
            h[4 * q + 2] = __float2bfloat16_rn(acc[4 * q + 2] * gelu_grad(z.z));
            h[4 * q + 3] = __float2bfloat16_rn(acc[4 * q + 3] * gelu_grad(z.w));
          }
        }
        if (g.H) {
          uint4 *dh = reinterpret_cast<uint4 *>(g.H + static_cast<size_t>(row) * g.ldh + nc);
          dh[0] = *reinterpret_cast<const uint4 *>(&h[0]);
          dh[1] = *reinterpret_cast<const uint4 *>(&h[8]);
        }
        if (g.Ht) {
#pragma unroll
          for (int j = 0; j < 16; ++j) g.Ht[static_cast<size_t>(nc + j) * g.ldht + row] = h[j];
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
  }
}

template <int BN>
cudaError_t launch_tile(const GemmArgs &g, cudaStream_t stream) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(umma_gemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         Tile<BN>::kSmemBytes);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  dim3 grid(g.N / BN, g.M / kBM, g.ksplit);
  umma_gemm_kernel<BN><<<grid, kThreads, Tile<BN>::kSmemBytes, stream>>>(g);
  return cudaGetLastError();
}

}  // namespace

namespace {
int g_tile_choice = 0;  // 0 automatic, else 128 or 256
}  // namespace

void set_gemm_tile(int bn) { g_tile_choice = bn; }

bool gemm_wide(int n) { return n % 256 == 0 && g_tile_choice != 128; }

int gemm_stages(int n) { return gemm_wide(n) ? Tile<256>::kStages : Tile<128>::kStages; }

cudaError_t launch_umma_gemm(const GemmArgs &g, cudaStream_t stream) {
  return gemm_wide(g.N) ? launch_tile<256>(g, stream) : launch_tile<128>(g, stream);
}

cudaError_t gemm_error_flag(unsigned *out, bool reset) {
  cudaError_t e = cudaMemcpyFromSymbol(out, g_gemm_error, sizeof(unsigned));
  if (e != cudaSuccess || !reset) return e;
  const unsigned zero = 0;
  return cudaMemcpyToSymbol(g_gemm_error, &zero, sizeof(unsigned));
}

}  // namespace rrtmg

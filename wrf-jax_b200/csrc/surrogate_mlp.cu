// Fused surrogate inference: the four layers of the radiation MLP
// (512 -> 512 -> 512 -> 512 -> 128, GELU between) and the decode with the
// energy gate in one persistent kernel, so hidden activations never leave
// the SM.
//
// One CTA per SM walks 128-row tiles (a row is one model column).  Per tile:
//   * the BF16 feature tile (128 x 512, 128 KB) arrives by one bulk copy into
//     the activation buffer, already in the 128-byte swizzled K-major layout
//     (rrtmg_sur_features with x_layout = 1 writes it that way);
//   * each layer's weights stream through three 32 KB shared-memory stages
//     (bulk copies of a pre-packed weight image, rrtmg_sur_pack_weights);
//     one thread issues tcgen05.mma (M = 128, N = 256 per half, K = 16) into
//     tensor memory: layers 0-2 fill columns 0-511, layer 3 columns 384-511;
//   * twelve epilogue warps read the accumulator back (tcgen05.ld, warp w
//     owns lanes 32 (w mod 4) .. and one of three column groups), add the bias,
//     apply GELU and write the BF16 result over the activation buffer as the
//     next layer's A operand, each chunk's accumulator read in flight while
//     the previous chunk is processed.  A hidden layer's two N halves are
//     pipelined against the MMAs: the first half's GELU runs while the
//     second half's MMAs still read the activation tile, so it is parked in
//     tensor memory (packed BF16 pairs) and copied into K blocks 0-3 once the
//     layer's MMAs are done; the next layer's MMAs over K blocks 0-3 then run
//     while the epilogue turns the second half into K blocks 4-7;
//   * after layer 3 two groups denormalize the outputs and write the WRF
//     fields directly (LW group: LW heating, glw, lwupb; SW group: SW
//     heating, swdnb, swupb), with the energy gate of rrtmg_sur_decode; their
//     level fields were prefetched into L2 when the tile started.
// The next tile's features load while the decode runs, and its layer-0 MMAs
// into columns 0-255 overlap the decode's reads of columns 384-511.
//
// Arithmetic is the unfused path's, operation for operation (same MMA
// shapes and K order, same epilogue and decode expressions), so both paths
// give the same bits.
//
// Warp roles (512 threads): warp 0 lane 0 issues the MMAs, warp 1 lane 0 the
// bulk copies, warps 4-15 run the epilogues (warps 2-3 idle: each epilogue
// warp must sit on the lane quarter its warp index selects); warp 0 also owns
// the tensor memory.  Every wait is an mbarrier wait bounded by the global timer; a role
// that gives up raises a shared abort flag the others poll, the copies and
// MMAs in flight are drained (again bounded), and the kernel sets a sticky
// error flag the host reads with rrtmg_gemm_error.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "surrogate_kernels.h"
#include "umma_common.cuh"

namespace rrtmg {
namespace {

using namespace umma;

constexpr int kRows = 128;                       // rows per tile
constexpr int kWidth = 512;                      // K of every layer, N of layers 0-2
constexpr int kOutCols = 128;                    // N of layer 3
constexpr int kKb = 64;                          // K per block (one 128-byte swizzle row)
constexpr int kNkb = kWidth / kKb;               // 8
constexpr uint32_t kActBlock = kRows * kKb * 2;  // 16 KB: one K block of the activation tile
constexpr uint32_t kActBytes = kActBlock * kNkb; // 128 KB
constexpr uint32_t kStageBytes = 256 * kKb * 2;  // 32 KB: 256 weight rows x 64 K
constexpr int kStages = 3;
constexpr int kSmemBytes = static_cast<int>(kActBytes + kStages * kStageBytes) + 1024;
constexpr int kThreads = 512;                    // 16 warps: 4 per scheduler, 128 registers each
constexpr int kEpiWarp0 = 4;                     // warps 4-15: epilogue
constexpr int kEpiWarps = 12;
constexpr int kDecodeWarps = 8;                  // epilogue groups 0 (LW) and 1 (SW) decode
constexpr int kDecBatch = 10;                    // levels per batch of decode loads
constexpr int kLoadsHidden = 3 * 2 * kNkb;       // 48 stage loads of 32 KB (layers 0-2, two halves)
constexpr int kLoadsPerTile = kLoadsHidden + kNkb;  // + 8 stage loads of 16 KB (layer 3)
constexpr uint32_t kOutCol0 = 384;               // tensor-memory column of layer 3's output 0
constexpr int kNk = 50;                          // levels of the network's columns

__device__ unsigned g_mlp_error;

// Weight stage load j (0..55) of a tile: offset into the packed image and size.
__device__ __forceinline__ uint32_t load_offset(int j) {
  return j < kLoadsHidden ? static_cast<uint32_t>(j) * kStageBytes
                          : static_cast<uint32_t>(kLoadsHidden) * kStageBytes +
                                static_cast<uint32_t>(j - kLoadsHidden) * (kStageBytes / 2);
}
__device__ __forceinline__ uint32_t load_bytes(int j) { return j < kLoadsHidden ? kStageBytes : kStageBytes / 2; }

struct Bars {
  uint64_t full[kStages], empty[kStages];
  uint64_t act_full;      // feature tile landed (tx)
  uint64_t act_free;      // layer-3 MMAs done reading the activation buffer (commit)
  uint64_t acc_full[2];   // a hidden layer's first / both halves' MMAs complete (commit)
  uint64_t acc3_full;     // layer 3's MMAs complete (commit)
  uint64_t act_ready[2];  // epilogue wrote K blocks 0-3 / 4-7 of the next A operand (12 warps)
  uint64_t tmem_free;  // decode read layer 3's accumulator (8 decode warps)
  uint64_t sw_done;    // SW half of the decode published its gate result (4 warps)
  uint64_t mma_done;   // drain at exit (commit)
};

// All lanes wait; the warp agrees on the outcome.
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity, const volatile int *abort) {
  const bool ok = mbar_wait_or_abort(bar, parity, abort);
  return __all_sync(0xffffffffu, ok);
}

__device__ __forceinline__ void fail(volatile int *abort) {
  *abort = 1;
  atomicOr(&g_mlp_error, 1u);
}

__device__ __forceinline__ float dec(uint32_t acc, const float *bias, const float *mean, const float *stdv, int f) {
  // the unfused path: Y = acc + bias (F32 epilogue), then Y * out_std + out_mean
  const float y = __uint_as_float(acc) + bias[f];
  return y * stdv[f] + mean[f];
}

// Decode of one column by one side: HALF 0 writes the LW heating, glw and
// lwupb, HALF 1 the SW heating (zero at night), swdnb and swupb; returns
// whether that side fails the energy gate.  y: the side's 50 denormalized
// heating rates; y2a, y2b: its two surface fluxes; ytop: its model-top net
// flux.  Expressions follow rrtmg_sur_decode operation for operation
// (sur_tendency, sur_flux_term); the level fields are read in batches so
// their loads overlap.
template <int HALF>
__device__ __forceinline__ bool decode_side(const SurMlpArgs &a, int col, const float (&y)[kNk], float y2a,
                                            float y2b, float ytop) {
  const int ny = a.ny;
  const int i = col / ny, jj = col - i * ny;
  const size_t q0 = static_cast<size_t>(i) * kNk * ny + jj;
  const size_t l0 = static_cast<size_t>(i) * (kNk + 1) * ny + jj;
  const bool day = __ldg(a.coszr + col) > 0.0f;
  float *__restrict__ out = HALF == 0 ? a.rthratenlw : a.rthratensw;
  float s = 0.0f;
#pragma unroll
  for (int k0 = 0; k0 < kNk; k0 += kDecBatch) {
    float pi[kDecBatch], pw[kDecBatch + 1];
#pragma unroll
    for (int b = 0; b < kDecBatch; ++b) pi[b] = __ldg(a.pi3d + q0 + static_cast<size_t>(k0 + b) * ny);
#pragma unroll
    for (int b = 0; b <= kDecBatch; ++b) pw[b] = __ldg(a.p8w + l0 + static_cast<size_t>(k0 + b) * ny);
#pragma unroll
    for (int b = 0; b < kDecBatch; ++b) {
      float hr = y[k0 + b];
      if (HALF == 1 && !day) hr = 0.0f;
      out[q0 + static_cast<size_t>(k0 + b) * ny] = sur_tendency(hr, pi[b]);
      const float dp = (pw[b] - pw[b + 1]) * 0.01f;
      s += sur_flux_term(hr, dp);
    }
  }
  if (HALF == 0) {
    a.glw[col] = y2a;
    a.lwupb[col] = y2b;
    const float lw_res = fabsf(((y2b - y2a) - ytop) - s);
    return !(lw_res <= a.energy_tol);
  } else {
    const float swdnb = day ? y2a : 0.0f, swupb = day ? y2b : 0.0f;
    a.swdnb[col] = swdnb;
    a.swupb[col] = swupb;
    const float sw_res = day ? fabsf((ytop - (swdnb - swupb)) - s) : 0.0f;
    return !(sw_res <= a.energy_tol);
  }
}

// Layer 3's outputs for one side of one row, read from tensor memory and
// denormalized, then the decode; arrives on tmem_free once the accumulator
// has been read.  Output columns: LW heating f = 0..49, SW heating 50..99,
// glw 100, lwupb 101, swdnb 102, swupb 103, LW and SW model-top net 104, 105.
template <int HALF>
__device__ __forceinline__ bool decode_row(const SurMlpArgs &a, uint32_t cb, int col, bool live, int lane,
                                           uint32_t tmem_free_bar) {
  constexpr int f0 = HALF == 0 ? 0 : 48;
  const float *b3 = a.bias[3], *om = a.out_mean, *os = a.out_std;
  // one 16-column read at a time keeps the register footprint small
  uint32_t v[16];
  tmem_ld16(cb + 96, v);  // f = 96 .. 111: f = 100 + d sits at v[4 + d]
  tmem_ld_wait();
  const float y2a = dec(v[HALF == 0 ? 4 : 6], b3, om, os, 2 * kNk + (HALF == 0 ? 0 : 2));
  const float y2b = dec(v[HALF == 0 ? 5 : 7], b3, om, os, 2 * kNk + (HALF == 0 ? 1 : 3));
  const float ytop = dec(v[HALF == 0 ? 8 : 9], b3, om, os, 2 * kNk + (HALF == 0 ? 4 : 5));
  float y[kNk];
#pragma unroll
  for (int ch = 0; ch < 4; ++ch) {
    tmem_ld16(cb + f0 + ch * 16, v);
    tmem_ld_wait();
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const int f = f0 + ch * 16 + e;
      const int k = HALF == 0 ? f : f - kNk;
      if (k >= 0 && k < kNk) y[k] = dec(v[e], b3, om, os, f);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncwarp();
  if (lane == 0) mbar_arrive(tmem_free_bar);
  if (!live) return false;
  return decode_side<HALF>(a, col, y, y2a, y2b, ytop);
}

// 16 accumulator columns of this thread's row (K = c .. c + 15 of the next
// layer): + bias, GELU, BF16 pairs.
__device__ __forceinline__ void gelu_pack(const uint32_t (&v)[16], const float *bias, int c, uint32_t (&p)[8]) {
  const float4 *b4 = reinterpret_cast<const float4 *>(bias + c);
  float b[16];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float4 t = __ldg(b4 + q);
    b[4 * q] = t.x; b[4 * q + 1] = t.y; b[4 * q + 2] = t.z; b[4 * q + 3] = t.w;
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float x0 = __uint_as_float(v[2 * j]) + b[2 * j];
    const float x1 = __uint_as_float(v[2 * j + 1]) + b[2 * j + 1];
    const __nv_bfloat162 h2 = __floats2bfloat162_rn(gelu(x0), gelu(x1));
    p[j] = *reinterpret_cast<const uint32_t *>(&h2);
  }
}

// Eight BF16 pairs as K = c .. c + 15 of row r of the activation tile (two
// 16-byte chunks in the swizzled layout).
__device__ __forceinline__ void act_store(const uint32_t (&p)[8], int c, uint8_t *act, int r) {
  uint8_t *blk = act + (c / kKb) * kActBlock;
  const int kc = (c % kKb) / 8;
  *reinterpret_cast<uint4 *>(blk + swz(r, kc)) = make_uint4(p[0], p[1], p[2], p[3]);
  *reinterpret_cast<uint4 *>(blk + swz(r, kc + 1)) = make_uint4(p[4], p[5], p[6], p[7]);
}

__global__ void __launch_bounds__(kThreads, 1) mlp_kernel(SurMlpArgs a, int ntiles) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) Bars bars;
  __shared__ uint32_t tmem_sh;
  __shared__ volatile int abort_sh;
  __shared__ int sw_fail[kRows];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint8_t *base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t *act = base;
  uint8_t *stage0 = base + kActBytes;
  const uint32_t act_s = smem_u32(act), stage_s = smem_u32(stage0);
  auto bar = [](uint64_t &b) { return smem_u32(&b); };

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 32) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(bar(bars.full[s]), 1);
      mbar_init(bar(bars.empty[s]), 1);
    }
    mbar_init(bar(bars.act_full), 1);
    mbar_init(bar(bars.act_free), 1);
    for (int h = 0; h < 2; ++h) {
      mbar_init(bar(bars.acc_full[h]), 1);
      mbar_init(bar(bars.act_ready[h]), kEpiWarps);
    }
    mbar_init(bar(bars.acc3_full), 1);
    mbar_init(bar(bars.tmem_free), kDecodeWarps);
    mbar_init(bar(bars.sw_done), kDecodeWarps / 2);
    mbar_init(bar(bars.mma_done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_sh = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_sh;
  const uint8_t *X = static_cast<const uint8_t *>(a.X);
  const uint8_t *W = static_cast<const uint8_t *>(a.W);

  if (warp == 1) {
    // ---------------- producer: bulk copies ----------------
    if (lane == 0) {
      uint32_t li = 0;
      int it = 0, last_tile_it = -1;
      for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        if (it > 0 && !mbar_wait_or_abort(bar(bars.act_free), (it - 1) & 1, &abort_sh)) {
          fail(&abort_sh);
          break;
        }
        mbar_expect_tx(bar(bars.act_full), kActBytes);
        bulk_g2s(act_s, X + static_cast<size_t>(tile) * kActBytes, kActBytes, bar(bars.act_full));
        last_tile_it = it;
        bool ok = true;
        for (int j = 0; j < kLoadsPerTile; ++j, ++li) {
          const int s = static_cast<int>(li % kStages);
          if (li >= kStages && !mbar_wait_or_abort(bar(bars.empty[s]), ((li / kStages) - 1) & 1, &abort_sh)) {
            ok = false;
            break;
          }
          mbar_expect_tx(bar(bars.full[s]), load_bytes(j));
          bulk_g2s(stage_s + s * kStageBytes, W + load_offset(j), load_bytes(j), bar(bars.full[s]));
        }
        if (!ok) {
          fail(&abort_sh);
          break;
        }
      }
      // drain: every copy this thread issued has landed before the CTA exits
      if (last_tile_it >= 0) mbar_wait(bar(bars.act_full), last_tile_it & 1);
      for (uint32_t q = li > kStages ? li - kStages : 0; q < li; ++q)
        mbar_wait(bar(bars.full[q % kStages]), (q / kStages) & 1);
    }
  } else if (warp == 0) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t kIdescHidden = idesc_bf16(kRows, 256);
      constexpr uint32_t kIdescOut = idesc_bf16(kRows, kOutCols);
      uint32_t li = 0, ready[2] = {0, 0};
      int it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++it) {
        if (!mbar_wait_or_abort(bar(bars.act_full), it & 1, &abort_sh)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        for (int layer = 0; layer < 4 && ok; ++layer) {
          // the epilogue's K blocks 0-3 (act_ready[0]) and 4-7 (act_ready[1])
          // of this layer's A operand; layer 3 also writes columns the
          // epilogue's second half reads, so it waits for both first
          auto wait_ready = [&](int h) {
            if (!mbar_wait_or_abort(bar(bars.act_ready[h]), ready[h] & 1, &abort_sh)) return false;
            ++ready[h];
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            return true;
          };
          if (layer == 3 && !(wait_ready(0) && wait_ready(1))) {
            ok = false;
            break;
          }
          const int halves = layer < 3 ? 2 : 1;
          for (int h = 0; h < halves && ok; ++h) {
            if (layer == 0 && h == 1 && it > 0) {
              if (!mbar_wait_or_abort(bar(bars.tmem_free), (it - 1) & 1, &abort_sh)) {
                ok = false;
                break;
              }
              asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            }
            const uint32_t d = tmem + (layer < 3 ? static_cast<uint32_t>(h) * 256u : kOutCol0);
            const uint32_t idesc = layer < 3 ? kIdescHidden : kIdescOut;
            for (int kb = 0; kb < kNkb; ++kb, ++li) {
              if (layer > 0 && layer < 3 && h == 0 && (kb == 0 || kb == kNkb / 2) && !wait_ready(kb == 0 ? 0 : 1)) {
                ok = false;
                break;
              }
              const int s = static_cast<int>(li % kStages);
              if (!mbar_wait_or_abort(bar(bars.full[s]), (li / kStages) & 1, &abort_sh)) {
                ok = false;
                break;
              }
              asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
              const uint32_t ab = act_s + kb * kActBlock, bb = stage_s + s * kStageBytes;
#pragma unroll
              for (int kk = 0; kk < kKb / 16; ++kk)
                umma_bf16(d, smem_desc(ab + kk * 32), smem_desc(bb + kk * 32), idesc, (kb | kk) != 0 ? 1u : 0u);
              umma_commit(bar(bars.empty[s]));
            }
            if (!ok) break;
            umma_commit(bar(layer < 3 ? bars.acc_full[h] : bars.acc3_full));
          }
          if (!ok) break;
          if (layer == 3) umma_commit(bar(bars.act_free));
        }
      }
      if (!ok) fail(&abort_sh);
      // drain: every MMA this thread issued has completed before the CTA exits
      umma_commit(bar(bars.mma_done));
      mbar_wait(bar(bars.mma_done), 0);
    }
  } else if (warp >= kEpiWarp0) {
    // ---------------- epilogue / decode ----------------
    const int quarter = warp & 3;                  // tensor-memory lanes 32 * quarter ..
    const int group = (warp - kEpiWarp0) >> 2;     // column group 0-2; decode side 0 / 1
    const int r = quarter * 32 + lane;             // tile row of this thread
    const uint32_t trow = tmem + (static_cast<uint32_t>(quarter * 32) << 16);
    uint32_t acc_uses[2] = {0, 0};
    int it = 0;
    bool ok = true;
    // 16-column chunks of each 256-column half: group 0 takes 0-5, group 1
    // 6-10, group 2 11-15
    const int ch0 = group == 0 ? 0 : (group == 1 ? 6 : 11);
    const int ch1 = group == 0 ? 6 : (group == 1 ? 11 : 16);
    auto wait_acc = [&](int h) {
      if (!warp_wait(bar(bars.acc_full[h]), acc_uses[h] & 1, &abort_sh)) return false;
      ++acc_uses[h];
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      return true;
    };
    // generic-proxy writes -> visible to the tensor cores; tensor-memory
    // accesses done; then one arrival per warp
    auto publish = [&](int h) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(bars.act_ready[h]));
    };
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++it) {
      const int col = tile * kRows + r;
      const bool live = col < a.ncol;
      if (group < 2 && live) {
        // the decode's level fields: into L2 now, read after layer 3
        const int i = col / a.ny, jj = col - i * a.ny;
        const float *pp = (group == 0 ? a.p8w : a.pi3d);
        const size_t base = group == 0 ? static_cast<size_t>(i) * (kNk + 1) * a.ny + jj
                                       : static_cast<size_t>(i) * kNk * a.ny + jj;
        const int levels = group == 0 ? kNk + 1 : kNk;
        for (int k = 0; k < levels; ++k)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(pp + base + static_cast<size_t>(k) * a.ny));
      }
      // Per hidden layer: the first half's accumulator (columns 0-255) is
      // ready while the second half's MMAs still read the activation tile,
      // so its GELU result is parked in tensor memory, packed BF16 pairs in
      // the group's own columns (chunk k at 16 ch0 + 8 (k - ch0), behind the
      // columns still to be read); once the layer's MMAs are done it is
      // copied into K blocks 0-3 of the tile (the next layer's first MMAs
      // start on them) while the second half is processed into K blocks 4-7.
      for (int layer = 0; layer < 3 && ok; ++layer) {
        const float *bias = a.bias[layer];
        if (!wait_acc(0)) {
          ok = false;
          break;
        }
        {
          uint32_t va[16], vb[16], p[8];
          tmem_ld16(trow + ch0 * 16, va);
#pragma unroll 1
          for (int ch = ch0; ch < ch1; ch += 2) {
            tmem_ld_wait();
            if (ch + 1 < ch1) tmem_ld16(trow + (ch + 1) * 16, vb);
            gelu_pack(va, bias, ch * 16, p);
            tmem_st8(trow + 16 * ch0 + 8 * (ch - ch0), p);
            if (ch + 1 < ch1) {
              tmem_ld_wait();
              if (ch + 2 < ch1) tmem_ld16(trow + (ch + 2) * 16, va);
              gelu_pack(vb, bias, (ch + 1) * 16, p);
              tmem_st8(trow + 16 * ch0 + 8 * (ch + 1 - ch0), p);
            }
          }
          tmem_st_wait();
        }
        if (!wait_acc(1)) {
          ok = false;
          break;
        }
        {
          uint32_t p[8];
#pragma unroll 1
          for (int ch = ch0; ch < ch1; ++ch) {
            tmem_ld8(trow + 16 * ch0 + 8 * (ch - ch0), p);
            tmem_ld_wait();
            act_store(p, ch * 16, act, r);
          }
        }
        publish(0);
        {
          const uint32_t th = trow + 256u;
          uint32_t va[16], vb[16], p[8];
          tmem_ld16(th + ch0 * 16, va);
#pragma unroll 1
          for (int ch = ch0; ch < ch1; ch += 2) {
            tmem_ld_wait();
            if (ch + 1 < ch1) tmem_ld16(th + (ch + 1) * 16, vb);
            gelu_pack(va, bias, 256 + ch * 16, p);
            act_store(p, 256 + ch * 16, act, r);
            if (ch + 1 < ch1) {
              tmem_ld_wait();
              if (ch + 2 < ch1) tmem_ld16(th + (ch + 2) * 16, va);
              gelu_pack(vb, bias, 256 + (ch + 1) * 16, p);
              act_store(p, 256 + (ch + 1) * 16, act, r);
            }
          }
        }
        publish(1);
      }
      if (!ok) break;
      // ---- layer 3: decode (groups 0 and 1) ----
      if (group >= 2) continue;
      if (!warp_wait(bar(bars.acc3_full), it & 1, &abort_sh)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t cb = trow + kOutCol0;
      if (group == 1) {
        const bool gate_fail = decode_row<1>(a, cb, col, live, lane, bar(bars.tmem_free));
        sw_fail[r] = gate_fail ? 1 : 0;
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(bars.sw_done));
      } else {
        const bool gate_fail = decode_row<0>(a, cb, col, live, lane, bar(bars.tmem_free));
        if (!warp_wait(bar(bars.sw_done), it & 1, &abort_sh)) {
          ok = false;
          break;
        }
        if (live) {
          unsigned f = a.flags[col];
          if (gate_fail || sw_fail[r]) f |= 2u;
          a.flags[col] = f;
        }
      }
    }
    if (!ok) fail(&abort_sh);
  }

  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
  }
}

// Packed weight image: stage load j of a tile (the order the kernel consumes
// them) holds, in the 128-byte swizzled K-major layout, rows h*256 .. +255 of
// layer L (j = 16 L + 8 h + kb, L < 3) or all 128 rows of layer 3
// (j = 48 + kb), K = 64 kb .. 64 kb + 63.  One thread per 16-byte chunk.
__global__ void pack_weights_kernel(const __nv_bfloat16 *W0, const __nv_bfloat16 *W1, const __nv_bfloat16 *W2,
                                    const __nv_bfloat16 *W3, uint8_t *img) {
  const uint32_t chunk = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t byte = chunk * 16u;
  const uint32_t hidden_bytes = kLoadsHidden * kStageBytes;
  if (byte >= hidden_bytes + kNkb * (kStageBytes / 2)) return;
  int layer, kb, row;
  uint32_t within;
  if (byte < hidden_bytes) {
    const uint32_t j = byte / kStageBytes;
    within = byte % kStageBytes;
    layer = static_cast<int>(j / 16);
    const int h = static_cast<int>((j % 16) / 8);
    kb = static_cast<int>(j % 8);
    row = h * 256 + static_cast<int>(within / 128);
  } else {
    const uint32_t rem = byte - hidden_bytes;
    layer = 3;
    kb = static_cast<int>(rem / (kStageBytes / 2));
    within = rem % (kStageBytes / 2);
    row = static_cast<int>(within / 128);
  }
  const int r = static_cast<int>(within / 128) & 255;
  const int pos = static_cast<int>((within % 128) / 16);
  const int kc = pos ^ (r & 7);
  const __nv_bfloat16 *Wl = layer == 0 ? W0 : layer == 1 ? W1 : layer == 2 ? W2 : W3;
  const uint4 v = *reinterpret_cast<const uint4 *>(Wl + static_cast<size_t>(row) * kWidth + kb * kKb + kc * 8);
  *reinterpret_cast<uint4 *>(img + byte) = v;
}

constexpr int kMaxDevices = 64;
int g_sm_count[kMaxDevices];  // 0 until the device is configured

}  // namespace

size_t sur_weight_image_bytes() { return static_cast<size_t>(kLoadsHidden) * kStageBytes + kNkb * (kStageBytes / 2); }

cudaError_t launch_sur_pack_weights(const void *const W[4], void *image, cudaStream_t s) {
  const size_t chunks = sur_weight_image_bytes() / 16;
  pack_weights_kernel<<<static_cast<unsigned>((chunks + 255) / 256), 256, 0, s>>>(
      static_cast<const __nv_bfloat16 *>(W[0]), static_cast<const __nv_bfloat16 *>(W[1]),
      static_cast<const __nv_bfloat16 *>(W[2]), static_cast<const __nv_bfloat16 *>(W[3]),
      static_cast<uint8_t *>(image));
  return cudaGetLastError();
}

cudaError_t launch_sur_mlp(const SurMlpArgs &a, cudaStream_t s) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (g_sm_count[dev] == 0) {
    e = cudaFuncSetAttribute(mlp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e != cudaSuccess) return e;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    g_sm_count[dev] = sms;
  }
  const int ntiles = (a.ncol + kRows - 1) / kRows;
  const int grid = ntiles < g_sm_count[dev] ? ntiles : g_sm_count[dev];
  mlp_kernel<<<grid, kThreads, kSmemBytes, s>>>(a, ntiles);
  return cudaGetLastError();
}

cudaError_t mlp_error_flag(unsigned *out, bool reset) {
  cudaError_t e = cudaMemcpyFromSymbol(out, g_mlp_error, sizeof(unsigned));
  if (e != cudaSuccess || !reset) return e;
  const unsigned zero = 0;
  return cudaMemcpyToSymbol(g_mlp_error, &zero, sizeof(unsigned));
}

}  // namespace rrtmg

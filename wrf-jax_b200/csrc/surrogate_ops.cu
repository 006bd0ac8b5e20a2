// Radiation surrogate: feature/target construction, training kernels (batch
// gather, loss gradient, bias gradients, split-K reduction, Adam), inference
// decode with the per-column gate, and the fallback gather/scatter that hands
// rejected columns to the plain RRTMG kernels.
//
// Column c = i * ny + j of a WRF-layout domain; 3-D fields (nx, nk, ny) at
// (i * nk + k) * ny + j, level fields (nx, nk + 1, ny), 2-D fields (nx, ny).
//
// Feature vector of a column (kSurFeatures = 9 * nk + 4, padded with zeros to
// the row length): per level k, at f * nk + k,
//   f = 0 t3d [K], 1 ln p3d [Pa], 2 qv, 3 qc, 4 qi, 5 qs [kg/kg], 6 cldfra,
//       7 o3, 8 layer thickness p8w[k] - p8w[k+1] [Pa];
// then tsk, albedo, coszr, emiss.  Target vector (kSurTargets = 2 * nk + 6):
// LW heating [K/day] per level, SW heating per level, glw (LW down at the
// surface), lwupb, swdnb, swupb [W/m2], then the LW and SW net fluxes at the
// model top implied by the heating profile (the energy-gate quantities).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "surrogate_kernels.h"

namespace rrtmg {
namespace {

// heatfac = g * 86400 / (cp * 100): K/day per (W/m2 per hPa)  (lw:5706, sw:2289)
constexpr float kHeatfac = (9.8066f * 8.6400e4f) / (1004.5f * 1.0e2f);

__device__ __forceinline__ size_t idx3(int c, int k, int nk, int ny) {
  const int i = c / ny, j = c - i * ny;
  return (static_cast<size_t>(i) * nk + k) * ny + j;
}

// Value of feature f (f < 9 nk + 4) of column c.
__device__ __forceinline__ float feature_value(const SurFeatureArgs &a, int c, int f) {
  const int nk = a.nk, ny = a.ny;
  if (f >= 9 * nk) {
    switch (f - 9 * nk) {
      case 0: return a.tsk[c];
      case 1: return a.albedo[c];
      case 2: return a.coszr[c];
      default: return a.emiss[c];
    }
  }
  const int field = f / nk, k = f - field * nk;
  const size_t q = idx3(c, k, nk, ny);
  switch (field) {
    case 0: return a.t3d[q];
    case 1: return logf(a.p3d[q]);
    case 2: return a.qv[q];
    case 3: return a.qc[q];
    case 4: return a.qi[q];
    case 5: return a.qs[q];
    case 6: return a.cldfra[q];
    case 7: return a.o3[q];
    default: return a.p8w[idx3(c, k, nk + 1, ny)] - a.p8w[idx3(c, k + 1, nk + 1, ny)];
  }
}

// A block owns kFeatCols consecutive columns and walks the features in chunks
// of kFeatChunk: each thread evaluates one (column, feature) at a time with
// the columns fastest (coalesced field reads), the chunk is staged in shared
// memory, and the rows of the row-major outputs are written contiguously.
constexpr int kFeatCols = 64, kFeatChunk = 64;

__global__ void __launch_bounds__(256) features_kernel(SurFeatureArgs a) {
  __shared__ float tile[kFeatChunk][kFeatCols + 1];
  __shared__ int oob[kFeatCols];
  const int c0 = blockIdx.x * kFeatCols;
  const int nf = 9 * a.nk + 4;
  const int width = a.X ? a.ldx : nf;
  __nv_bfloat16 *X = static_cast<__nv_bfloat16 *>(a.X), *Xt = static_cast<__nv_bfloat16 *>(a.Xt);
  for (int i = threadIdx.x; i < kFeatCols; i += blockDim.x) oob[i] = 0;
  __syncthreads();
  for (int f0 = 0; f0 < width; f0 += kFeatChunk) {
    // evaluate: thread -> (feature, column) with the column fastest
    for (int e = threadIdx.x; e < kFeatChunk * kFeatCols; e += blockDim.x) {
      const int lf = e / kFeatCols, lc = e - lf * kFeatCols;
      const int f = f0 + lf, c = c0 + lc;
      float v = 0.0f;
      if (c < a.ncol && f < nf) {
        v = feature_value(a, c, f);
        if (a.lo && (v < a.lo[f] || v > a.hi[f])) oob[lc] = 1;
      }
      tile[lf][lc] = v;
    }
    __syncthreads();
    // store: thread -> (column, feature) with the feature fastest (row-major rows)
    for (int e = threadIdx.x; e < kFeatChunk * kFeatCols; e += blockDim.x) {
      const int lc = e / kFeatChunk, lf = e - lc * kFeatChunk;
      const int f = f0 + lf, c = c0 + lc;
      if (c >= a.ncol || f >= width) continue;
      const size_t row = static_cast<size_t>(a.row_offset + c);
      const float v = tile[lf][lc];
      if (a.raw && f < nf) a.raw[row * a.ldf + f] = v;
      if (X) X[row * a.ldx + f] = __float2bfloat16_rn(f < nf ? (v - a.mean[f]) * a.rstd[f] : 0.0f);
    }
    if (Xt) {
      // transposed copy: thread -> (feature, column) with the column fastest
      for (int e = threadIdx.x; e < kFeatChunk * kFeatCols; e += blockDim.x) {
        const int lf = e / kFeatCols, lc = e - lf * kFeatCols;
        const int f = f0 + lf, c = c0 + lc;
        if (c >= a.ncol || f >= a.ldx) continue;
        const float v = tile[lf][lc];
        Xt[static_cast<size_t>(f) * a.ldxt + a.row_offset + c] =
            __float2bfloat16_rn(f < nf ? (v - a.mean[f]) * a.rstd[f] : 0.0f);
      }
    }
    __syncthreads();
  }
  if (a.flags) {
    for (int lc = threadIdx.x; lc < kFeatCols; lc += blockDim.x) {
      const int c = c0 + lc;
      if (c < a.ncol) a.flags[c] = oob[lc] ? 1u : 0u;
    }
  }
}

// Inference features, one thread per column: the thread walks its column's
// features 16 at a time (field reads coalesced across the warp's consecutive
// columns), normalizes them, and writes 32 contiguous bytes of its output row:
// row-major X, or (kTiled) the swizzled 128-row tiles of the fused inference
// kernel, where chunks 2p and 2p + 1 of a row stay one 32-byte pair.  Values,
// rounding and range flags are those of features_kernel.
constexpr int kRowThreads = 128, kMaxFeatures = 512;

template <bool kTiled>
__global__ void __launch_bounds__(kRowThreads) features_rows_kernel(SurFeatureArgs a) {
  __shared__ float4 st[kMaxFeatures];  // mean, rstd, lo, hi
  __shared__ const float *src[13];
  const int nk = a.nk, ny = a.ny, nf = 9 * nk + 4;
  for (int f = threadIdx.x; f < nf; f += blockDim.x)
    st[f] = make_float4(a.mean[f], a.rstd[f], a.lo ? a.lo[f] : -__int_as_float(0x7f800000),
                        a.hi ? a.hi[f] : __int_as_float(0x7f800000));
  if (threadIdx.x == 0) {
    src[0] = a.t3d; src[1] = a.p3d; src[2] = a.qv; src[3] = a.qc; src[4] = a.qi; src[5] = a.qs;
    src[6] = a.cldfra; src[7] = a.o3; src[8] = a.p8w;
    src[9] = a.tsk; src[10] = a.albedo; src[11] = a.coszr; src[12] = a.emiss;
  }
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncol) return;
  const int i = c / ny, j = c - i * ny;
  const size_t b3 = static_cast<size_t>(i) * nk * ny + j, bl = static_cast<size_t>(i) * (nk + 1) * ny + j;
  const size_t row = static_cast<size_t>(a.row_offset) + c;
  uint8_t *xrow;
  if (kTiled) {
    xrow = static_cast<uint8_t *>(a.X) + (row >> 7) * 131072u;
  } else {
    xrow = static_cast<uint8_t *>(a.X) + row * a.ldx * 2;
  }
  const int rr = static_cast<int>(row & 127);
  unsigned oob = 0;
  int fld = 0, k = 0;  // field and level of the next feature
  for (int f0 = 0; f0 < a.ldx; f0 += 16) {
    float v[16], w[16];
    {
      int fl = fld, kk = k;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        v[e] = 0.0f;
        w[e] = 0.0f;
        if (f0 + e < nf) {
          if (fl < 9) {
            const float *p = src[fl] + (fl == 8 ? bl : b3) + static_cast<size_t>(kk) * ny;
            v[e] = __ldg(p);
            if (fl == 8) w[e] = __ldg(p + ny);
            if (++kk == nk) {
              kk = 0;
              ++fl;
            }
          } else {
            v[e] = __ldg(src[9 + kk] + c);
            ++kk;
          }
        }
      }
    }
    uint32_t pk[8];
#pragma unroll
    for (int e = 0; e < 16; e += 2) {
      float x[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int f = f0 + e + u;
        float val = 0.0f;
        if (f < nf) {
          float r = v[e + u];
          if (fld == 1) r = logf(r);
          else if (fld == 8) r = r - w[e + u];
          const float4 sf = st[f];
          if (r < sf.z || r > sf.w) oob = 1u;
          val = (r - sf.x) * sf.y;
          if (fld < 9) {
            if (++k == nk) {
              k = 0;
              ++fld;
            }
          } else {
            ++k;
          }
        }
        x[u] = val;
      }
      const __nv_bfloat162 h = __floats2bfloat162_rn(x[0], x[1]);
      pk[e / 2] = *reinterpret_cast<const uint32_t *>(&h);
    }
    const int q = f0 / 8;
    const uint4 lo4 = make_uint4(pk[0], pk[1], pk[2], pk[3]), hi4 = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    if (kTiled) {
      uint8_t *blk = xrow + (q >> 3) * 16384;
      *reinterpret_cast<uint4 *>(blk + rr * 128 + (((q & 7) ^ (rr & 7)) << 4)) = lo4;
      *reinterpret_cast<uint4 *>(blk + rr * 128 + ((((q + 1) & 7) ^ (rr & 7)) << 4)) = hi4;
    } else {
      *reinterpret_cast<uint4 *>(xrow + f0 * 2) = lo4;
      if (f0 + 8 < a.ldx) *reinterpret_cast<uint4 *>(xrow + f0 * 2 + 16) = hi4;
    }
  }
  if (a.flags) a.flags[c] = oob;
}

// Features of a 50-level column with every index resolved at compile time:
// word W (features 2W, 2W + 1) of the output row is one expansion of
// RRTMG_FEAT_WORD(W), W = 0..255, so each load is a running field pointer,
// each statistics read a constant shared-memory slot, and words leave four at
// a time as 16-byte chunks.  A thread's chunks go to its row of the warp's
// shared staging line (at the chunk's swizzled tile position); after each
// 64-feature group the warp writes the 32 rows out as whole 128-byte lines
// (feat_flush), so no line is left half written in L2 while the rest of its
// row is computed.  Values, rounding and range flags are those of
// features_kernel.
constexpr int kFeatNk = 50;

// Writes the warp's staging line (32 rows x 8 chunks of 64-feature group kb)
// to X: lane = 4 x row + position pair, so each store instruction covers
// whole 128-byte row lines.  Slot p of row r holds chunk p ^ (row & 7).
template <bool kTiled>
__device__ __forceinline__ void feat_flush(uint8_t *X, const uint4 *stage, size_t row0, int kb, int lane,
                                           int nrows) {
  __syncwarp();
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int r = t * 8 + (lane >> 2), p0 = (lane & 3) * 2;
    if (r < nrows) {
      const size_t row = row0 + r;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int p = p0 + h;
        const uint4 v = stage[r * 8 + p];
        if (kTiled)
          *reinterpret_cast<uint4 *>(X + (row >> 7) * 131072u + kb * 16384 + (row & 127) * 128 + p * 16) = v;
        else
          *reinterpret_cast<uint4 *>(X + row * 1024 + (kb * 8 + (p ^ static_cast<int>(row & 7))) * 16) = v;
      }
    }
  }
  __syncwarp();
}

// One output word; a macro (not a function) so the 256 expansions stay in one
// straight-line body with every array index a constant.
#define RRTMG_FEAT_WORD(W)                                                                        \
  {                                                                                               \
    constexpr int W_ = (W), f_ = 2 * W_, NK_ = kFeatNk;                                           \
    if constexpr (f_ < 9 * NK_ + 4) {                                                             \
      float r0, r1;                                                                               \
      if constexpr (f_ < 8 * NK_) {                                                               \
        constexpr int F_ = f_ / NK_, k_ = f_ % NK_;                                               \
        if constexpr (k_ == 0) cur = pf[F_];                                                      \
        r0 = __ldg(cur);                                                                          \
        r1 = __ldg(cur + nys);                                                                    \
        cur += 2 * nys;                                                                           \
        if constexpr (F_ == 1) {                                                                  \
          r0 = logf(r0);                                                                          \
          r1 = logf(r1);                                                                          \
        }                                                                                         \
      } else if constexpr (f_ < 9 * NK_) {                                                        \
        constexpr int k_ = f_ - 8 * NK_;                                                          \
        if constexpr (k_ == 0) {                                                                  \
          cur = p8;                                                                               \
          pbelow = __ldg(cur);                                                                    \
        }                                                                                         \
        const float pm_ = __ldg(cur + nys), pt_ = __ldg(cur + 2 * nys);                           \
        cur += 2 * nys;                                                                           \
        r0 = pbelow - pm_;                                                                        \
        r1 = pm_ - pt_;                                                                           \
        pbelow = pt_;                                                                             \
      } else {                                                                                    \
        constexpr int q_ = f_ - 9 * NK_;                                                          \
        r0 = __ldg(two[q_]);                                                                      \
        r1 = __ldg(two[q_ + 1]);                                                                  \
      }                                                                                           \
      const float4 s0 = st[f_], s1 = st[f_ + 1];                                                  \
      oob |= static_cast<unsigned>((r0 < s0.z) | (r0 > s0.w) | (r1 < s1.z) | (r1 > s1.w));        \
      const __nv_bfloat162 h_ = __floats2bfloat162_rn((r0 - s0.x) * s0.y, (r1 - s1.x) * s1.y);    \
      ring[W_ % 4] = *reinterpret_cast<const uint32_t *>(&h_);                                    \
    } else {                                                                                      \
      ring[W_ % 4] = 0u;                                                                          \
    }                                                                                             \
    if constexpr (W_ % 4 == 3) {                                                                  \
      constexpr int q_ = W_ / 4;                                                                  \
      const uint4 v_ = make_uint4(ring[0], ring[1], ring[2], ring[3]);                            \
      line[(q_ & 7) ^ swz] = v_;                                                                  \
      if constexpr (q_ % 8 == 7) feat_flush<kTiled>(X, stage, row0, q_ / 8, lane, nrows);         \
    }                                                                                             \
  }
#define RRTMG_FEAT_W4(b) RRTMG_FEAT_WORD(b) RRTMG_FEAT_WORD((b) + 1) RRTMG_FEAT_WORD((b) + 2) RRTMG_FEAT_WORD((b) + 3)
#define RRTMG_FEAT_W16(b) RRTMG_FEAT_W4(b) RRTMG_FEAT_W4((b) + 4) RRTMG_FEAT_W4((b) + 8) RRTMG_FEAT_W4((b) + 12)
#define RRTMG_FEAT_W64(b) RRTMG_FEAT_W16(b) RRTMG_FEAT_W16((b) + 16) RRTMG_FEAT_W16((b) + 32) RRTMG_FEAT_W16((b) + 48)

// 7 resident blocks (72 registers; the field pointers spill and come back
// from L1): 0.56 ms at 1M columns against 0.71 ms at 6 blocks (80 registers)
// and 0.58 ms at 8 (64 registers, more spills).
template <bool kTiled>
__global__ void __launch_bounds__(kRowThreads, 7) features_nk50_kernel(SurFeatureArgs a) {
  constexpr int NK = kFeatNk, kNf = 9 * NK + 4;
  __shared__ float4 st[kNf];
  __shared__ uint4 stages[kRowThreads / 32][32 * 8];  // per warp: 32 rows x one 128-byte line
  for (int f = threadIdx.x; f < kNf; f += blockDim.x)
    st[f] = make_float4(a.mean[f], a.rstd[f], a.lo ? a.lo[f] : -__int_as_float(0x7f800000),
                        a.hi ? a.hi[f] : __int_as_float(0x7f800000));
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int c_raw = blockIdx.x * blockDim.x + threadIdx.x;
  const int warp_c0 = c_raw - lane;
  if (warp_c0 >= a.ncol) return;  // the whole warp
  const int nrows = min(32, a.ncol - warp_c0);
  const int c = min(c_raw, a.ncol - 1);  // lanes past the end repeat the last column, unwritten
  const int ny = a.ny;
  const size_t nys = static_cast<size_t>(ny);
  const int i = c / ny, j = c - i * ny;
  const size_t b3 = static_cast<size_t>(i) * NK * ny + j, bl = static_cast<size_t>(i) * (NK + 1) * ny + j;
  const float *const pf[8] = {a.t3d + b3, a.p3d + b3, a.qv + b3, a.qc + b3, a.qi + b3, a.qs + b3, a.cldfra + b3,
                              a.o3 + b3};
  const float *const p8 = a.p8w + bl;
  const float *const two[4] = {a.tsk + c, a.albedo + c, a.coszr + c, a.emiss + c};
  uint8_t *const X = static_cast<uint8_t *>(a.X);
  const size_t row0 = static_cast<size_t>(a.row_offset) + warp_c0;
  const int swz = static_cast<int>((row0 + lane) & 7);
  uint4 *const stage = stages[threadIdx.x >> 5];
  uint4 *const line = stage + lane * 8;
  unsigned oob = 0;
  uint32_t ring[4];
  const float *cur = nullptr;  // next level of the field being read
  float pbelow = 0.0f;         // p8w at the lower interface of the next thickness pair
  RRTMG_FEAT_W64(0) RRTMG_FEAT_W64(64) RRTMG_FEAT_W64(128) RRTMG_FEAT_W64(192)
  if (a.flags && c_raw < a.ncol) a.flags[c] = oob;
}
#undef RRTMG_FEAT_W64
#undef RRTMG_FEAT_W16
#undef RRTMG_FEAT_W4
#undef RRTMG_FEAT_WORD

__global__ void targets_kernel(SurTargetArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncol) return;
  const int nk = a.nk, ny = a.ny;
  float *t = a.T + static_cast<size_t>(a.row_offset + c) * a.ldt;
  float slw = 0.0f, ssw = 0.0f;
  for (int k = 0; k < nk; ++k) {
    const size_t q = idx3(c, k, nk, ny);
    const float pi = a.pi3d[q];
    const float hlw = a.rthratenlw[q] * 86400.0f * pi;
    const float hsw = a.rthratensw[q] * 86400.0f * pi;
    t[k] = hlw;
    t[nk + k] = hsw;
    const float dp = (a.p8w[idx3(c, k, nk + 1, ny)] - a.p8w[idx3(c, k + 1, nk + 1, ny)]) * 0.01f;
    slw += hlw * dp / kHeatfac;
    ssw += hsw * dp / kHeatfac;
  }
  const float glw = a.glw[c], lwupb = a.lwupb[c], swdnb = a.swdnb[c], swupb = a.swupb[c];
  t[2 * nk + 0] = glw;
  t[2 * nk + 1] = lwupb;
  t[2 * nk + 2] = swdnb;
  t[2 * nk + 3] = swupb;
  // LW: hr = heatfac (Fn_k - Fn_k+1) / dp with Fn = up - down; SW: Fn = down - up
  t[2 * nk + 4] = (lwupb - glw) - slw;
  t[2 * nk + 5] = (swdnb - swupb) + ssw;
  for (int f = 2 * nk + 6; f < a.ldt; ++f) t[f] = 0.0f;
}

// Per-feature mean and 1/std (and min/max) over rows [0, n): one block per
// feature, fixed reduction order.
__global__ void column_stats_kernel(const float *F, int n, int ld, int nf, float *mean, float *rstd, float *lo,
                                    float *hi) {
  const int f = blockIdx.x;
  if (f >= nf) return;
  __shared__ double s1[256], s2[256];
  __shared__ float smin[256], smax[256];
  double a1 = 0.0, a2 = 0.0;
  float mn = 3.0e38f, mx = -3.0e38f;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const float v = F[static_cast<size_t>(r) * ld + f];
    a1 += v;
    a2 += static_cast<double>(v) * v;
    mn = fminf(mn, v);
    mx = fmaxf(mx, v);
  }
  s1[threadIdx.x] = a1; s2[threadIdx.x] = a2; smin[threadIdx.x] = mn; smax[threadIdx.x] = mx;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
      smin[threadIdx.x] = fminf(smin[threadIdx.x], smin[threadIdx.x + w]);
      smax[threadIdx.x] = fmaxf(smax[threadIdx.x], smax[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double m = s1[0] / n;
    const double var = s2[0] / n - m * m;
    mean[f] = static_cast<float>(m);
    rstd[f] = var > 1.0e-20 ? static_cast<float>(1.0 / sqrt(var)) : 0.0f;
    if (lo) lo[f] = smin[0];
    if (hi) hi[f] = smax[0];
  }
}

__global__ void normalize_kernel(const float *in, int ldi, int n, int nf, const float *mean, const float *rstd,
                                 void *out, int ldo, int out_bf16) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<size_t>(n) * ldo) return;
  const int r = static_cast<int>(i / ldo), f = static_cast<int>(i - static_cast<size_t>(r) * ldo);
  const float v = f < nf ? (in[static_cast<size_t>(r) * ldi + f] - mean[f]) * rstd[f] : 0.0f;
  if (out_bf16) static_cast<__nv_bfloat16 *>(out)[i] = __float2bfloat16_rn(v);
  else static_cast<float *>(out)[i] = v;
}

// Batch gather: Xb[b] = X[idx[b]] (BF16), Xbt = Xb^T, Tb[b] = T[idx[b]] (FP32).
__global__ void gather_kernel(const __nv_bfloat16 *X, int ldx, const float *T, int ldt, const int *idx, int B,
                              __nv_bfloat16 *Xb, __nv_bfloat16 *Xbt, int ldxbt, float *Tb) {
  __shared__ __nv_bfloat16 tile[32][33];
  const int b0 = blockIdx.x * 32, f0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const int b = b0 + r, f = f0 + tx;
    if (b < B && f < ldx) {
      const __nv_bfloat16 v = X[static_cast<size_t>(idx[b]) * ldx + f];
      Xb[static_cast<size_t>(b) * ldx + f] = v;
      tile[r][tx] = v;
    }
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int f = f0 + r, b = b0 + tx;
    if (b < B && f < ldx) Xbt[static_cast<size_t>(f) * ldxbt + b] = tile[tx][r];
  }
  if (blockIdx.y == 0 && Tb) {
    for (int r = ty; r < 32; r += 8) {
      const int b = b0 + r;
      if (b >= B) continue;
      for (int f = tx; f < ldt; f += 32) Tb[static_cast<size_t>(b) * ldt + f] = T[static_cast<size_t>(idx[b]) * ldt + f];
    }
  }
}

// dY = weight * 2 (Y - T) / count as BF16 (row-major and transposed), and the
// weighted squared error summed into loss[0].
__global__ void loss_grad_kernel(const float *Y, const float *T, const float *w, int B, int ld, float scale,
                                 __nv_bfloat16 *dY, __nv_bfloat16 *dYt, int lddyt, float *loss) {
  __shared__ __nv_bfloat16 tile[32][33];
  __shared__ float part[256];
  const int b0 = blockIdx.x * 32, f0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  float acc = 0.0f;
  for (int r = ty; r < 32; r += 8) {
    const int b = b0 + r, f = f0 + tx;
    float g = 0.0f;
    if (b < B && f < ld) {
      const float d = Y[static_cast<size_t>(b) * ld + f] - T[static_cast<size_t>(b) * ld + f];
      acc += w[f] * d * d;
      g = w[f] * 2.0f * d * scale;
      dY[static_cast<size_t>(b) * ld + f] = __float2bfloat16_rn(g);
    }
    tile[r][tx] = __float2bfloat16_rn(g);
  }
  part[ty * 32 + tx] = acc;
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int f = f0 + r, b = b0 + tx;
    if (b < B && f < ld) dYt[static_cast<size_t>(f) * lddyt + b] = tile[tx][r];
  }
  for (int s = 128; s > 0; s >>= 1) {
    if (ty * 32 + tx < s) part[ty * 32 + tx] += part[ty * 32 + tx + s];
    __syncthreads();
  }
  if (tx == 0 && ty == 0 && loss) atomicAdd(loss, part[0]);
}

// db[n] = sum_b Gt[n][b] (BF16 rows), one block per row, fixed order.
__global__ void row_sum_kernel(const __nv_bfloat16 *Gt, int ld, int B, float *db) {
  __shared__ float part[256];
  float acc = 0.0f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) acc += __bfloat162float(Gt[static_cast<size_t>(blockIdx.x) * ld + b]);
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[blockIdx.x] = part[0];
}

__global__ void reduce_splits_kernel(const float *P, int splits, size_t n, float *G) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = P[i];
  for (int z = 1; z < splits; ++z) s += P[static_cast<size_t>(z) * n + i];
  G[i] = s;
}

// Adam on an FP32 master [rows][cols]; writes the BF16 copy and its transpose.
__global__ void adam_kernel(SurAdamArgs a) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const size_t n = static_cast<size_t>(a.rows) * a.cols;
  if (i >= n) return;
  const float g = a.grad[i];
  const float m = a.beta1 * a.m[i] + (1.0f - a.beta1) * g;
  const float v = a.beta2 * a.v[i] + (1.0f - a.beta2) * g * g;
  a.m[i] = m;
  a.v[i] = v;
  const float mhat = m / a.bc1, vhat = v / a.bc2;
  const float w = a.w[i] - a.lr * (mhat / (sqrtf(vhat) + a.eps) + a.weight_decay * a.w[i]);
  a.w[i] = w;
  const int r = static_cast<int>(i / a.cols), c = static_cast<int>(i - static_cast<size_t>(r) * a.cols);
  if (a.wb) static_cast<__nv_bfloat16 *>(a.wb)[static_cast<size_t>(r) * a.ldwb + c] = __float2bfloat16_rn(w);
  if (a.wbt) static_cast<__nv_bfloat16 *>(a.wbt)[static_cast<size_t>(c) * a.ldwbt + r] = __float2bfloat16_rn(w);
}

// Decode normalized network outputs into WRF fields and apply the energy gate.
// A block of kDecCols columns first copies their output rows (contiguous) into
// shared memory, then each thread decodes one column.
constexpr int kDecCols = 64, kDecWidth = 128;

__global__ void __launch_bounds__(kDecCols) decode_kernel(SurDecodeArgs a) {
  __shared__ float ys[kDecCols][kDecWidth + 1];
  const int c0 = blockIdx.x * kDecCols;
  const int nk = a.nk, ny = a.ny;
  const int width = 2 * nk + 6;
  for (int e = threadIdx.x; e < kDecCols * width; e += blockDim.x) {
    const int lc = e / width, f = e - lc * width;
    const int c = c0 + lc;
    ys[lc][f] = c < a.ncol ? a.Y[static_cast<size_t>(c) * a.ldy + f] * a.out_std[f] + a.out_mean[f] : 0.0f;
  }
  __syncthreads();
  const int c = c0 + threadIdx.x;
  if (c >= a.ncol) return;
  const float *y = ys[threadIdx.x];
  const bool day = a.coszr[c] > 0.0f;
  float slw = 0.0f, ssw = 0.0f;
  for (int k = 0; k < nk; ++k) {
    const size_t q = idx3(c, k, nk, ny);
    const float pi = a.pi3d[q];
    const float hlw = y[k];
    const float hsw = day ? y[nk + k] : 0.0f;
    a.rthratenlw[q] = sur_tendency(hlw, pi);
    a.rthratensw[q] = sur_tendency(hsw, pi);
    const float dp = (a.p8w[idx3(c, k, nk + 1, ny)] - a.p8w[idx3(c, k + 1, nk + 1, ny)]) * 0.01f;
    slw += sur_flux_term(hlw, dp);
    ssw += sur_flux_term(hsw, dp);
  }
  const float glw = y[2 * nk], lwupb = y[2 * nk + 1];
  const float swdnb = day ? y[2 * nk + 2] : 0.0f, swupb = day ? y[2 * nk + 3] : 0.0f;
  a.glw[c] = glw;
  a.lwupb[c] = lwupb;
  a.swdnb[c] = swdnb;
  a.swupb[c] = swupb;
  // energy gate: column-integrated heating against net surface minus model-top flux
  const float lw_res = fabsf(((lwupb - glw) - y[2 * nk + 4]) - slw);
  const float sw_res = day ? fabsf((y[2 * nk + 5] - (swdnb - swupb)) - ssw) : 0.0f;
  unsigned f = a.flags[c];
  if (!(lw_res <= a.energy_tol) || !(sw_res <= a.energy_tol)) f |= 2u;
  a.flags[c] = f;
}

__global__ void timestamp_kernel(unsigned long long *slot) {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  *slot = t;
}

// Append flagged columns to a list (one atomic per warp).
__global__ void compact_kernel(const unsigned *flags, int ncol, int *list, int *count) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool sel = c < ncol && flags[c] != 0u;
  const unsigned ballot = __ballot_sync(0xffffffffu, sel);
  int base = 0;
  if (lane == 0 && ballot) base = atomicAdd(count, __popc(ballot));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (sel) list[base + __popc(ballot & ((1u << lane) - 1u))] = c;
}

// Gather (to_compact = 1) or scatter (0) a field between a domain and the
// compact (1, nz, n) domain of listed columns.
__global__ void move_columns_kernel(const int *list, const int *count, int max_n, int nz, int ny, const float *src,
                                    float *dst, int to_compact, int stride, int offset) {
  const int n = min(*count, max_n);  // the compact side holds max_n columns
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nz) return;
  const int k = t / n, j = t - k * n;
  const int c = list[j];
  const size_t full = idx3(c, k, nz, ny);
  const size_t comp = static_cast<size_t>(k) * stride + offset + j;
  if (to_compact) dst[comp] = src[full];
  else dst[full] = src[comp];
}

// Several fields in one launch: blockIdx.y = field, grid-stride over its
// (level, listed column) pairs.
__global__ void move_fields_kernel(const int *list, const int *count, int max_n, int ny, rrtmg_sur_fields f,
                                   int to_compact, int stride, int offset) {
  const int field = blockIdx.y;
  const int n = min(*count, max_n), nz = f.nz[field];  // the compact side holds max_n columns
  const float *src = f.src[field];
  float *dst = f.dst[field];
  const long long total = static_cast<long long>(n) * nz;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(t / n), j = static_cast<int>(t - static_cast<long long>(k) * n);
    const int c = list[j];
    const size_t full = idx3(c, k, nz, ny);
    const size_t comp = static_cast<size_t>(k) * stride + offset + j;
    if (to_compact) dst[comp] = src[full];
    else dst[full] = src[comp];
  }
}

}  // namespace

cudaError_t launch_sur_move_fields(const int *list, const int *count, int max_n, int ny, const rrtmg_sur_fields &f,
                                   int to_compact, int stride, int offset, cudaStream_t s) {
  int max_nz = 0;
  for (int i = 0; i < f.nfields; ++i) max_nz = f.nz[i] > max_nz ? f.nz[i] : max_nz;
  const long long total = static_cast<long long>(max_n) * max_nz;
  if (total == 0 || f.nfields == 0) return cudaSuccess;
  long long blocks = (total + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  move_fields_kernel<<<dim3(static_cast<unsigned>(blocks), f.nfields), 256, 0, s>>>(list, count, max_n, ny, f,
                                                                                     to_compact, stride, offset);
  return cudaGetLastError();
}

cudaError_t launch_sur_features(const SurFeatureArgs &a, cudaStream_t s) {
  const unsigned row_blocks = static_cast<unsigned>((a.ncol + kRowThreads - 1) / kRowThreads);
  const bool rows_ok = a.X && !a.raw && !a.Xt && a.ldx % 8 == 0 && 9 * a.nk + 4 <= kMaxFeatures &&
                       (reinterpret_cast<uintptr_t>(a.X) & 15u) == 0;
  if (a.x_layout == 1 && !rows_ok) return cudaErrorInvalidValue;
  if (rows_ok && a.nk == kFeatNk && a.ldx == 512) {
    if (a.x_layout == 1)
      features_nk50_kernel<true><<<row_blocks, kRowThreads, 0, s>>>(a);
    else
      features_nk50_kernel<false><<<row_blocks, kRowThreads, 0, s>>>(a);
    return cudaGetLastError();
  }
  if (a.x_layout == 1)
    features_rows_kernel<true><<<row_blocks, kRowThreads, 0, s>>>(a);
  else if (a.x_layout == 0 && rows_ok)
    features_rows_kernel<false><<<row_blocks, kRowThreads, 0, s>>>(a);
  else
    features_kernel<<<(a.ncol + kFeatCols - 1) / kFeatCols, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_sur_targets(const SurTargetArgs &a, cudaStream_t s) {
  targets_kernel<<<(a.ncol + 127) / 128, 128, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_sur_column_stats(const float *F, int n, int ld, int nf, float *mean, float *rstd, float *lo,
                                    float *hi, cudaStream_t s) {
  column_stats_kernel<<<nf, 256, 0, s>>>(F, n, ld, nf, mean, rstd, lo, hi);
  return cudaGetLastError();
}

cudaError_t launch_sur_normalize(const float *in, int ldi, int n, int nf, const float *mean, const float *rstd,
                                 void *out, int ldo, int out_bf16, cudaStream_t s) {
  const size_t total = static_cast<size_t>(n) * ldo;
  normalize_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(in, ldi, n, nf, mean, rstd, out, ldo,
                                                                              out_bf16);
  return cudaGetLastError();
}

cudaError_t launch_sur_gather(const __nv_bfloat16 *X, int ldx, const float *T, int ldt, const int *idx, int B,
                              __nv_bfloat16 *Xb, __nv_bfloat16 *Xbt, int ldxbt, float *Tb, cudaStream_t s) {
  dim3 grid((B + 31) / 32, (ldx + 31) / 32);
  gather_kernel<<<grid, dim3(32, 8), 0, s>>>(X, ldx, T, ldt, idx, B, Xb, Xbt, ldxbt, Tb);
  return cudaGetLastError();
}

cudaError_t launch_sur_loss_grad(const float *Y, const float *T, const float *w, int B, int ld, float scale,
                                 __nv_bfloat16 *dY, __nv_bfloat16 *dYt, int lddyt, float *loss, cudaStream_t s) {
  dim3 grid((B + 31) / 32, (ld + 31) / 32);
  loss_grad_kernel<<<grid, dim3(32, 8), 0, s>>>(Y, T, w, B, ld, scale, dY, dYt, lddyt, loss);
  return cudaGetLastError();
}

cudaError_t launch_sur_row_sum(const __nv_bfloat16 *Gt, int ld, int rows, int B, float *db, cudaStream_t s) {
  row_sum_kernel<<<rows, 256, 0, s>>>(Gt, ld, B, db);
  return cudaGetLastError();
}

cudaError_t launch_sur_reduce_splits(const float *P, int splits, size_t n, float *G, cudaStream_t s) {
  reduce_splits_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(P, splits, n, G);
  return cudaGetLastError();
}

cudaError_t launch_sur_adam(const SurAdamArgs &a, cudaStream_t s) {
  const size_t n = static_cast<size_t>(a.rows) * a.cols;
  adam_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_sur_decode(const SurDecodeArgs &a, cudaStream_t s) {
  decode_kernel<<<(a.ncol + kDecCols - 1) / kDecCols, kDecCols, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_sur_compact(const unsigned *flags, int ncol, int *list, int *count, cudaStream_t s) {
  compact_kernel<<<(ncol + 255) / 256, 256, 0, s>>>(flags, ncol, list, count);
  return cudaGetLastError();
}

cudaError_t launch_sur_move_columns(const int *list, const int *count, int max_n, int nz, int ny, const float *src,
                                    float *dst, int to_compact, int stride, int offset, cudaStream_t s) {
  const long long total = static_cast<long long>(max_n) * nz;
  if (total == 0) return cudaSuccess;
  move_columns_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(list, count, max_n, nz, ny, src,
                                                                                 dst, to_compact, stride, offset);
  return cudaGetLastError();
}

cudaError_t launch_timestamp(unsigned long long *slot, cudaStream_t s) {
  timestamp_kernel<<<1, 1, 0, s>>>(slot);
  return cudaGetLastError();
}

}  // namespace rrtmg

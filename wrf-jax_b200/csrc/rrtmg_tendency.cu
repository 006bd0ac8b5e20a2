// Radiation tendency chain after the RRTMG calls, fused: LW + SW heating,
// mass coupling over the tile, accumulation into the potential-temperature
// tendency over the a2a region.  One thread per element, threads over the
// south-north index (the fastest one), blocks over west-east x level rows.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>

#include "../../include/rrtmg_tendency.h"

namespace {

constexpr int kThreads = 256;

// Half-open index ranges in memory coordinates.
struct Box {
  int i0, i1, k0, k1, j0, j1;
  __device__ __forceinline__ bool has(int i, int k, int j) const {
    return (i >= i0) & (i < i1) & (k >= k0) & (k < k1) & (j >= j0) & (j < j1);
  }
};

struct TendArgs {
  int nx, nk, ny;
  const float *lw, *sw, *c1, *c2, *mut;
  float *rthraten, *rt_tendf;
  int couple;
  Box tile, a2a;
};

__global__ void __launch_bounds__(kThreads) tendency_kernel(const TendArgs a) {
  const int j = blockIdx.x * kThreads + threadIdx.x;
  if (j >= a.ny) return;
  const int rows = a.nx * a.nk;
  for (int row = blockIdx.y; row < rows; row += gridDim.y) {
    const int i = row / a.nk, k = row - i * a.nk;
    const size_t e = static_cast<size_t>(row) * a.ny + j;
    // runtime.py:7946
    float r = a.sw ? __fadd_rn(__ldg(a.lw + e), __ldg(a.sw + e)) : __ldg(a.lw + e);
    // module_em.py:597-601: factor = c1 * mut (rounded) + c2 (rounded); field * factor
    if (a.couple && a.tile.has(i, k, j)) {
      const float factor = __fadd_rn(__fmul_rn(__ldg(a.c1 + k), __ldg(a.mut + static_cast<size_t>(i) * a.ny + j)),
                                     __ldg(a.c2 + k));
      r = __fmul_rn(r, factor);
    }
    if (a.rthraten) a.rthraten[e] = r;
    // module_physics_addtendc.py:204: lvar.at[region].add(rvar[region])
    if (a.rt_tendf && a.a2a.has(i, k, j)) a.rt_tendf[e] = __fadd_rn(a.rt_tendf[e], r);
  }
}

// Four consecutive south-north elements per thread (ny % 4 == 0, 16-byte
// aligned arrays) and two rows per iteration: six 16-byte loads in flight per
// thread, enough to cover DRAM latency at full occupancy.
__device__ __forceinline__ float4 ld4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }

__device__ __forceinline__ void tendency4(const TendArgs &a, int row, int j, float4 lw, float4 sw, float4 t) {
  const int i = row / a.nk, k = row - i * a.nk;
  const size_t e = static_cast<size_t>(row) * a.ny + j;
  float r[4] = {lw.x, lw.y, lw.z, lw.w};
  const float s[4] = {sw.x, sw.y, sw.z, sw.w};
  float tt[4] = {t.x, t.y, t.z, t.w};
  float m[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  const bool couple_row = a.couple && (i >= a.tile.i0) & (i < a.tile.i1) & (k >= a.tile.k0) & (k < a.tile.k1);
  if (couple_row) {
    const float4 mm = ld4(a.mut + static_cast<size_t>(i) * a.ny + j);
    m[0] = mm.x; m[1] = mm.y; m[2] = mm.z; m[3] = mm.w;
  }
  const float c1 = couple_row ? __ldg(a.c1 + k) : 0.0f, c2 = couple_row ? __ldg(a.c2 + k) : 0.0f;
  const bool add_row = (i >= a.a2a.i0) & (i < a.a2a.i1) & (k >= a.a2a.k0) & (k < a.a2a.k1);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (a.sw) r[q] = __fadd_rn(r[q], s[q]);
    if (couple_row && (j + q >= a.tile.j0) & (j + q < a.tile.j1)) r[q] = __fmul_rn(r[q], __fadd_rn(__fmul_rn(c1, m[q]), c2));
    if (add_row && (j + q >= a.a2a.j0) & (j + q < a.a2a.j1)) tt[q] = __fadd_rn(tt[q], r[q]);
  }
  if (a.rthraten) *reinterpret_cast<float4 *>(a.rthraten + e) = make_float4(r[0], r[1], r[2], r[3]);
  if (a.rt_tendf && add_row) *reinterpret_cast<float4 *>(a.rt_tendf + e) = make_float4(tt[0], tt[1], tt[2], tt[3]);
}

__global__ void __launch_bounds__(kThreads) tendency_kernel_vec4(const TendArgs a) {
  const int j = (blockIdx.x * kThreads + threadIdx.x) * 4;
  if (j >= a.ny) return;
  const int rows = a.nx * a.nk;
  const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  for (int row = 2 * blockIdx.y; row < rows; row += 2 * gridDim.y) {
    const bool two = row + 1 < rows;
    const size_t e0 = static_cast<size_t>(row) * a.ny + j, e1 = e0 + a.ny;
    const float4 lw0 = ld4(a.lw + e0), lw1 = two ? ld4(a.lw + e1) : zero;
    const float4 sw0 = a.sw ? ld4(a.sw + e0) : zero, sw1 = (a.sw && two) ? ld4(a.sw + e1) : zero;
    const float4 t0 = a.rt_tendf ? *reinterpret_cast<const float4 *>(a.rt_tendf + e0) : zero;
    const float4 t1 = (a.rt_tendf && two) ? *reinterpret_cast<const float4 *>(a.rt_tendf + e1) : zero;
    tendency4(a, row, j, lw0, sw0, t0);
    if (two) tendency4(a, row + 1, j, lw1, sw1, t1);
  }
}

Box make_box(int i0, int i1, int k0, int k1, int j0, int j1, const rrtmg_tendency_bounds &b) {
  // inclusive Fortran bounds -> half-open memory ranges (empty when reversed)
  Box x;
  x.i0 = i0 - b.ims;
  x.i1 = std::max(i1 - b.ims + 1, x.i0);
  x.k0 = k0 - b.kms;
  x.k1 = std::max(k1 - b.kms + 1, x.k0);
  x.j0 = j0 - b.jms;
  x.j1 = std::max(j1 - b.jms + 1, x.j0);
  return x;
}

}  // namespace

extern "C" rrtmg_status rrtmg_radiation_tendency(const rrtmg_tendency_bounds *bp, const float *lw, const float *sw,
                                                 const float *c1, const float *c2, const float *mut, int couple,
                                                 float *rthraten, float *rt_tendf, void *stream) {
  if (!bp || !lw || (!rthraten && !rt_tendf)) return RRTMG_BAD_ARG;
  if (couple && (!c1 || !c2 || !mut)) return RRTMG_BAD_ARG;
  const rrtmg_tendency_bounds &b = *bp;
  const long long nx = static_cast<long long>(b.ime) - b.ims + 1, nk = static_cast<long long>(b.kme) - b.kms + 1,
                  ny = static_cast<long long>(b.jme) - b.jms + 1;
  if (nx < 1 || nk < 1 || ny < 1 || nx * nk * ny > INT_MAX) return RRTMG_BAD_ARG;
  TendArgs a{};
  a.nx = static_cast<int>(nx);
  a.nk = static_cast<int>(nk);
  a.ny = static_cast<int>(ny);
  a.lw = lw;
  a.sw = sw;
  a.c1 = c1;
  a.c2 = c2;
  a.mut = mut;
  a.rthraten = rthraten;
  a.rt_tendf = rt_tendf;
  a.couple = couple != 0;
  // calculate_phy_tend's region (module_em.py:577-593)
  const int itf = std::min(b.ite, b.ide - 1), jtf = std::min(b.jte, b.jde - 1), ktf = std::min(b.kte, b.kde - 1);
  a.tile = make_box(b.its, itf, b.kts, ktf, b.jts, jtf, b);
  // add_a2a's region (module_physics_addtendc.py:131-170)
  int i0 = b.its, i1 = itf, j0 = b.jts, j1 = jtf;
  if (b.specified || b.nested) {
    i0 = std::max(b.ids + 1, b.its);
    i1 = std::min(b.ide - 2, b.ite);
    j0 = std::max(b.jds + 1, b.jts);
    j1 = std::min(b.jde - 2, b.jte);
  }
  if (b.periodic_x) {
    i0 = b.its;
    i1 = itf;
  }
  a.a2a = make_box(i0, i1, b.kts, ktf, j0, j1, b);
  auto aligned = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  const bool vec4 = (a.ny % 4 == 0) && aligned(lw) && aligned(sw) && aligned(mut) && aligned(rthraten) &&
                    aligned(rt_tendf);
  const long long rows = nx * nk;
  const int per_thread = vec4 ? 4 : 1, rows_per_iter = vec4 ? 2 : 1;
  const int bx = static_cast<int>((a.ny + static_cast<long long>(kThreads) * per_thread - 1) /
                                  (static_cast<long long>(kThreads) * per_thread));
  // one block per row (pair) up to the grid's y limit; more rows loop
  const int by = static_cast<int>(std::min<long long>((rows + rows_per_iter - 1) / rows_per_iter, 65535));
  const dim3 grid(bx, by);
  if (vec4)
    tendency_kernel_vec4<<<grid, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(a);
  else
    tendency_kernel<<<grid, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(a);
  return cudaGetLastError() == cudaSuccess ? RRTMG_OK : RRTMG_CUDA;
}

extern "C" rrtmg_status rrtmg_phy_ra_ten(const rrtmg_tendency_bounds *b, float *rt_tendf, const float *rthraten,
                                         void *stream) {
  if (!rt_tendf) return RRTMG_BAD_ARG;
  return rrtmg_radiation_tendency(b, rthraten, nullptr, nullptr, nullptr, nullptr, 0, nullptr, rt_tendf, stream);
}

// McICA stochastic cloud masks on the GPU.
//
// Reference: generate_stochastic_clouds_overlap2 and the KISS stream
// (src/wrf_jax/physics/module_ra_rrtmg_common.py:964-1153).  The stream of one
// column is seeded from the fractional digits of its four lowest layer
// pressures and consumed in (subcolumn, layer) order after `skip` discarded
// draws (150 for LW, 1 for SW).  Here one thread owns one (column, subcolumn):
// it jumps the four KISS recurrences straight to draw skip + g*nlay with a
// host-computed jump (integer arithmetic, identical to sequential stepping),
// runs the maximum-random overlap chain up the column, and each warp ballots
// its 32 cloudy bits per layer into one mask word.
//
// Mask layout: mask[(l * words + w) * ncol + c], bit (g % 32) of word g / 32.
#include "rrtmg_device.cuh"
#include "rrtmg_kernels.h"

namespace rrtmg {

__global__ void __launch_bounds__(256) mcica_mask_kernel(McicaArgs a) {
  const int warps_per_col = a.words;
  const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int col = gwarp / warps_per_col;
  const int w = gwarp - col * warps_per_col;
  if (col >= a.ncol || dead_column(a.live, col)) return;  // whole warp exits together
  const int g = w * 32 + lane;
  const bool active = g < a.nsub;
  const int i = col / a.ny, j = col - i * a.ny;
  const int nk = a.nk;

  // seeds from pmid = play * 100 of the four lowest layers (common:1000-1004)
  Kiss s;
  {
    float pm[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float play = pa_to_hpa(ld(a.p3d + (static_cast<size_t>(i) * nk + k) * a.ny + j));
      pm[k] = play * 100.0f;
    }
    s.s1 = kiss_seed(pm[0]);
    s.s2 = kiss_seed(pm[1]);
    s.s3 = kiss_seed(pm[2]);
    s.s4 = kiss_seed(pm[3]);
  }
  if (active) s = kiss_jump(s, a.jumps[g]);

  float cdf_prev = 0.0f, thr_prev = 1.0f;
  for (int l = 0; l < a.nlay; ++l) {
    float cld = 0.0f;
    if (l < nk) cld = ld(a.cldfra + (static_cast<size_t>(i) * nk + l) * a.ny + j);
    if (cld < 1.0e-20f) cld = 0.0f;
    bool cloudy = false;
    if (active) {
      const float ran = s.next();
      float cdf = ran;
      if (l > 0) cdf = (cdf_prev > thr_prev) ? cdf_prev : ran * thr_prev;
      cloudy = a.enabled && (cdf >= 1.0f - cld);
      cdf_prev = cdf;
      thr_prev = 1.0f - cld;
    }
    const unsigned word = __ballot_sync(0xffffffffu, cloudy);
    if (lane == 0) a.mask[(static_cast<size_t>(l) * warps_per_col + w) * a.ncol + col] = word;
  }
}

cudaError_t launch_mcica(const McicaArgs &a, cudaStream_t stream) {
  const int threads = 256;
  const long long total = static_cast<long long>(a.ncol) * a.words * 32;
  const int blocks = static_cast<int>((total + threads - 1) / threads);
  mcica_mask_kernel<<<blocks, threads, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace rrtmg

// Per-column status of the last LW / SW call (rrtmg_last_column_errors).
//
// The reference has no runtime checks on its inputs (NaN, ordering or range
// errors propagate silently into the outputs).  While column status is
// enabled on a context, every LW / SW call ends with one extra launch of
// column_status_kernel on the call's stream: a thread per column reads the
// column's inputs and outputs once (level-major, so a warp's loads at each
// level are 32 consecutive floats) and writes a bitmask of the conditions
// below into the context's status array for that side.
#include <cuda_runtime.h>

#include "rrtmg_kernels.h"

namespace rrtmg {
namespace {

__device__ __forceinline__ bool finite(float v) { return isfinite(v); }

// T outside the Planck / reference-temperature tables: LW indexes
// totplnk with clip(int(T - 159), 1, 180), so T < 160 K or T >= 340 K is
// clamped to the table's edge.
__device__ __forceinline__ bool temp_out(float t) { return !(t >= 160.0f && t < 340.0f); }

__device__ __forceinline__ bool frac_out(float v) { return !(v >= 0.0f && v <= 1.0f); }

__global__ void __launch_bounds__(256) column_status_kernel(StatusArgs a) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= a.ncol) return;
  const int i = col / a.ny, j = col - i * a.ny;
  const size_t b3 = static_cast<size_t>(i) * a.nk * a.ny + j;
  const size_t bw = static_cast<size_t>(i) * (a.nk + 1) * a.ny + j;
  const size_t ny = static_cast<size_t>(a.ny);
  uint32_t s = 0;
  bool bad_in = false, bad_out = false;
  // inputs: level fields, then layer fields
  float pw_prev = 0.0f;
  for (int k = 0; k <= a.nk; ++k) {
    const float pw = ld(a.in.p8w + bw + k * ny), tw = ld(a.in.t8w + bw + k * ny);
    bad_in |= !finite(pw) || !finite(tw);
    if (temp_out(tw)) s |= RRTMG_COL_TEMPERATURE_RANGE;
    if (k > 0 && !(pw < pw_prev)) s |= RRTMG_COL_PRESSURE_ORDER;
    pw_prev = pw;
  }
  for (int k = 0; k < a.nk; ++k) {
    const size_t o = b3 + k * ny;
    const float p = ld(a.in.p3d + o), t = ld(a.in.t3d + o), cf = ld(a.in.cldfra + o);
    const float qv = ld(a.in.qv + o), qc = ld(a.in.qc + o), qi = ld(a.in.qi + o), qs = ld(a.in.qs + o);
    const float o3 = ld(a.in.o3 + o), pi = ld(a.in.pi3d + o);
    bad_in |= !finite(p) || !finite(t) || !finite(cf) || !finite(qv) || !finite(qc) || !finite(qi) ||
              !finite(qs) || !finite(o3) || !finite(pi);
    if (temp_out(t)) s |= RRTMG_COL_TEMPERATURE_RANGE;
    if (frac_out(cf)) s |= RRTMG_COL_FRACTION_RANGE;
    // the layer's pressure lies between its interfaces
    const float pb = ld(a.in.p8w + bw + k * ny), pt = ld(a.in.p8w + bw + (k + 1) * ny);
    if (!(p <= pb && p >= pt)) s |= RRTMG_COL_PRESSURE_ORDER;
    if (a.has_req) {
      bad_in |= !finite(ld(a.in.re_cloud + o)) || !finite(ld(a.in.re_ice + o)) || !finite(ld(a.in.re_snow + o));
    }
  }
  const float tsk = ld(a.in.tsk + col);
  bad_in |= !finite(tsk) || !finite(ld(a.in.xland + col)) || !finite(ld(a.in.xice + col)) ||
            !finite(ld(a.in.snow + col));
  if (temp_out(tsk)) s |= RRTMG_COL_TEMPERATURE_RANGE;
  if (a.side == 0) {
    const float e = ld(a.in.emiss + col);
    bad_in |= !finite(e);
    if (frac_out(e)) s |= RRTMG_COL_FRACTION_RANGE;
  } else {
    const float al = ld(a.in.albedo + col), cz = ld(a.in.coszr + col);
    bad_in |= !finite(al) || !finite(cz);
    if (frac_out(al) || cz > 1.0f) s |= RRTMG_COL_FRACTION_RANGE;
  }
  // outputs of this call
  for (int k = 0; k < a.nk; ++k) {
    const size_t o = b3 + k * ny;
    bad_out |= !finite(a.rthraten[o]) || !finite(a.rthratenc[o]);
  }
  for (int q = 0; q < a.n2d; ++q) bad_out |= !finite(a.out2d[q][col]);
  if (bad_in) s |= RRTMG_COL_NONFINITE_INPUT;
  if (bad_out) s |= RRTMG_COL_NONFINITE_OUTPUT;
  a.status[col] = s;
}

}  // namespace

cudaError_t launch_column_status(const StatusArgs &a, cudaStream_t stream) {
  if (a.ncol <= 0) return cudaSuccess;
  column_status_kernel<<<(a.ncol + 255) / 256, 256, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace rrtmg

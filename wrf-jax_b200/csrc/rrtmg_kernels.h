// Kernel argument blocks and launchers (internal to librrtmg_b200.so).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/rrtmg_b200.h"
#include "rrtmg_device.cuh"

namespace rrtmg {

// Columns at or past a device-side live count are skipped (null: all).
__device__ __forceinline__ bool dead_column(const int *live, int col) { return live && col >= *live; }

struct McicaArgs {
  int ncol, ny, nk, nlay, nsub, words, enabled;
  const float *p3d, *cldfra;
  const KissJump *jumps;  // one per subcolumn
  uint32_t *mask;         // (nlay, words, ncol)
  const int *live;        // null, or a device count of leading columns to process
};

// Per-column inputs shared by LW and SW (WRF layout, device pointers).
struct ColumnInputs {
  const float *p3d, *p8w, *pi3d, *t3d, *t8w, *tsk;
  const float *qv, *qc, *qi, *qs, *cldfra, *o3;
  const float *emiss, *albedo, *coszr, *xland, *xice, *snow;
  const float *re_cloud, *re_ice, *re_snow;
  // SW only, optional (all four or none): Noah-MP albedos of xland < 1.5 columns
  const float *alswvisdir, *alswvisdif, *alswnirdir, *alswnirdif;
};

struct LwArgs {
  int nx, ny, nk, nlay, ncol;
  float co2, n2o, ch4, cfc11, cfc12;
  int has_reqc, has_reqi, has_reqs, icloud, icld;
  int inflg, iceflg, liqflg;
  ColumnInputs in;
  const uint32_t *mask;
  float *rthraten, *rthratenc;
  float *upt, *uptc, *dnt, *dntc, *upb, *upbc, *dnb, *dnbc, *glw, *olr, *lwcf;
  float *zero2[4];  // *cln fields, written as zeros
  float *scratch;       // sweep schedule: lw_scratch_floats(nlay, chunk_capacity) floats
  int chunk_capacity;   // columns per chunk of the sweep schedule
  int chunk_first, chunk_count;  // the chunk being launched
  const int *live;  // null, or a device count of leading columns to process
  int fp64_from;    // FP64 mode: first layer with a binary64 heating rate; kMaxLay + 1 = off
};

// default columns per chunk of the LW sweep schedule (its scratch takes about
// 107 KB per column at nk = 50 and a 50 hPa top)
constexpr int kLwChunkColumns = 16384;
// no longer used by the LW path (every domain runs the sweep schedule); kept
// as the default of the schedule field that used to select the split schedule
constexpr int kLwSplitMaxColumns = 2048;

struct SwArgs {
  int nx, ny, nk, nlay, ncol;
  float co2, n2o, ch4, solcon;
  int has_reqc, has_reqi, has_reqs, icloud, icld;
  int inflg, iceflg, liqflg;
  ColumnInputs in;
  const uint32_t *mask;
  float *rthraten, *rthratenc;
  float *upt, *uptc, *dnt, *dntc, *upb, *upbc, *dnb, *dnbc;
  float *swcf, *gsw, *swddir, *swddni, *swddif, *swdownc, *swddnic, *swddirc, *coszr_out;
  float *zero2[4];
  int *nday;     // scratch: number of day columns (set by the compaction kernel)
  int *daylist;  // scratch: ncol entries, day column indices
  float *records;      // scratch: sw_record_floats(nk, chunk_capacity) floats
  int chunk_capacity;  // day-list slots per chunk of the sweep schedule
  int chunk_first, chunk_count;  // the chunk being launched (set by launch_sw_columns)
  const int *live;     // null, or a device count of leading columns to process
  int fp64_from;       // FP64 mode: first layer with a binary64 heating rate; kMaxLay + 1 = off
  int fp64_reftra;     // FP64 mode: reftra in binary64 where zwo >= 0.999 or zto1 < 0.1
};

// default day-list slots per chunk of the SW sweep schedule (its records take
// about 64 KB per slot at nk = 50)
constexpr int kSwChunkColumns = 32768;
// no longer used by the SW path (every domain runs the sweep schedule); kept
// as the default of the schedule field that used to select it
constexpr int kSwSplitMaxColumns = 4096;

cudaError_t launch_mcica(const McicaArgs &a, cudaStream_t stream);
// fused schedule (one thread per column, no scratch)
cudaError_t launch_lw(const Tables &T, const LwArgs &a, cudaStream_t stream);
// sweep schedule, one chunk of columns (a.chunk_first, a.chunk_count) at a
// time: the optics launches (column set-up, layer set-up, gas optics), then
// the sweep launch (radiative transfer, flux sums, heating, outputs)
size_t lw_scratch_floats(int nlay, int chunk);
cudaError_t launch_lw_chunk_optics(const Tables &T, const LwArgs &a, cudaStream_t stream);
cudaError_t launch_lw_chunk_sweep(const Tables &T, const LwArgs &a, cudaStream_t stream);
// day-column compaction (writes the night columns; needs a.nday and a.daylist,
// 1 + ncol ints), then per chunk of day-list slots the optics launches (column
// set-up, layer optics, solar source) and the sweep launch
cudaError_t launch_sw_daylist(const SwArgs &a, cudaStream_t stream);
size_t sw_record_floats(int nk, int chunk);
cudaError_t launch_sw_chunk_optics(const Tables &T, const SwArgs &a, cudaStream_t stream);
cudaError_t launch_sw_chunk_sweep(const Tables &T, const SwArgs &a, cudaStream_t stream);

// Per-column status of one LW (side 0) or SW (side 1) call: its inputs and
// outputs (rrtmg_last_column_errors).
struct StatusArgs {
  int ncol, nx, ny, nk, side, has_req;
  ColumnInputs in;
  const float *rthraten, *rthratenc;
  const float *out2d[8];
  int n2d;
  uint32_t *status;  // ncol words
};
cudaError_t launch_column_status(const StatusArgs &a, cudaStream_t stream);

// Radiation prologue (cloud fraction, cos zenith, CAM ozone).  Constants of
// the SVML sin/cos emulation in the reference's order (svml.sinf: 12,
// svml.cosf: 14 values).
struct SvmlConsts {
  float s[12];
  float c[14];
};

struct PrologueArgs {
  int nx, nk, ny;
  const float *qv, *qc, *qi, *qs, *t, *p;  // (nx, nk, ny)
  const float *xlat, *xlong;               // (nx, ny)
  float *cldfra, *o33d, *coszr;            // outputs; null: not computed
  int *condensate;                         // null, or a zeroed device flag
  float tloctm0, sin_declin, cos_declin;
  SvmlConsts svml;
  const float *oz_plev, *oz_lat, *oz_tab;  // device climatology: (levsiz), (latsiz), (12, latsiz, levsiz)
  int levsiz, latsiz, month_lo, month_hi;
  float fact_lo, fact_hi;
};

size_t prologue_smem_bytes(int levsiz, int latsiz);

// Makes `device` current for the guard's lifetime and restores the caller's
// current device when it goes out of scope, so an entry point leaves the
// calling thread's device as it found it.
class DeviceGuard {
 public:
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&prev_) != cudaSuccess) {
      cudaGetLastError();
      prev_ = -1;
    }
    status_ = prev_ == device ? cudaSuccess : cudaSetDevice(device);
    switched_ = status_ == cudaSuccess && prev_ >= 0 && prev_ != device;
  }
  ~DeviceGuard() {
    if (switched_) cudaSetDevice(prev_);
  }
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;
  cudaError_t status() const { return status_; }

 private:
  int prev_ = -1;
  bool switched_ = false;
  cudaError_t status_ = cudaSuccess;
};

// Records an error of a call without a context (text for rrtmg_last_error(NULL)).
rrtmg_status create_error(rrtmg_status status, const std::string &message);
cudaError_t launch_prologue(const PrologueArgs &a, cudaStream_t stream);

}  // namespace rrtmg

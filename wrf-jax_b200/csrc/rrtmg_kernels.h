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
  float *terms;     // band-group schedule scratch, lw_terms_floats(nk, chunk_count) floats
  float *optics;    // g-point split schedule: lw_optics_floats(nlay, chunk_count) floats, else null
  int chunk_first, chunk_count;  // columns of one band-group/finish launch pair
  const int *live;  // null, or a device count of leading columns to process
};

// default columns per band-group/finish launch pair (the term scratch holds one chunk)
constexpr int kLwChunkColumns = 131072;
// Domains of at most this many columns run the LW g-point split schedule
// (its optics scratch: 1,376 bytes per column and layer).
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
// band-group schedule (thread per column and band group), then the finish
// kernel (ordered band sums, fluxes, heating); both need a.terms
size_t lw_terms_floats(int nk, int ncol);
cudaError_t launch_lw_groups(const Tables &T, const LwArgs &a, cudaStream_t stream);
cudaError_t launch_lw_finish(const LwArgs &a, cudaStream_t stream);
// g-point split schedule for small domains (columns chunk_first ..): fills the
// same band terms as launch_lw_groups.
cudaError_t launch_lw_gsplit(const Tables &T, const LwArgs &a, cudaStream_t stream);
size_t lw_optics_floats(int nlay, int ncol);
// day-column compaction (writes the night columns), then the column kernel over
// the day columns; both need a.nday and a.daylist (1 + ncol ints)
cudaError_t launch_sw_daylist(const SwArgs &a, cudaStream_t stream);
size_t sw_record_floats(int nk, int chunk);
cudaError_t launch_sw_columns(const Tables &T, const SwArgs &a, cudaStream_t stream);

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

// C-ABI of librrtmg_b200.so: context creation (table upload), the LW and SW
// radiation calls, and error reporting.  See include/rrtmg_b200.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/rrtmg_b200.h"
#include "../../include/rrtmg_prologue.h"
#include "rrtmg_device.cuh"
#include "rrtmg_kernels.h"
#include "kiss_jump_host.h"

using namespace rrtmg;

namespace {

struct Entry {
  uint32_t dtype, ndim, shape[4];
  uint64_t offset, nbytes;
};

std::mutex g_create_mutex;
std::string g_create_error;

}  // namespace

struct rrtmg_ctx {
  int device = 0;
  std::vector<unsigned char> host_blob;
  std::map<std::string, Entry> entries;
  void *dev_blob = nullptr;
  Tables tables{};
  std::mutex mutex;
  std::string last_error;
  // KISS jump tables keyed by (nlay, nsub, skip); never freed before destroy
  std::map<std::tuple<int, int, int>, KissJump *> jumps;
  // stream-ordered per-call scratch; keeps its memory between calls
  cudaMemPool_t pool = nullptr;
  // launch schedule (rrtmg_set_schedule)
  int lw_chunk = kLwChunkColumns, sw_chunk = kSwChunkColumns, sw_split_max = kSwSplitMaxColumns;
  int lw_split_max = kLwSplitMaxColumns;
  // optional per-phase timing: a ring of calls per side (0 LW, 1 SW); each
  // call records events between its phases (McICA, then per chunk the optics
  // launches and the sweep launch), marks[side][slot] of them
  bool timing = false;
  std::vector<std::vector<cudaEvent_t>> events[2];
  std::vector<int> marks[2];
  int timing_next[2] = {0, 0};
  int timing_count[2] = {0, 0};
  // per-column status (rrtmg_last_column_errors): one array per side, grown
  // as needed; retired arrays stay allocated until destroy because queued
  // status launches may still write them
  bool colstatus = false;
  uint32_t *status_buf[2] = {nullptr, nullptr};
  size_t status_cap[2] = {0, 0};
  int status_ncol[2] = {-1, -1};
  std::vector<uint32_t *> retired_status;
  // radiation prologue: SVML sin/cos constants from the blob, and the CAM
  // ozone climatology (plev, lat, then the (12, latsiz, levsiz) table in one
  // allocation); replaced climatologies stay allocated until destroy because
  // queued launches may still read them
  SvmlConsts svml{};
  bool have_svml = false;
  float *ozone = nullptr;
  int oz_levsiz = 0, oz_latsiz = 0;
  std::vector<float *> retired_ozone;
};

namespace {
constexpr int kTimingSlots = 256;

// Claims the next timing slot of `side`, or -1 when timing is off.
int timing_slot(rrtmg_ctx *ctx, int side) {
  std::lock_guard<std::mutex> lk(ctx->mutex);
  if (!ctx->timing) return -1;
  const int slot = ctx->timing_next[side];
  ctx->timing_next[side] = (slot + 1) % kTimingSlots;
  if (ctx->timing_count[side] < kTimingSlots) ++ctx->timing_count[side];
  ctx->marks[side][slot] = 0;
  return slot;
}

// Records the slot's next event on `stream` (events are created on first use).
void timing_mark(rrtmg_ctx *ctx, int side, int slot, cudaStream_t stream) {
  if (slot < 0) return;
  cudaEvent_t ev = nullptr;
  {
    std::lock_guard<std::mutex> lk(ctx->mutex);
    std::vector<cudaEvent_t> &v = ctx->events[side][slot];
    const int m = ctx->marks[side][slot];
    if (m == static_cast<int>(v.size())) {
      cudaEvent_t fresh = nullptr;
      if (cudaEventCreate(&fresh) != cudaSuccess) {
        cudaGetLastError();
        return;
      }
      v.push_back(fresh);
    }
    ev = v[m];
    ctx->marks[side][slot] = m + 1;
  }
  cudaEventRecord(ev, stream);
}
}  // namespace

namespace {

rrtmg_status fail(rrtmg_ctx *ctx, rrtmg_status st, const std::string &msg) {
  if (ctx) {
    std::lock_guard<std::mutex> lk(ctx->mutex);
    ctx->last_error = msg;
  } else {
    std::lock_guard<std::mutex> lk(g_create_mutex);
    g_create_error = msg;
  }
  return st;
}

}  // namespace

rrtmg_status rrtmg::create_error(rrtmg_status status, const std::string &message) {
  return fail(nullptr, status, message);
}

namespace {

rrtmg_status cuda_fail(rrtmg_ctx *ctx, cudaError_t e, const char *what) {
  return fail(ctx, RRTMG_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// nbytes equals the element size of dtype (0 f32, 1 i32, 2 f64, 3 u64) times
// the product of the first ndim extents (ndim <= 4).
bool entry_size_matches(uint32_t dtype, uint32_t ndim, const uint32_t *shape, uint64_t nbytes) {
  static const uint64_t kSize[4] = {4, 4, 8, 8};
  if (dtype > 3 || ndim > 4) return false;
  uint64_t count = 1;
  for (uint32_t d = 0; d < ndim; ++d) {
    if (shape[d] != 0 && count > UINT64_MAX / 8 / shape[d]) return false;
    count *= shape[d];
  }
  return count * kSize[dtype] == nbytes;
}

bool parse_blob(rrtmg_ctx *ctx, std::string &err) {
  const auto &raw = ctx->host_blob;
  if (raw.size() < 16 || std::memcmp(raw.data(), "RRTMGB2\0", 8) != 0) {
    err = "not an RRTMG table blob";
    return false;
  }
  uint32_t version, count;
  std::memcpy(&version, raw.data() + 8, 4);
  std::memcpy(&count, raw.data() + 12, 4);
  if (version != 1) {
    err = "unsupported table blob version";
    return false;
  }
  size_t pos = 16;
  for (uint32_t i = 0; i < count; ++i, pos += 88) {
    if (pos + 88 > raw.size()) {
      err = "truncated table blob header";
      return false;
    }
    char name[49] = {0};
    std::memcpy(name, raw.data() + pos, 48);
    Entry e;
    std::memcpy(&e.dtype, raw.data() + pos + 48, 4);
    std::memcpy(&e.ndim, raw.data() + pos + 52, 4);
    std::memcpy(e.shape, raw.data() + pos + 56, 16);
    std::memcpy(&e.offset, raw.data() + pos + 72, 8);
    std::memcpy(&e.nbytes, raw.data() + pos + 80, 8);
    if (e.offset > raw.size() || e.nbytes > raw.size() - e.offset) {
      err = std::string("table entry out of range: ") + name;
      return false;
    }
    if (!entry_size_matches(e.dtype, e.ndim, e.shape, e.nbytes)) {
      err = std::string("table entry size does not match its shape and type: ") + name;
      return false;
    }
    ctx->entries[name] = e;
  }
  return true;
}

template <typename T>
const T *dev_ptr(rrtmg_ctx *ctx, const std::string &name, int *count = nullptr) {
  auto it = ctx->entries.find(name);
  if (it == ctx->entries.end()) {
    if (count) *count = 0;
    return nullptr;
  }
  if (count) *count = static_cast<int>(it->second.nbytes / sizeof(T));
  return reinterpret_cast<const T *>(static_cast<const unsigned char *>(ctx->dev_blob) + it->second.offset);
}

template <typename T>
const T *host_ptr(rrtmg_ctx *ctx, const std::string &name, int *count = nullptr) {
  auto it = ctx->entries.find(name);
  if (it == ctx->entries.end()) {
    if (count) *count = 0;
    return nullptr;
  }
  if (count) *count = static_cast<int>(it->second.nbytes / sizeof(T));
  return reinterpret_cast<const T *>(ctx->host_blob.data() + it->second.offset);
}

// Ozone climatology work profile (module_ra_rrtmg_common.py:343-372), binary32.
void o3_work_profile(rrtmg_ctx *ctx, float *o3wrk, float *ppwrkh) {
  const float *o3sum = host_ptr<float>(ctx, "o3sum");
  const float *ppsum = host_ptr<float>(ctx, "ppsum");
  const float *o3win = host_ptr<float>(ctx, "o3win");
  const float *ppwin = host_ptr<float>(ctx, "ppwin");
  volatile float t;
  o3wrk[0] = 0.5f * (o3sum[0] + o3win[0]);
  for (int i = 0; i < 30; ++i) {
    t = (o3win[i + 1] - o3win[i]) / (ppwin[i + 1] - ppwin[i]);
    const float slope = t;
    t = slope * (ppsum[i + 1] - ppwin[i]);
    const float prod = t;
    const float interp = o3win[i] + prod;
    o3wrk[i + 1] = 0.5f * (interp + o3sum[i + 1]);
  }
  ppwrkh[0] = 1100.0f;
  for (int i = 0; i < 30; ++i) ppwrkh[i + 1] = 0.5f * (ppsum[i + 1] + ppsum[i]);
  ppwrkh[31] = 0.0f;
}

bool fill_tables(rrtmg_ctx *ctx, std::string &err) {
  Tables &T = ctx->tables;
  static const int lw_ngc[16] = {10, 12, 16, 14, 16, 8, 12, 8, 12, 6, 8, 8, 4, 2, 2, 2};
  static const int sw_ngc[14] = {6, 12, 8, 8, 10, 10, 2, 10, 8, 6, 6, 8, 6, 12};
  for (int b = 0; b < kLwBands; ++b) {
    const std::string p = "lw" + std::to_string(b + 1) + ".";
    LwBand &B = T.lw[b];
    int n = 0;
    B.ka = dev_ptr<float>(ctx, p + "ka", &n);
    B.ka_rows = n / lw_ngc[b];
    B.kb = dev_ptr<float>(ctx, p + "kb", &n);
    B.kb_rows = B.kb ? n / lw_ngc[b] : 0;
    B.fracrefa = dev_ptr<float>(ctx, p + "fracrefa");
    B.fracrefb = dev_ptr<float>(ctx, p + "fracrefb");
    B.selfref = dev_ptr<float>(ctx, p + "selfref");
    B.forref = dev_ptr<float>(ctx, p + "forref");
    B.ka_mn2 = dev_ptr<float>(ctx, p + "ka_mn2");
    B.kb_mn2 = dev_ptr<float>(ctx, p + "kb_mn2");
    B.ka_mn2o = dev_ptr<float>(ctx, p + "ka_mn2o");
    B.kb_mn2o = dev_ptr<float>(ctx, p + "kb_mn2o");
    B.ka_mo3 = dev_ptr<float>(ctx, p + "ka_mo3");
    B.kb_mo3 = dev_ptr<float>(ctx, p + "kb_mo3");
    B.ka_mco2 = dev_ptr<float>(ctx, p + "ka_mco2");
    B.kb_mco2 = dev_ptr<float>(ctx, p + "kb_mco2");
    B.ka_mco = dev_ptr<float>(ctx, p + "ka_mco");
    B.ka_mo2 = dev_ptr<float>(ctx, p + "ka_mo2");
    B.kb_mo2 = dev_ptr<float>(ctx, p + "kb_mo2");
    B.ccl4 = dev_ptr<float>(ctx, p + "ccl4");
    B.cfc11adj = dev_ptr<float>(ctx, p + "cfc11adj");
    B.cfc12 = dev_ptr<float>(ctx, p + "cfc12");
    B.cfc22adj = dev_ptr<float>(ctx, p + "cfc22adj");
    if (!B.ka || !B.fracrefa || !B.selfref || !B.forref) {
      err = "table blob lacks longwave band " + std::to_string(b + 1);
      return false;
    }
  }
  for (int b = 0; b < kSwBands; ++b) {
    const std::string p = "sw" + std::to_string(b + 16) + ".";
    SwBand &B = T.sw[b];
    int n = 0;
    B.ka = dev_ptr<float>(ctx, p + "ka");
    B.kb = dev_ptr<float>(ctx, p + "kb");
    B.selfref = dev_ptr<float>(ctx, p + "selfref");
    B.forref = dev_ptr<float>(ctx, p + "forref", &n);
    B.forref_rows = B.forref ? n / sw_ngc[b] : 0;
    B.sfluxref = dev_ptr<float>(ctx, p + "sfluxref", &n);
    B.sflux_cols = B.sfluxref ? n / sw_ngc[b] : 0;
    B.rayla = dev_ptr<float>(ctx, p + "rayla");
    B.raylb = dev_ptr<float>(ctx, p + "raylb");
    B.absch4 = dev_ptr<float>(ctx, p + "absch4");
    B.abso3a = dev_ptr<float>(ctx, p + "abso3a");
    B.abso3b = dev_ptr<float>(ctx, p + "abso3b");
    B.absh2o = dev_ptr<float>(ctx, p + "absh2o");
    B.absco2 = dev_ptr<float>(ctx, p + "absco2");
    const float *rayl = host_ptr<float>(ctx, p + "rayl", &n);
    if (rayl && n == 1) {
      B.rayl = rayl[0];
      B.rayl_g = nullptr;
    } else {
      B.rayl = 0.0f;
      B.rayl_g = dev_ptr<float>(ctx, p + "rayl");
    }
    auto scalar = [&](const char *f) {
      const float *v = host_ptr<float>(ctx, p + f);
      return v ? v[0] : 0.0f;
    };
    B.strrat = scalar("strrat");
    B.strrat1 = scalar("strrat1");
    B.givfac = scalar("givfac");
    B.scalekur = scalar("scalekur");
    const int32_t *lr = host_ptr<int32_t>(ctx, p + "layreffr");
    B.layreffr = lr ? lr[0] : 0;
    if (!B.sfluxref) {
      err = "table blob lacks shortwave band " + std::to_string(b + 16);
      return false;
    }
  }
  T.lw_preflog = dev_ptr<float>(ctx, "lw.preflog");
  T.lw_tref = dev_ptr<float>(ctx, "lw.tref");
  T.chi_mls = dev_ptr<float>(ctx, "lw.chi_mls");
  T.totplnk = dev_ptr<float>(ctx, "lw.totplnk");
  T.absice3 = dev_ptr<float>(ctx, "lw.absice3");
  T.absliq1 = dev_ptr<float>(ctx, "lw.absliq1");
  int n = 0;
  T.lw_pade_tau = dev_ptr<float>(ctx, "lw.pade_tau_tbl", &n);
  T.lw_ntbl = n - 1;
  T.lw_pade_exp = dev_ptr<float>(ctx, "lw.pade_exp_tbl");
  T.lw_pade_tfn = dev_ptr<float>(ctx, "lw.pade_tfn_tbl");
  const float *bp = host_ptr<float>(ctx, "lw.pade_bpade");
  T.lw_bpade = bp ? bp[0] : 0.0f;
  T.sw_preflog = dev_ptr<float>(ctx, "sw.preflog");
  T.sw_tref = dev_ptr<float>(ctx, "sw.tref");
  T.extliq1 = dev_ptr<float>(ctx, "sw.extliq1");
  T.ssaliq1 = dev_ptr<float>(ctx, "sw.ssaliq1");
  T.asyliq1 = dev_ptr<float>(ctx, "sw.asyliq1");
  T.extice3 = dev_ptr<float>(ctx, "sw.extice3");
  T.ssaice3 = dev_ptr<float>(ctx, "sw.ssaice3");
  T.asyice3 = dev_ptr<float>(ctx, "sw.asyice3");
  T.fdlice3 = dev_ptr<float>(ctx, "sw.fdlice3");
  T.sw_pade_exp = dev_ptr<float>(ctx, "sw.pade_exp_tbl", &n);
  T.sw_ntbl = n - 1;
  const float *sbp = host_ptr<float>(ctx, "sw.pade_bpade");
  T.sw_bpade = sbp ? sbp[0] : 0.0f;
  T.retab = dev_ptr<float>(ctx, "retab");
  T.pprof = dev_ptr<float>(ctx, "lw_buffer_pprof", &n);
  T.nprof = n;
  T.tprof = dev_ptr<float>(ctx, "lw_buffer_tprof");
  o3_work_profile(ctx, T.o3wrk, T.ppwrkh);
  T.logf_tab = dev_ptr<double>(ctx, "glibc.logf_invc_logc");
  const double *lp = host_ptr<double>(ctx, "glibc.logf_ln2_poly");
  T.expf_tab = dev_ptr<unsigned long long>(ctx, "glibc.expf_tab");
  const double *ep = host_ptr<double>(ctx, "glibc.expf_invln2n_poly");
  if (!T.lw_preflog || !T.chi_mls || !T.totplnk || !T.absice3 || !T.absliq1 || !T.lw_pade_tau ||
      !T.sw_preflog || !T.extliq1 || !T.extice3 || !T.sw_pade_exp || !T.retab || !T.pprof || !T.tprof ||
      !T.logf_tab || !lp || !T.expf_tab || !ep || !host_ptr<float>(ctx, "o3sum")) {
    err = "table blob is missing required tables";
    return false;
  }
  T.logf_ln2 = lp[0];
  T.logf_a0 = lp[1];
  T.logf_a1 = lp[2];
  T.logf_a2 = lp[3];
  T.expf_invln2n = ep[0];
  T.expf_c0 = ep[1];
  T.expf_c1 = ep[2];
  T.expf_c2 = ep[3];
  int ns = 0, nc = 0;
  const float *ss = host_ptr<float>(ctx, "svml.sinf", &ns);
  const float *sc = host_ptr<float>(ctx, "svml.cosf", &nc);
  if (ss && sc && ns == 12 && nc == 14) {
    std::memcpy(ctx->svml.s, ss, sizeof(ctx->svml.s));
    std::memcpy(ctx->svml.c, sc, sizeof(ctx->svml.c));
    ctx->have_svml = true;
  }
  return true;
}

rrtmg_status get_jumps(rrtmg_ctx *ctx, int nlay, int nsub, int skip, const KissJump **out) {
  std::lock_guard<std::mutex> lk(ctx->mutex);
  auto key = std::make_tuple(nlay, nsub, skip);
  auto it = ctx->jumps.find(key);
  if (it != ctx->jumps.end()) {
    *out = it->second;
    return RRTMG_OK;
  }
  // offsets skip + g * nlay
  std::vector<KissJump> host(nsub);
  kiss_jumps(static_cast<uint64_t>(skip), nlay, nsub, host.data());
  KissJump *dev = nullptr;
  cudaError_t e = cudaMalloc(&dev, sizeof(KissJump) * nsub);
  if (e != cudaSuccess) {
    ctx->last_error = std::string("cudaMalloc(jump table): ") + cudaGetErrorString(e);
    return RRTMG_CUDA;
  }
  e = cudaMemcpy(dev, host.data(), sizeof(KissJump) * nsub, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(dev);
    ctx->last_error = std::string("cudaMemcpy(jump table): ") + cudaGetErrorString(e);
    return RRTMG_CUDA;
  }
  ctx->jumps[key] = dev;
  *out = dev;
  return RRTMG_OK;
}

rrtmg_status finish_create(rrtmg_ctx *ctx, int device, rrtmg_ctx **out) {
  std::string err;
  if (!parse_blob(ctx, err)) {
    delete ctx;
    return fail(nullptr, RRTMG_BAD_ARG, err);
  }
  DeviceGuard guard(device);
  cudaError_t e = guard.status();
  if (e != cudaSuccess) {
    delete ctx;
    return cuda_fail(nullptr, e, "cudaSetDevice");
  }
  ctx->device = device;
  e = cudaMalloc(&ctx->dev_blob, ctx->host_blob.size());
  if (e != cudaSuccess) {
    delete ctx;
    return cuda_fail(nullptr, e, "cudaMalloc(tables)");
  }
  e = cudaMemcpy(ctx->dev_blob, ctx->host_blob.data(), ctx->host_blob.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(ctx->dev_blob);
    delete ctx;
    return cuda_fail(nullptr, e, "cudaMemcpy(tables)");
  }
  if (!fill_tables(ctx, err)) {
    cudaFree(ctx->dev_blob);
    delete ctx;
    return fail(nullptr, RRTMG_BAD_ARG, err);
  }
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  e = cudaMemPoolCreate(&ctx->pool, &props);
  if (e == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (e != cudaSuccess) {
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    cudaFree(ctx->dev_blob);
    delete ctx;
    return cuda_fail(nullptr, e, "cudaMemPoolCreate(scratch pool)");
  }
  *out = ctx;
  return RRTMG_OK;
}

void cloud_flags(const rrtmg_config *c, int *inflg, int *iceflg, int *liqflg) {
  *inflg = 2;
  *iceflg = 3;
  *liqflg = 1;
  if (c->icloud != 0) {
    if (c->has_reqc) *inflg = 3;
    if (c->has_reqi) { *inflg = 4; *iceflg = 4; }
    if (c->has_reqs) { *inflg = 5; *iceflg = 5; }
    if (!c->has_reqs && c->has_reqi && c->has_reqc) { *inflg = 5; *iceflg = 5; }
  }
}

rrtmg_status check_config(rrtmg_ctx *ctx, const rrtmg_config *cfg) {
  if (!ctx || !cfg) return fail(ctx, RRTMG_BAD_ARG, "null context or config");
  if (cfg->nx <= 0 || cfg->ny <= 0) return fail(ctx, RRTMG_BAD_ARG, "nx and ny must be positive");
  if (cfg->nk < 4) return fail(ctx, RRTMG_BAD_ARG, "nk must be at least 4 (McICA seeds read four layers)");
  if (static_cast<long long>(cfg->nx) * cfg->ny > (1ll << 30))
    return fail(ctx, RRTMG_BAD_ARG, "too many columns in one call");
  if (cfg->fp64_steps != 0 && cfg->fp64_steps != 1) return fail(ctx, RRTMG_BAD_ARG, "fp64_steps must be 0 or 1");
  return RRTMG_OK;
}

ColumnInputs common_inputs(const float *p3d, const float *p8w, const float *pi3d, const float *t3d, const float *t8w,
                           const float *tsk, const float *qv, const float *qc, const float *qi, const float *qs,
                           const float *cldfra, const float *o3, const float *xland, const float *xice,
                           const float *snow, const float *rec, const float *rei, const float *res) {
  ColumnInputs in{};
  in.p3d = p3d; in.p8w = p8w; in.pi3d = pi3d; in.t3d = t3d; in.t8w = t8w; in.tsk = tsk;
  in.qv = qv; in.qc = qc; in.qi = qi; in.qs = qs; in.cldfra = cldfra; in.o3 = o3;
  in.xland = xland; in.xice = xice; in.snow = snow;
  in.re_cloud = rec; in.re_ice = rei; in.re_snow = res;
  return in;
}

bool any_null(std::initializer_list<const void *> ptrs) {
  for (const void *p : ptrs)
    if (!p) return true;
  return false;
}

}  // namespace

extern "C" {

int rrtmg_lw_nlayers(double p_top, int nk) {
  const double layers_above = p_top * 0.01 / 4.0;
  return (nk + 1) + static_cast<int>(layers_above + 0.5) - 1;
}

rrtmg_status rrtmg_create_from_memory(const void *blob, size_t nbytes, int device, rrtmg_ctx **out) {
  if (!blob || !out || nbytes < 16) return fail(nullptr, RRTMG_BAD_ARG, "null blob or output pointer");
  auto *ctx = new rrtmg_ctx();
  ctx->host_blob.assign(static_cast<const unsigned char *>(blob), static_cast<const unsigned char *>(blob) + nbytes);
  return finish_create(ctx, device, out);
}

rrtmg_status rrtmg_create(const char *path, int device, rrtmg_ctx **out) {
  if (!path || !out) return fail(nullptr, RRTMG_BAD_ARG, "null path or output pointer");
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(nullptr, RRTMG_BAD_ARG, std::string("cannot open table blob ") + path);
  auto *ctx = new rrtmg_ctx();
  ctx->host_blob.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return finish_create(ctx, device, out);
}

void rrtmg_destroy(rrtmg_ctx *ctx) {
  if (!ctx) return;
  DeviceGuard guard(ctx->device);
  cudaDeviceSynchronize();
  for (auto &kv : ctx->jumps) cudaFree(kv.second);
  cudaFree(ctx->ozone);
  for (float *p : ctx->retired_ozone) cudaFree(p);
  for (uint32_t *p : ctx->status_buf) cudaFree(p);
  for (uint32_t *p : ctx->retired_status) cudaFree(p);
  cudaFree(ctx->dev_blob);
  if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
  for (auto &side : ctx->events)
    for (auto &slot : side)
      for (cudaEvent_t ev : slot) cudaEventDestroy(ev);
  delete ctx;
}

const char *rrtmg_last_error(const rrtmg_ctx *ctx) {
  if (!ctx) return g_create_error.c_str();
  return ctx->last_error.c_str();
}

const char *rrtmg_status_string(rrtmg_status s) {
  switch (s) {
    case RRTMG_OK: return "ok";
    case RRTMG_BAD_ARG: return "bad argument";
    case RRTMG_UNSUPPORTED_OPTION: return "unsupported option";
    case RRTMG_CUDA: return "CUDA error";
    case RRTMG_TIMEOUT: return "timeout";
  }
  return "unknown status";
}

// When column status is enabled: the status array of `side` for ncol
// columns (grown with cudaMalloc when needed), else null.
static uint32_t *status_target(rrtmg_ctx *ctx, int side, int ncol, cudaError_t *err) {
  *err = cudaSuccess;
  std::lock_guard<std::mutex> lk(ctx->mutex);
  if (!ctx->colstatus) return nullptr;
  if (ctx->status_cap[side] < static_cast<size_t>(ncol)) {
    uint32_t *fresh = nullptr;
    *err = cudaMalloc(&fresh, sizeof(uint32_t) * static_cast<size_t>(ncol));
    if (*err != cudaSuccess) return nullptr;
    if (ctx->status_buf[side]) ctx->retired_status.push_back(ctx->status_buf[side]);
    ctx->status_buf[side] = fresh;
    ctx->status_cap[side] = static_cast<size_t>(ncol);
  }
  ctx->status_ncol[side] = ncol;
  return ctx->status_buf[side];
}

// Per-call scratch: carved in order from a caller's workspace (each piece on
// a 256-byte boundary), or taken from the context's stream-ordered pool and
// returned to it by release().
extern "C++" {
struct CallScratch {
  rrtmg_ctx *ctx;
  cudaStream_t stream;
  unsigned char *ws;
  size_t ws_bytes, used = 0;
  std::vector<void *> pooled;
  CallScratch(rrtmg_ctx *c, cudaStream_t s, void *w, size_t wb)
      : ctx(c), stream(s), ws(static_cast<unsigned char *>(w)), ws_bytes(wb) {}
  static size_t aligned(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }
  template <typename T>
  cudaError_t take(T **p, size_t bytes) {
    if (ws) {
      if (aligned(used) + bytes > ws_bytes) return cudaErrorMemoryAllocation;
      *p = reinterpret_cast<T *>(ws + aligned(used));
      used = aligned(used) + bytes;
      return cudaSuccess;
    }
    void *q = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&q, bytes, ctx->pool, stream);
    if (e == cudaSuccess) {
      pooled.push_back(q);
      *p = static_cast<T *>(q);
    }
    return e;
  }
  cudaError_t release() {
    cudaError_t first = cudaSuccess;
    for (auto it = pooled.rbegin(); it != pooled.rend(); ++it) {
      cudaError_t e = cudaFreeAsync(*it, stream);
      if (first == cudaSuccess) first = e;
    }
    pooled.clear();
    return first;
  }
};
}  // extern "C++"

// Scratch pieces of one call, in the order the calls take them.
static size_t lw_chunk_columns(rrtmg_ctx *ctx, int ncol) {
  std::lock_guard<std::mutex> lk(ctx->mutex);
  return static_cast<size_t>(ncol < ctx->lw_chunk ? ncol : ctx->lw_chunk);
}
static size_t sw_chunk_columns(rrtmg_ctx *ctx, int ncol) {
  std::lock_guard<std::mutex> lk(ctx->mutex);
  return static_cast<size_t>(ncol < ctx->sw_chunk ? ncol : ctx->sw_chunk);
}
static size_t lw_workspace_bytes(rrtmg_ctx *ctx, const rrtmg_config *cfg) {
  const int nlay = rrtmg_lw_nlayers(cfg->p_top, cfg->nk);
  const size_t ncol = static_cast<size_t>(cfg->nx) * cfg->ny;
  const size_t chunk = lw_chunk_columns(ctx, static_cast<int>(ncol));
  return CallScratch::aligned(static_cast<size_t>(nlay) * kLwMaskWords * ncol * sizeof(uint32_t)) +
         CallScratch::aligned(lw_scratch_floats(nlay, static_cast<int>(chunk)) * sizeof(float));
}
static size_t sw_workspace_bytes(rrtmg_ctx *ctx, const rrtmg_config *cfg) {
  const int nlay = cfg->nk + 1;
  const size_t ncol = static_cast<size_t>(cfg->nx) * cfg->ny;
  const size_t chunk = sw_chunk_columns(ctx, static_cast<int>(ncol));
  return CallScratch::aligned(static_cast<size_t>(nlay) * kSwMaskWords * ncol * sizeof(uint32_t)) +
         CallScratch::aligned((ncol + 1) * sizeof(int)) +
         CallScratch::aligned(sw_record_floats(cfg->nk, static_cast<int>(chunk)) * sizeof(float));
}

// live: null, or a device count; columns at or past it are skipped.  ws: null
// (scratch from the context's pool), or a caller's workspace of ws_bytes.
static rrtmg_status lwrad_impl(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_lw_in *in, rrtmg_lw_out *out,
                               void *stream_ptr, const int *live, void *ws = nullptr, size_t ws_bytes = 0) {
  rrtmg_status st = check_config(ctx, cfg);
  if (st != RRTMG_OK) return st;
  if (!in || !out) return fail(ctx, RRTMG_BAD_ARG, "null input or output block");
  if (any_null({in->p3d, in->p8w, in->pi3d, in->t3d, in->t8w, in->tsk, in->qv3d, in->qc3d, in->qi3d, in->qs3d,
                in->cldfra3d, in->o33d, in->emiss, in->xland, in->xice, in->snow, in->re_cloud, in->re_ice,
                in->re_snow}))
    return fail(ctx, RRTMG_BAD_ARG, "a required LW input pointer is null");
  if (any_null({out->rthratenlw, out->rthratenlwc, out->lwupt, out->lwuptc, out->lwuptcln, out->lwdnt, out->lwdntc,
                out->lwdntcln, out->lwupb, out->lwupbc, out->lwupbcln, out->lwdnb, out->lwdnbc, out->lwdnbcln,
                out->glw, out->olr, out->lwcf}))
    return fail(ctx, RRTMG_BAD_ARG, "a required LW output pointer is null");
  const int nlay = rrtmg_lw_nlayers(cfg->p_top, cfg->nk);
  if (nlay > kMaxLay || nlay - cfg->nk > kMaxBuf || nlay < cfg->nk)
    return fail(ctx, RRTMG_BAD_ARG, "too many layers (nk and p_top exceed the kernel's layer capacity)");
  int inflg, iceflg, liqflg;
  cloud_flags(cfg, &inflg, &iceflg, &liqflg);
  const int icld = cfg->cldovrlp;
  if (icld >= 1 && (inflg < 2 || iceflg < 3 || liqflg != 1))
    return fail(ctx, RRTMG_UNSUPPORTED_OPTION, "cloud optics option not supported by cldprmc_lw");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  DeviceGuard guard(ctx->device);
  cudaError_t e = guard.status();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  const int ncol = cfg->nx * cfg->ny;
  const KissJump *jumps = nullptr;
  st = get_jumps(ctx, nlay, kLwGpts, 150, &jumps);
  if (st != RRTMG_OK) return st;
  uint32_t *mask = nullptr;
  float *scratch = nullptr;
  const size_t mask_bytes = static_cast<size_t>(nlay) * kLwMaskWords * ncol * sizeof(uint32_t);
  const int chunk = static_cast<int>(lw_chunk_columns(ctx, ncol));
  if (ws && ws_bytes < lw_workspace_bytes(ctx, cfg))
    return fail(ctx, RRTMG_BAD_ARG, "workspace smaller than rrtmg_lw_workspace_bytes");
  CallScratch sc(ctx, stream, ws, ws_bytes);
  e = sc.take(&mask, mask_bytes);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "scratch (mcica mask)");
  e = sc.take(&scratch, lw_scratch_floats(nlay, chunk) * sizeof(float));
  if (e != cudaSuccess) {
    sc.release();
    return cuda_fail(ctx, e, "scratch (lw layer records)");
  }

  const int tslot = timing_slot(ctx, 0);
  timing_mark(ctx, 0, tslot, stream);
  McicaArgs m{};
  m.ncol = ncol; m.ny = cfg->ny; m.nk = cfg->nk; m.nlay = nlay; m.nsub = kLwGpts; m.words = kLwMaskWords;
  m.enabled = icld >= 1;
  m.live = live;
  m.p3d = in->p3d; m.cldfra = in->cldfra3d; m.jumps = jumps; m.mask = mask;
  e = launch_mcica(m, stream);
  timing_mark(ctx, 0, tslot, stream);
  if (e != cudaSuccess) {
    sc.release();
    return cuda_fail(ctx, e, "mcica kernel launch");
  }
  LwArgs a{};
  a.live = live;
  a.fp64_from = cfg->fp64_steps ? fp64_first_layer(cfg->nk) : kMaxLay + 1;
  a.nx = cfg->nx; a.ny = cfg->ny; a.nk = cfg->nk; a.nlay = nlay; a.ncol = ncol;
  a.co2 = cfg->co2vmr; a.n2o = cfg->n2ovmr; a.ch4 = cfg->ch4vmr; a.cfc11 = cfg->cfc11vmr; a.cfc12 = cfg->cfc12vmr;
  a.has_reqc = cfg->has_reqc; a.has_reqi = cfg->has_reqi; a.has_reqs = cfg->has_reqs; a.icloud = cfg->icloud;
  a.icld = icld; a.inflg = inflg; a.iceflg = iceflg; a.liqflg = liqflg;
  a.in = common_inputs(in->p3d, in->p8w, in->pi3d, in->t3d, in->t8w, in->tsk, in->qv3d, in->qc3d, in->qi3d,
                       in->qs3d, in->cldfra3d, in->o33d, in->xland, in->xice, in->snow, in->re_cloud, in->re_ice,
                       in->re_snow);
  a.in.emiss = in->emiss;
  a.mask = mask;
  a.rthraten = out->rthratenlw; a.rthratenc = out->rthratenlwc;
  a.upt = out->lwupt; a.uptc = out->lwuptc; a.dnt = out->lwdnt; a.dntc = out->lwdntc;
  a.upb = out->lwupb; a.upbc = out->lwupbc; a.dnb = out->lwdnb; a.dnbc = out->lwdnbc;
  a.glw = out->glw; a.olr = out->olr; a.lwcf = out->lwcf;
  a.zero2[0] = out->lwuptcln; a.zero2[1] = out->lwdntcln; a.zero2[2] = out->lwupbcln; a.zero2[3] = out->lwdnbcln;
  a.scratch = scratch;
  a.chunk_capacity = chunk;
  // chunks of columns, each through its optics and then its sweep, reusing the scratch
  for (int first = 0; first < ncol && e == cudaSuccess; first += chunk) {
    a.chunk_first = first;
    a.chunk_count = ncol - first < chunk ? ncol - first : chunk;
    e = launch_lw_chunk_optics(ctx->tables, a, stream);
    timing_mark(ctx, 0, tslot, stream);
    if (e == cudaSuccess) e = launch_lw_chunk_sweep(ctx->tables, a, stream);
    timing_mark(ctx, 0, tslot, stream);
  }
  if (e == cudaSuccess && !live) {
    cudaError_t es = cudaSuccess;
    uint32_t *status = status_target(ctx, 0, ncol, &es);
    if (es != cudaSuccess) e = es;
    if (status) {
      StatusArgs sa{};
      sa.ncol = ncol; sa.nx = cfg->nx; sa.ny = cfg->ny; sa.nk = cfg->nk; sa.side = 0;
      sa.has_req = cfg->has_reqc || cfg->has_reqi || cfg->has_reqs;
      sa.in = a.in;
      sa.rthraten = out->rthratenlw; sa.rthratenc = out->rthratenlwc;
      const float *o2[8] = {out->lwupt, out->lwuptc, out->lwdnt, out->lwdntc, out->lwupb, out->lwupbc,
                            out->lwdnb, out->lwdnbc};
      for (int q = 0; q < 8; ++q) sa.out2d[q] = o2[q];
      sa.n2d = 8;
      sa.status = status;
      e = launch_column_status(sa, stream);
    }
  }
  cudaError_t ef = sc.release();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "lw kernel launch");
  if (ef != cudaSuccess) return cuda_fail(ctx, ef, "cudaFreeAsync(lw scratch)");
  return RRTMG_OK;
}

static rrtmg_status swrad_impl(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_sw_in *in, rrtmg_sw_out *out,
                               void *stream_ptr, const int *live, void *ws = nullptr, size_t ws_bytes = 0) {
  rrtmg_status st = check_config(ctx, cfg);
  if (st != RRTMG_OK) return st;
  if (!in || !out) return fail(ctx, RRTMG_BAD_ARG, "null input or output block");
  if (any_null({in->p3d, in->p8w, in->pi3d, in->t3d, in->t8w, in->tsk, in->qv3d, in->qc3d, in->qi3d, in->qs3d,
                in->cldfra3d, in->o33d, in->albedo, in->coszr, in->xland, in->xice, in->snow, in->re_cloud,
                in->re_ice, in->re_snow}))
    return fail(ctx, RRTMG_BAD_ARG, "a required SW input pointer is null");
  if (any_null({out->rthratensw, out->rthratenswc, out->swupt, out->swuptc, out->swuptcln, out->swdnt, out->swdntc,
                out->swdntcln, out->swupb, out->swupbc, out->swupbcln, out->swdnb, out->swdnbc, out->swdnbcln,
                out->swcf, out->gsw, out->swddir, out->swddni, out->swddif, out->swdownc, out->swddnic, out->swddirc,
                out->coszr}))
    return fail(ctx, RRTMG_BAD_ARG, "a required SW output pointer is null");
  const int nlay = cfg->nk + 1;
  if (nlay > kMaxLay) return fail(ctx, RRTMG_BAD_ARG, "too many layers for the kernel's layer capacity");
  int inflg, iceflg, liqflg;
  cloud_flags(cfg, &inflg, &iceflg, &liqflg);
  const int icld = cfg->icloud == 0 ? 0 : cfg->cldovrlp;
  if (icld >= 1 && (inflg < 2 || iceflg < 3 || liqflg != 1))
    return fail(ctx, RRTMG_UNSUPPORTED_OPTION, "cloud optics option not supported by cldprmc_sw");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  DeviceGuard guard(ctx->device);
  cudaError_t e = guard.status();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  const int ncol = cfg->nx * cfg->ny;
  const KissJump *jumps = nullptr;
  st = get_jumps(ctx, nlay, kSwGpts, 1, &jumps);
  if (st != RRTMG_OK) return st;
  uint32_t *mask = nullptr;
  int *daylist = nullptr;
  const size_t mask_bytes = static_cast<size_t>(nlay) * kSwMaskWords * ncol * sizeof(uint32_t);
  if (ws && ws_bytes < sw_workspace_bytes(ctx, cfg))
    return fail(ctx, RRTMG_BAD_ARG, "workspace smaller than rrtmg_sw_workspace_bytes");
  CallScratch sc(ctx, stream, ws, ws_bytes);
  e = sc.take(&mask, mask_bytes);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "scratch (mcica mask)");
  e = sc.take(&daylist, (static_cast<size_t>(ncol) + 1) * sizeof(int));
  if (e != cudaSuccess) {
    sc.release();
    return cuda_fail(ctx, e, "scratch (day list)");
  }
  const int tslot = timing_slot(ctx, 1);
  timing_mark(ctx, 1, tslot, stream);
  McicaArgs m{};
  m.ncol = ncol; m.ny = cfg->ny; m.nk = cfg->nk; m.nlay = nlay; m.nsub = kSwGpts; m.words = kSwMaskWords;
  m.enabled = icld >= 1;
  m.live = live;
  m.p3d = in->p3d; m.cldfra = in->cldfra3d; m.jumps = jumps; m.mask = mask;
  e = launch_mcica(m, stream);
  timing_mark(ctx, 1, tslot, stream);
  if (e != cudaSuccess) {
    sc.release();
    return cuda_fail(ctx, e, "mcica kernel launch");
  }
  SwArgs a{};
  a.live = live;
  a.fp64_from = cfg->fp64_steps ? fp64_first_layer(cfg->nk) : kMaxLay + 1;
  a.fp64_reftra = cfg->fp64_steps != 0;
  a.nx = cfg->nx; a.ny = cfg->ny; a.nk = cfg->nk; a.nlay = nlay; a.ncol = ncol;
  a.co2 = cfg->co2vmr; a.n2o = cfg->n2ovmr; a.ch4 = cfg->ch4vmr; a.solcon = cfg->solcon;
  a.has_reqc = cfg->has_reqc; a.has_reqi = cfg->has_reqi; a.has_reqs = cfg->has_reqs; a.icloud = cfg->icloud;
  a.icld = icld; a.inflg = inflg; a.iceflg = iceflg; a.liqflg = liqflg;
  a.in = common_inputs(in->p3d, in->p8w, in->pi3d, in->t3d, in->t8w, in->tsk, in->qv3d, in->qc3d, in->qi3d,
                       in->qs3d, in->cldfra3d, in->o33d, in->xland, in->xice, in->snow, in->re_cloud, in->re_ice,
                       in->re_snow);
  a.in.albedo = in->albedo;
  a.in.coszr = in->coszr;
  {
    const int given = (in->alswvisdir != nullptr) + (in->alswvisdif != nullptr) + (in->alswnirdir != nullptr) +
                      (in->alswnirdif != nullptr);
    if (given != 0 && given != 4) {
      sc.release();
      return fail(ctx, RRTMG_BAD_ARG, "pass all four Noah-MP albedo fields or none");
    }
    if (given == 4) {
      a.in.alswvisdir = in->alswvisdir;
      a.in.alswvisdif = in->alswvisdif;
      a.in.alswnirdir = in->alswnirdir;
      a.in.alswnirdif = in->alswnirdif;
    }
  }
  a.mask = mask;
  a.rthraten = out->rthratensw; a.rthratenc = out->rthratenswc;
  a.upt = out->swupt; a.uptc = out->swuptc; a.dnt = out->swdnt; a.dntc = out->swdntc;
  a.upb = out->swupb; a.upbc = out->swupbc; a.dnb = out->swdnb; a.dnbc = out->swdnbc;
  a.swcf = out->swcf; a.gsw = out->gsw; a.swddir = out->swddir; a.swddni = out->swddni; a.swddif = out->swddif;
  a.swdownc = out->swdownc; a.swddnic = out->swddnic; a.swddirc = out->swddirc; a.coszr_out = out->coszr;
  a.zero2[0] = out->swuptcln; a.zero2[1] = out->swdntcln; a.zero2[2] = out->swupbcln; a.zero2[3] = out->swdnbcln;
  a.nday = daylist + ncol;
  a.daylist = daylist;
  a.chunk_capacity = static_cast<int>(sw_chunk_columns(ctx, ncol));
  float *records = nullptr;
  e = sc.take(&records, sw_record_floats(cfg->nk, a.chunk_capacity) * sizeof(float));
  if (e != cudaSuccess) {
    sc.release();
    return cuda_fail(ctx, e, "scratch (sw layer records)");
  }
  a.records = records;
  // the day count is known only on the device: the chunks cover all ncol
  // list slots, and slots at or beyond the day count exit at once; the day
  // list counts with the first chunk's optics
  e = launch_sw_daylist(a, stream);
  for (int first = 0; first < ncol && e == cudaSuccess; first += a.chunk_capacity) {
    a.chunk_first = first;
    a.chunk_count = ncol - first < a.chunk_capacity ? ncol - first : a.chunk_capacity;
    e = launch_sw_chunk_optics(ctx->tables, a, stream);
    timing_mark(ctx, 1, tslot, stream);
    if (e == cudaSuccess) e = launch_sw_chunk_sweep(ctx->tables, a, stream);
    timing_mark(ctx, 1, tslot, stream);
  }
  if (e == cudaSuccess && !live) {
    cudaError_t es = cudaSuccess;
    uint32_t *status = status_target(ctx, 1, ncol, &es);
    if (es != cudaSuccess) e = es;
    if (status) {
      StatusArgs sa{};
      sa.ncol = ncol; sa.nx = cfg->nx; sa.ny = cfg->ny; sa.nk = cfg->nk; sa.side = 1;
      sa.has_req = cfg->has_reqc || cfg->has_reqi || cfg->has_reqs;
      sa.in = a.in;
      sa.rthraten = out->rthratensw; sa.rthratenc = out->rthratenswc;
      const float *o2[8] = {out->swupt, out->swuptc, out->swdnt, out->swdntc, out->swupb, out->swupbc,
                            out->swdnb, out->swdnbc};
      for (int q = 0; q < 8; ++q) sa.out2d[q] = o2[q];
      sa.n2d = 8;
      sa.status = status;
      e = launch_column_status(sa, stream);
    }
  }
  cudaError_t ef = sc.release();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "sw kernel launch");
  if (ef != cudaSuccess) return cuda_fail(ctx, ef, "cudaFreeAsync(sw scratch)");
  return RRTMG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
rrtmg_status rrtmg_lwrad(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_lw_in *in, rrtmg_lw_out *out,
                         void *stream) {
  return lwrad_impl(ctx, cfg, in, out, stream, nullptr);
}

rrtmg_status rrtmg_swrad(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_sw_in *in, rrtmg_sw_out *out,
                         void *stream) {
  return swrad_impl(ctx, cfg, in, out, stream, nullptr);
}

static bool device_count(const int *p) {
  cudaPointerAttributes at{};
  if (!p || cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

rrtmg_status rrtmg_lwrad_live(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_lw_in *in, rrtmg_lw_out *out,
                              const int *live_count, void *stream) {
  if (!device_count(live_count)) return fail(ctx, RRTMG_BAD_ARG, "live_count must be a device pointer");
  return lwrad_impl(ctx, cfg, in, out, stream, live_count);
}

rrtmg_status rrtmg_swrad_live(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_sw_in *in, rrtmg_sw_out *out,
                              const int *live_count, void *stream) {
  if (!device_count(live_count)) return fail(ctx, RRTMG_BAD_ARG, "live_count must be a device pointer");
  return swrad_impl(ctx, cfg, in, out, stream, live_count);
}

size_t rrtmg_lw_workspace_bytes(rrtmg_ctx *ctx, const rrtmg_config *cfg) {
  if (check_config(ctx, cfg) != RRTMG_OK) return 0;
  const int nlay = rrtmg_lw_nlayers(cfg->p_top, cfg->nk);
  if (nlay > kMaxLay || nlay - cfg->nk > kMaxBuf || nlay < cfg->nk) return 0;
  const KissJump *jumps = nullptr;  // built here, ahead of the first call
  {
    DeviceGuard guard(ctx->device);
    if (guard.status() != cudaSuccess || get_jumps(ctx, nlay, kLwGpts, 150, &jumps) != RRTMG_OK) return 0;
  }
  return lw_workspace_bytes(ctx, cfg);
}

size_t rrtmg_sw_workspace_bytes(rrtmg_ctx *ctx, const rrtmg_config *cfg) {
  if (check_config(ctx, cfg) != RRTMG_OK || cfg->nk + 1 > kMaxLay) return 0;
  const KissJump *jumps = nullptr;
  {
    DeviceGuard guard(ctx->device);
    if (guard.status() != cudaSuccess || get_jumps(ctx, cfg->nk + 1, kSwGpts, 1, &jumps) != RRTMG_OK) return 0;
  }
  return sw_workspace_bytes(ctx, cfg);
}

rrtmg_status rrtmg_lwrad_ws(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_lw_in *in, rrtmg_lw_out *out,
                            void *workspace, size_t workspace_bytes, void *stream) {
  if (!workspace) return fail(ctx, RRTMG_BAD_ARG, "null workspace");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0) return fail(ctx, RRTMG_BAD_ARG, "workspace not 256-byte aligned");
  return lwrad_impl(ctx, cfg, in, out, stream, nullptr, workspace, workspace_bytes);
}

rrtmg_status rrtmg_swrad_ws(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_sw_in *in, rrtmg_sw_out *out,
                            void *workspace, size_t workspace_bytes, void *stream) {
  if (!workspace) return fail(ctx, RRTMG_BAD_ARG, "null workspace");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0) return fail(ctx, RRTMG_BAD_ARG, "workspace not 256-byte aligned");
  return swrad_impl(ctx, cfg, in, out, stream, nullptr, workspace, workspace_bytes);
}

// rrtmg_lwrad_static_scratch: the LW call with its McICA scratch in fixed
// file-scope device arrays instead of a per-call stream-ordered allocation.
//
// Scratch: g_static_mask holds kStaticMaskWords 32-bit words (32 MiB); a call
// needs nlay * 5 * nx * ny of them and is rejected with RRTMG_BAD_ARG above
// that.  g_static_jumps holds the 140 KISS jumps of every layer count the
// kernels accept (slot nlay, 2.7 MB); they are written once per device, so a
// call only selects its slot and copies nothing.  Nothing has to start at
// zero: the McICA kernel writes every mask word the LW kernel then reads.
//
// Set-up: the first call on each device, with that device current, looks up
// both symbols (cudaGetSymbolAddress) and fills the jump table with one
// synchronous copy; that first call should come before any stream capture
// begins.  Later calls, with any nlay, enqueue only the two kernels.  The
// scratch is shared by every context and stream on a device, so calls that
// overlap in time on one device race.
namespace {

constexpr size_t kStaticMaskWords = size_t(8) << 20;  // 32 MiB of mask words
constexpr int kStaticMaxDevices = 64;
constexpr int kStaticMinLay = 4;  // nlay >= nk >= 4

__device__ __align__(256) uint32_t g_static_mask[kStaticMaskWords];
__device__ __align__(256) KissJump g_static_jumps[kMaxLay + 1][kLwGpts];

struct StaticScratch {
  bool ready = false;
  uint32_t *mask = nullptr;
  KissJump *jumps = nullptr;  // slot nlay at jumps + nlay * kLwGpts
};

std::mutex g_static_mutex;
StaticScratch g_static_scratch[kStaticMaxDevices];

// One-time set-up of the current device's scratch (caller holds g_static_mutex).
cudaError_t static_scratch_setup(StaticScratch &s) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_static_mask);
  if (e != cudaSuccess) return e;
  s.mask = static_cast<uint32_t *>(p);
  e = cudaGetSymbolAddress(&p, g_static_jumps);
  if (e != cudaSuccess) return e;
  s.jumps = static_cast<KissJump *>(p);
  std::vector<KissJump> host(static_cast<size_t>(kMaxLay + 1) * kLwGpts, KissJump{});
  for (int nlay = kStaticMinLay; nlay <= kMaxLay; ++nlay)
    kiss_jumps(150ull, nlay, kLwGpts, host.data() + static_cast<size_t>(nlay) * kLwGpts);
  e = cudaMemcpy(s.jumps, host.data(), host.size() * sizeof(KissJump), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return e;
  s.ready = true;
  return cudaSuccess;
}

}  // namespace

extern "C" rrtmg_status rrtmg_lwrad_static_scratch(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_lw_in *in,
                                                   rrtmg_lw_out *out, void *stream_ptr) {
  rrtmg_status st = check_config(ctx, cfg);
  if (st != RRTMG_OK) return st;
  if (!in || !out) return fail(ctx, RRTMG_BAD_ARG, "null input or output block");
  if (any_null({in->p3d, in->p8w, in->pi3d, in->t3d, in->t8w, in->tsk, in->qv3d, in->qc3d, in->qi3d, in->qs3d,
                in->cldfra3d, in->o33d, in->emiss, in->xland, in->xice, in->snow, in->re_cloud, in->re_ice,
                in->re_snow}))
    return fail(ctx, RRTMG_BAD_ARG, "a required LW input pointer is null");
  if (any_null({out->rthratenlw, out->rthratenlwc, out->lwupt, out->lwuptc, out->lwuptcln, out->lwdnt, out->lwdntc,
                out->lwdntcln, out->lwupb, out->lwupbc, out->lwupbcln, out->lwdnb, out->lwdnbc, out->lwdnbcln,
                out->glw, out->olr, out->lwcf}))
    return fail(ctx, RRTMG_BAD_ARG, "a required LW output pointer is null");
  const int nlay = rrtmg_lw_nlayers(cfg->p_top, cfg->nk);
  if (nlay > kMaxLay || nlay - cfg->nk > kMaxBuf || nlay < cfg->nk)
    return fail(ctx, RRTMG_BAD_ARG, "too many layers (nk and p_top exceed the kernel's layer capacity)");
  const int ncol = cfg->nx * cfg->ny;
  const size_t words = static_cast<size_t>(nlay) * kLwMaskWords * static_cast<size_t>(ncol);
  if (words > kStaticMaskWords)
    return fail(ctx, RRTMG_BAD_ARG,
                "domain too large for the static McICA scratch: needs " + std::to_string(words) +
                    " mask words (nlay*5*nx*ny), the scratch holds " + std::to_string(kStaticMaskWords) +
                    "; use rrtmg_lwrad");
  int inflg, iceflg, liqflg;
  cloud_flags(cfg, &inflg, &iceflg, &liqflg);
  const int icld = cfg->cldovrlp;
  if (icld >= 1 && (inflg < 2 || iceflg < 3 || liqflg != 1))
    return fail(ctx, RRTMG_UNSUPPORTED_OPTION, "cloud optics option not supported by cldprmc_lw");
  if (ctx->device < 0 || ctx->device >= kStaticMaxDevices)
    return fail(ctx, RRTMG_BAD_ARG, "device ordinal beyond the static scratch's device slots");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  DeviceGuard guard(ctx->device);
  cudaError_t e = guard.status();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");

  uint32_t *mask = nullptr;
  KissJump *jumps = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_static_mutex);
    StaticScratch &s = g_static_scratch[ctx->device];
    if (!s.ready) {  // once per device, with that device current
      e = static_scratch_setup(s);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "static McICA scratch set-up");
    }
    mask = s.mask;
    jumps = s.jumps + static_cast<size_t>(nlay) * kLwGpts;
  }

  McicaArgs m{};
  m.ncol = ncol; m.ny = cfg->ny; m.nk = cfg->nk; m.nlay = nlay; m.nsub = kLwGpts; m.words = kLwMaskWords;
  m.enabled = icld >= 1;
  m.p3d = in->p3d; m.cldfra = in->cldfra3d; m.jumps = jumps; m.mask = mask;
  e = launch_mcica(m, stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "mcica kernel launch");
  LwArgs a{};
  a.fp64_from = cfg->fp64_steps ? fp64_first_layer(cfg->nk) : kMaxLay + 1;
  a.nx = cfg->nx; a.ny = cfg->ny; a.nk = cfg->nk; a.nlay = nlay; a.ncol = ncol;
  a.co2 = cfg->co2vmr; a.n2o = cfg->n2ovmr; a.ch4 = cfg->ch4vmr; a.cfc11 = cfg->cfc11vmr; a.cfc12 = cfg->cfc12vmr;
  a.has_reqc = cfg->has_reqc; a.has_reqi = cfg->has_reqi; a.has_reqs = cfg->has_reqs; a.icloud = cfg->icloud;
  a.icld = icld; a.inflg = inflg; a.iceflg = iceflg; a.liqflg = liqflg;
  a.in = common_inputs(in->p3d, in->p8w, in->pi3d, in->t3d, in->t8w, in->tsk, in->qv3d, in->qc3d, in->qi3d,
                       in->qs3d, in->cldfra3d, in->o33d, in->xland, in->xice, in->snow, in->re_cloud, in->re_ice,
                       in->re_snow);
  a.in.emiss = in->emiss;
  a.mask = mask;
  a.rthraten = out->rthratenlw; a.rthratenc = out->rthratenlwc;
  a.upt = out->lwupt; a.uptc = out->lwuptc; a.dnt = out->lwdnt; a.dntc = out->lwdntc;
  a.upb = out->lwupb; a.upbc = out->lwupbc; a.dnb = out->lwdnb; a.dnbc = out->lwdnbc;
  a.glw = out->glw; a.olr = out->olr; a.lwcf = out->lwcf;
  a.zero2[0] = out->lwuptcln; a.zero2[1] = out->lwdntcln; a.zero2[2] = out->lwupbcln; a.zero2[3] = out->lwdnbcln;
  e = launch_lw(ctx->tables, a, stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "lw kernel launch");
  return RRTMG_OK;
}

extern "C" rrtmg_status rrtmg_timing_enable(rrtmg_ctx *ctx, int enable) {
  if (!ctx) return fail(nullptr, RRTMG_BAD_ARG, "null context");
  std::lock_guard<std::mutex> lk(ctx->mutex);
  if (enable && ctx->events[0].empty()) {
    for (int side = 0; side < 2; ++side) {
      ctx->events[side].resize(kTimingSlots);
      ctx->marks[side].assign(kTimingSlots, 0);
    }
  }
  ctx->timing = enable != 0;
  ctx->timing_next[0] = ctx->timing_next[1] = 0;
  ctx->timing_count[0] = ctx->timing_count[1] = 0;
  return RRTMG_OK;
}

extern "C" int rrtmg_timing_read(rrtmg_ctx *ctx, int side, float *ms, int max_calls) {
  if (!ctx || side < 0 || side > 1 || !ms || max_calls <= 0) return -1;
  DeviceGuard guard(ctx->device);
  if (guard.status() != cudaSuccess) return -1;
  std::lock_guard<std::mutex> lk(ctx->mutex);
  if (ctx->events[side].empty()) return 0;
  const int count = ctx->timing_count[side] < max_calls ? ctx->timing_count[side] : max_calls;
  const int newest = (ctx->timing_next[side] + kTimingSlots - 1) % kTimingSlots;
  for (int q = 0; q < count; ++q) {
    // oldest of the returned calls first
    const int slot = (newest - (count - 1 - q) + kTimingSlots) % kTimingSlots;
    const std::vector<cudaEvent_t> &ev = ctx->events[side][slot];
    const int n = ctx->marks[side][slot];
    if (n < 2 || cudaEventSynchronize(ev[n - 1]) != cudaSuccess) return -1;
    // interval 0: McICA; odd intervals: a chunk's optics; even ones: its sweep
    float phase[3] = {0.0f, 0.0f, 0.0f};
    for (int m = 0; m + 1 < n; ++m) {
      float t = 0.0f;
      if (cudaEventElapsedTime(&t, ev[m], ev[m + 1]) != cudaSuccess) return -1;
      phase[m == 0 ? 0 : (m % 2 == 1 ? 1 : 2)] += t;
    }
    for (int k = 0; k < 3; ++k) ms[q * 3 + k] = phase[k];
  }
  return count;
}

extern "C" rrtmg_status rrtmg_column_status_enable(rrtmg_ctx *ctx, int enable) {
  if (!ctx) return fail(nullptr, RRTMG_BAD_ARG, "null context");
  std::lock_guard<std::mutex> lk(ctx->mutex);
  ctx->colstatus = enable != 0;
  return RRTMG_OK;
}

extern "C" rrtmg_status rrtmg_last_column_errors(rrtmg_ctx *ctx, int side, uint32_t *dev_status, int ncol,
                                                 void *stream_ptr) {
  if (!ctx) return fail(nullptr, RRTMG_BAD_ARG, "null context");
  if (side < 0 || side > 1 || !dev_status) return fail(ctx, RRTMG_BAD_ARG, "side must be 0 or 1, dev_status set");
  const uint32_t *src = nullptr;
  {
    std::lock_guard<std::mutex> lk(ctx->mutex);
    if (ctx->status_ncol[side] < 0 || !ctx->status_buf[side]) src = nullptr;
    else if (ctx->status_ncol[side] == ncol) src = ctx->status_buf[side];
  }
  if (!src) return fail(ctx, RRTMG_BAD_ARG, "no column status recorded for this side and column count");
  DeviceGuard guard(ctx->device);
  cudaError_t e = guard.status();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  e = cudaMemcpyAsync(dev_status, src, sizeof(uint32_t) * static_cast<size_t>(ncol), cudaMemcpyDeviceToDevice,
                      static_cast<cudaStream_t>(stream_ptr));
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(column status)");
  return RRTMG_OK;
}

extern "C" rrtmg_status rrtmg_set_schedule(rrtmg_ctx *ctx, const rrtmg_schedule *sch) {
  if (!ctx || !sch) return fail(ctx, RRTMG_BAD_ARG, "null context or schedule");
  const int lo = 1024, hi = 1 << 24;
  if (sch->lw_chunk_columns < lo || sch->lw_chunk_columns > hi || sch->sw_chunk_columns < lo ||
      sch->sw_chunk_columns > hi || sch->sw_split_max_columns < 0 || sch->sw_split_max_columns > 16384 ||
      sch->lw_split_max_columns < 0 || sch->lw_split_max_columns > 8192)
    return fail(ctx, RRTMG_BAD_ARG,
                "schedule out of range: chunks 1024..16777216 columns, split limits 0..16384 (SW) and "
                "0..8192 (LW) columns");
  std::lock_guard<std::mutex> lk(ctx->mutex);
  ctx->lw_chunk = sch->lw_chunk_columns;
  ctx->sw_chunk = sch->sw_chunk_columns;
  ctx->sw_split_max = sch->sw_split_max_columns;
  ctx->lw_split_max = sch->lw_split_max_columns;
  return RRTMG_OK;
}

extern "C" rrtmg_status rrtmg_get_schedule(const rrtmg_ctx *ctx, rrtmg_schedule *sch) {
  if (!ctx || !sch) return RRTMG_BAD_ARG;
  std::lock_guard<std::mutex> lk(const_cast<rrtmg_ctx *>(ctx)->mutex);
  sch->lw_chunk_columns = ctx->lw_chunk;
  sch->sw_chunk_columns = ctx->sw_chunk;
  sch->sw_split_max_columns = ctx->sw_split_max;
  sch->lw_split_max_columns = ctx->lw_split_max;
  return RRTMG_OK;
}

// ---------------------------------------------------------------------------
// radiation prologue (include/rrtmg_prologue.h)
// ---------------------------------------------------------------------------
extern "C" rrtmg_status rrtmg_set_ozone_climatology(rrtmg_ctx *ctx, const float *plev_pa, int levsiz,
                                                    const float *lat, int latsiz, const float *ozone) {
  if (!ctx) return fail(nullptr, RRTMG_BAD_ARG, "null context");
  if (!plev_pa || !lat || !ozone) return fail(ctx, RRTMG_BAD_ARG, "null climatology array");
  if (levsiz < 2 || levsiz > 128 || latsiz < 2 || latsiz > 256 || latsiz * levsiz > 12288)
    return fail(ctx, RRTMG_BAD_ARG, "climatology size outside 2..128 levels, 2..256 latitudes, 12288 points");
  for (int i = 0; i + 1 < levsiz; ++i)
    if (!(plev_pa[i] < plev_pa[i + 1])) return fail(ctx, RRTMG_BAD_ARG, "ozone pressures must be ascending");
  for (int i = 0; i + 1 < latsiz; ++i)
    if (!(lat[i] < lat[i + 1])) return fail(ctx, RRTMG_BAD_ARG, "ozone latitudes must be ascending");
  DeviceGuard guard(ctx->device);
  cudaError_t e = guard.status();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  const size_t tab = static_cast<size_t>(12) * latsiz * levsiz;
  float *buf = nullptr;
  e = cudaMalloc(&buf, sizeof(float) * (levsiz + latsiz + tab));
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(ozone climatology)");
  if ((e = cudaMemcpy(buf, plev_pa, sizeof(float) * levsiz, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(buf + levsiz, lat, sizeof(float) * latsiz, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(buf + levsiz + latsiz, ozone, sizeof(float) * tab, cudaMemcpyHostToDevice)) != cudaSuccess) {
    cudaFree(buf);
    return cuda_fail(ctx, e, "cudaMemcpy(ozone climatology)");
  }
  std::lock_guard<std::mutex> lk(ctx->mutex);
  if (ctx->ozone) ctx->retired_ozone.push_back(ctx->ozone);
  ctx->ozone = buf;
  ctx->oz_levsiz = levsiz;
  ctx->oz_latsiz = latsiz;
  return RRTMG_OK;
}

extern "C" rrtmg_status rrtmg_radiation_prologue(rrtmg_ctx *ctx, int nx, int nk, int ny,
                                                 const rrtmg_prologue_scalars *sc, const rrtmg_prologue_in *in,
                                                 rrtmg_prologue_out *out, void *stream_ptr) {
  if (!ctx) return fail(nullptr, RRTMG_BAD_ARG, "null context");
  if (!in || !out) return fail(ctx, RRTMG_BAD_ARG, "null input or output block");
  if (nx <= 0 || ny <= 0 || nk <= 0) return fail(ctx, RRTMG_BAD_ARG, "nx, nk and ny must be positive");
  if (static_cast<long long>(nx) * ny > (1ll << 30)) return fail(ctx, RRTMG_BAD_ARG, "too many columns in one call");
  const bool cld = out->cldfra3d, oz = out->o33d, cz = out->coszr, flag = out->condensate_present;
  if (cld && any_null({in->qv3d, in->qc3d, in->qi3d, in->qs3d, in->t3d, in->p3d}))
    return fail(ctx, RRTMG_BAD_ARG, "cloud fraction needs qv3d, qc3d, qi3d, qs3d, t3d and p3d");
  if (flag && any_null({in->qc3d, in->qi3d, in->qs3d}))
    return fail(ctx, RRTMG_BAD_ARG, "the condensate flag needs qc3d, qi3d and qs3d");
  if (oz && any_null({in->xlat, in->p3d})) return fail(ctx, RRTMG_BAD_ARG, "ozone needs xlat and p3d");
  if (cz && any_null({in->xlat, in->xlong})) return fail(ctx, RRTMG_BAD_ARG, "cos zenith needs xlat and xlong");
  if ((oz || cz) && !sc) return fail(ctx, RRTMG_BAD_ARG, "ozone and cos zenith need the step scalars");
  if (cz && !ctx->have_svml)
    return fail(ctx, RRTMG_BAD_ARG, "the table blob has no SVML sin/cos constants (rebuild it)");
  if (oz && (sc->month_lo < 0 || sc->month_lo > 11 || sc->month_hi < 0 || sc->month_hi > 11))
    return fail(ctx, RRTMG_BAD_ARG, "ozone months must be in 0..11");
  PrologueArgs a{};
  a.nx = nx;
  a.nk = nk;
  a.ny = ny;
  a.qv = in->qv3d; a.qc = in->qc3d; a.qi = in->qi3d; a.qs = in->qs3d; a.t = in->t3d; a.p = in->p3d;
  a.xlat = in->xlat;
  a.xlong = in->xlong;
  a.cldfra = out->cldfra3d;
  a.o33d = out->o33d;
  a.coszr = out->coszr;
  a.condensate = out->condensate_present;
  if (sc) {
    a.tloctm0 = sc->tloctm0;
    a.sin_declin = sc->sin_declin;
    a.cos_declin = sc->cos_declin;
    a.month_lo = sc->month_lo;
    a.month_hi = sc->month_hi;
    a.fact_lo = sc->fact_lo;
    a.fact_hi = sc->fact_hi;
  }
  bool have_ozone = false;
  {
    // fail() takes this mutex too: record under it, report after it
    std::lock_guard<std::mutex> lk(ctx->mutex);
    a.svml = ctx->svml;
    have_ozone = ctx->ozone != nullptr;
    if (oz && have_ozone) {
      a.levsiz = ctx->oz_levsiz;
      a.latsiz = ctx->oz_latsiz;
      a.oz_plev = ctx->ozone;
      a.oz_lat = ctx->ozone + a.levsiz;
      a.oz_tab = ctx->ozone + a.levsiz + a.latsiz;
    }
  }
  if (oz && !have_ozone) return fail(ctx, RRTMG_BAD_ARG, "no ozone climatology (rrtmg_set_ozone_climatology)");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  DeviceGuard guard(ctx->device);
  cudaError_t e = guard.status();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  if (flag && (e = cudaMemsetAsync(out->condensate_present, 0, sizeof(int), stream)) != cudaSuccess)
    return cuda_fail(ctx, e, "cudaMemsetAsync(condensate flag)");
  e = launch_prologue(a, stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "prologue kernel launch");
  return RRTMG_OK;
}

extern "C" rrtmg_status rrtmg_cal_cldfra1(rrtmg_ctx *ctx, int nx, int nk, int ny, const float *qv, const float *qc,
                                         const float *qi, const float *qs, const float *t_phy, const float *p_phy,
                                         float *cldfra, void *stream) {
  rrtmg_prologue_in in{};
  in.qv3d = qv; in.qc3d = qc; in.qi3d = qi; in.qs3d = qs; in.t3d = t_phy; in.p3d = p_phy;
  rrtmg_prologue_out out{};
  out.cldfra3d = cldfra;
  if (!cldfra) return fail(ctx, RRTMG_BAD_ARG, "null cldfra output");
  return rrtmg_radiation_prologue(ctx, nx, nk, ny, nullptr, &in, &out, stream);
}

extern "C" rrtmg_status rrtmg_calc_coszen(rrtmg_ctx *ctx, int nx, int ny, const float *xlat, const float *xlong,
                                         const rrtmg_prologue_scalars *sc, float *coszen, void *stream) {
  rrtmg_prologue_in in{};
  in.xlat = xlat;
  in.xlong = xlong;
  rrtmg_prologue_out out{};
  out.coszr = coszen;
  if (!coszen) return fail(ctx, RRTMG_BAD_ARG, "null coszen output");
  return rrtmg_radiation_prologue(ctx, nx, 1, ny, sc, &in, &out, stream);
}

extern "C" rrtmg_status rrtmg_cam_o3rad(rrtmg_ctx *ctx, int nx, int nk, int ny, const float *xlat, const float *p3d,
                                       const rrtmg_prologue_scalars *sc, float *o33d, void *stream) {
  rrtmg_prologue_in in{};
  in.xlat = xlat;
  in.p3d = p3d;
  rrtmg_prologue_out out{};
  out.o33d = o33d;
  if (!o33d) return fail(ctx, RRTMG_BAD_ARG, "null o33d output");
  return rrtmg_radiation_prologue(ctx, nx, nk, ny, sc, &in, &out, stream);
}

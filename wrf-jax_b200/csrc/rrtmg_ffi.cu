// XLA FFI custom-call handlers over the workspace entry points
// (include/rrtmg_xla_ffi.h).
//
// A handler checks the call frame completely on the host (operand and result
// counts, types and shapes, the attributes) before it touches the GPU, so a
// malformed call returns an XLA error and launches nothing.  The stream comes
// from XLA (XLA_FFI_Stream_Get); the device is the one holding the operands.
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>

#include "../../include/rrtmg_b200.h"
#include "../../include/rrtmg_xla_ffi.h"
#include "rrtmg_kernels.h"
#include "xla_ffi_abi.h"

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
std::string g_blob;                      // rrtmg_ffi_set_table_blob
rrtmg_ctx *g_ctx[kMaxDevices] = {};      // one context per device, never destroyed

XLA_FFI_Error *make_error(const XLA_FFI_CallFrame *f, XLA_FFI_Error_Code code, const std::string &msg) {
  XLA_FFI_Error_Create_Args a;
  std::memset(&a, 0, sizeof(a));
  a.struct_size = sizeof(a);
  a.message = msg.c_str();
  a.errc = code;
  return f->api->XLA_FFI_Error_Create(&a);
}

// Context of `device`, created on first use from the configured blob.
rrtmg_status context_for(int device, rrtmg_ctx **out, std::string &err) {
  if (device < 0 || device >= kMaxDevices) {
    err = "device ordinal out of range";
    return RRTMG_BAD_ARG;
  }
  std::lock_guard<std::mutex> lk(g_mutex);
  if (!g_ctx[device]) {
    std::string path = g_blob;
    if (path.empty()) {
      const char *env = std::getenv("RRTMG_TABLE_BLOB");
      if (env) path = env;
    }
    if (path.empty()) {
      err = "no table blob: call rrtmg_ffi_set_table_blob or set RRTMG_TABLE_BLOB";
      return RRTMG_BAD_ARG;
    }
    rrtmg_status st = rrtmg_create(path.c_str(), device, &g_ctx[device]);
    if (st != RRTMG_OK) {
      err = std::string("rrtmg_create: ") + rrtmg_last_error(nullptr);
      g_ctx[device] = nullptr;
      return st;
    }
  }
  *out = g_ctx[device];
  return RRTMG_OK;
}

// The call frame's scalar attribute `name` as a double (f32/f64/s32/s64).
bool attr_number(const XLA_FFI_Attrs &attrs, const char *name, double *v) {
  const size_t len = std::strlen(name);
  for (int64_t i = 0; i < attrs.size; ++i) {
    const XLA_FFI_ByteSpan *n = attrs.names[i];
    if (!n || n->len != len || std::memcmp(n->ptr, name, len) != 0) continue;
    if (attrs.types[i] != XLA_FFI_AttrType_SCALAR) return false;
    const XLA_FFI_Scalar *s = static_cast<const XLA_FFI_Scalar *>(attrs.attrs[i]);
    switch (s->dtype) {
      case XLA_FFI_DataType_F32: *v = *static_cast<const float *>(s->value); return true;
      case XLA_FFI_DataType_F64: *v = *static_cast<const double *>(s->value); return true;
      case XLA_FFI_DataType_S32: *v = *static_cast<const int32_t *>(s->value); return true;
      case XLA_FFI_DataType_S64: *v = static_cast<double>(*static_cast<const int64_t *>(s->value)); return true;
      default: return false;
    }
  }
  return false;
}

// Shapes (nx, nk, ny), (nx, nk + 1, ny) and (nx, ny) of the operands.
enum Shape { k3D, kLev, k2D };

bool check_buffer(const XLA_FFI_Buffer *b, XLA_FFI_DataType dtype, Shape shape, int64_t nx, int64_t nk, int64_t ny) {
  if (!b || b->dtype != dtype || !b->data) return false;
  if (shape == k2D) return b->rank == 2 && b->dims[0] == nx && b->dims[1] == ny;
  const int64_t levels = shape == kLev ? nk + 1 : nk;
  return b->rank == 3 && b->dims[0] == nx && b->dims[1] == levels && b->dims[2] == ny;
}

const XLA_FFI_Buffer *arg(const XLA_FFI_CallFrame *f, int i) {
  return static_cast<const XLA_FFI_Buffer *>(f->args.args[i]);
}
const XLA_FFI_Buffer *ret(const XLA_FFI_CallFrame *f, int i) {
  return static_cast<const XLA_FFI_Buffer *>(f->rets.rets[i]);
}

// Metadata query: the API version the handler was built for, no traits.
bool answer_metadata(XLA_FFI_CallFrame *f) {
  for (XLA_FFI_Extension_Base *e = f->extension_start; e; e = e->next) {
    if (e->type != XLA_FFI_Extension_Metadata) continue;
    XLA_FFI_Metadata *m = reinterpret_cast<XLA_FFI_Metadata_Extension *>(e)->metadata;
    m->api_version.major_version = 0;
    m->api_version.minor_version = 1;
    m->traits = 0;
    return true;
  }
  return false;
}

// The scalar attributes both sides share; nullptr on success, else the missing name.
const char *read_flags(const XLA_FFI_Attrs &attrs, rrtmg_config &c) {
  static const char *names[] = {"has_reqc", "has_reqi", "has_reqs", "icloud", "cldovrlp", "fp64_steps"};
  int *dst[] = {&c.has_reqc, &c.has_reqi, &c.has_reqs, &c.icloud, &c.cldovrlp, &c.fp64_steps};
  for (int q = 0; q < 6; ++q) {
    double v = 0.0;
    if (!attr_number(attrs, names[q], &v)) return names[q];
    *dst[q] = static_cast<int>(v);
  }
  return nullptr;
}

template <typename T>
XLA_FFI_Error *run(XLA_FFI_CallFrame *f, bool lw) {
  if (answer_metadata(f)) return nullptr;
  if (f->stage != XLA_FFI_ExecutionStage_EXECUTE) return nullptr;
  const int n_in = lw ? 20 : 21, n_out = lw ? 17 : 23;
  const bool sf8 = !lw && f->args.size == n_in + 4;
  if (f->args.size != n_in && !sf8)
    return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT,
                      lw ? "rrtmg_lwrad takes 20 operands" : "rrtmg_swrad takes 21 or 25 operands");
  if (f->rets.size != n_out + 1)
    return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT,
                      lw ? "rrtmg_lwrad has 17 results and a workspace" : "rrtmg_swrad has 23 results and a workspace");
  for (int64_t i = 0; i < f->args.size; ++i)
    if (f->args.types[i] != XLA_FFI_ArgType_BUFFER)
      return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT, "operands must be buffers");
  for (int64_t i = 0; i < f->rets.size; ++i)
    if (f->rets.types[i] != XLA_FFI_RetType_BUFFER)
      return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT, "results must be buffers");
  // domain from t3d (operand 3 of both sides)
  const XLA_FFI_Buffer *t3d = arg(f, 3);
  if (!t3d || t3d->rank != 3)
    return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT, "t3d must be (west_east, bottom_top, south_north)");
  const int64_t nx = t3d->dims[0], nk = t3d->dims[1], ny = t3d->dims[2];
  if (nx <= 0 || ny <= 0 || nk <= 0 || nx * ny > (int64_t(1) << 30) || nk > 4096)
    return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT, "domain size out of range");
  // operand shapes: rrtmg_lw_in / rrtmg_sw_in order
  static const Shape lw_shapes[20] = {k3D, kLev, k3D, k3D, kLev, k2D, k3D, k3D, k3D, k3D,
                                      k3D, k3D,  k3D, k2D, k2D,  k2D, k2D, k3D, k3D, k3D};
  static const Shape sw_shapes[25] = {k3D, kLev, k3D, k3D, kLev, k2D, k3D, k3D, k3D, k3D, k3D, k3D, k3D,
                                      k2D, k2D,  k2D, k2D, k2D,  k3D, k3D, k3D, k2D, k2D, k2D, k2D};
  for (int64_t i = 0; i < f->args.size; ++i)
    if (!check_buffer(arg(f, i), XLA_FFI_DataType_F32, lw ? lw_shapes[i] : sw_shapes[i], nx, nk, ny))
      return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT,
                        "operand " + std::to_string(i) + ": wrong type or shape (float32, WRF layout)");
  for (int i = 0; i < n_out; ++i)
    if (!check_buffer(ret(f, i), XLA_FFI_DataType_F32, i < 2 ? k3D : k2D, nx, nk, ny))
      return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT,
                        "result " + std::to_string(i) + ": wrong type or shape (float32, WRF layout)");
  const XLA_FFI_Buffer *ws = ret(f, n_out);
  if (!ws || ws->dtype != XLA_FFI_DataType_U8 || ws->rank != 1 || !ws->data)
    return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT, "the last result must be a uint8 workspace");
  // attributes
  rrtmg_config cfg{};
  cfg.nx = static_cast<int>(nx);
  cfg.ny = static_cast<int>(ny);
  cfg.nk = static_cast<int>(nk);
  double v = 0.0;
  static const char *lw_gas[] = {"co2vmr", "n2ovmr", "ch4vmr", "cfc11vmr", "cfc12vmr"};
  float *gas[] = {&cfg.co2vmr, &cfg.n2ovmr, &cfg.ch4vmr, &cfg.cfc11vmr, &cfg.cfc12vmr};
  const int ngas = lw ? 5 : 3;
  for (int q = 0; q < ngas; ++q) {
    if (!attr_number(f->attrs, lw_gas[q], &v))
      return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT, std::string("missing attribute ") + lw_gas[q]);
    *gas[q] = static_cast<float>(v);
  }
  if (lw) {
    if (!attr_number(f->attrs, "p_top", &v))
      return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT, "missing attribute p_top");
    cfg.p_top = v;
  } else {
    if (!attr_number(f->attrs, "solcon", &v))
      return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT, "missing attribute solcon");
    cfg.solcon = static_cast<float>(v);
  }
  if (const char *missing = read_flags(f->attrs, cfg))
    return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT, std::string("missing attribute ") + missing);
  // device of the operands, the context, XLA's stream
  cudaPointerAttributes pa{};
  if (cudaPointerGetAttributes(&pa, t3d->data) != cudaSuccess || pa.type != cudaMemoryTypeDevice) {
    cudaGetLastError();
    return make_error(f, XLA_FFI_Error_Code_INVALID_ARGUMENT, "operands must be in device memory");
  }
  rrtmg_ctx *ctx = nullptr;
  std::string err;
  if (context_for(pa.device, &ctx, err) != RRTMG_OK) return make_error(f, XLA_FFI_Error_Code_INTERNAL, err);
  XLA_FFI_Stream_Get_Args sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.struct_size = sizeof(sa);
  sa.ctx = f->ctx;
  if (XLA_FFI_Error *e = f->api->XLA_FFI_Stream_Get(&sa)) return e;
  const size_t ws_bytes = static_cast<size_t>(ws->dims[0]);
  T in{};
  const float **pin = reinterpret_cast<const float **>(&in);
  for (int64_t i = 0; i < f->args.size; ++i) pin[i] = static_cast<const float *>(arg(f, i)->data);
  rrtmg_status st;
  if constexpr (std::is_same_v<T, rrtmg_lw_in>) {
    rrtmg_lw_out out{};
    float **po = reinterpret_cast<float **>(&out);
    for (int i = 0; i < n_out; ++i) po[i] = static_cast<float *>(ret(f, i)->data);
    st = rrtmg_lwrad_ws(ctx, &cfg, &in, &out, ws->data, ws_bytes, sa.stream);
  } else {
    rrtmg_sw_out out{};
    float **po = reinterpret_cast<float **>(&out);
    for (int i = 0; i < n_out; ++i) po[i] = static_cast<float *>(ret(f, i)->data);
    st = rrtmg_swrad_ws(ctx, &cfg, &in, &out, ws->data, ws_bytes, sa.stream);
  }
  if (st == RRTMG_OK) return nullptr;
  const XLA_FFI_Error_Code code = st == RRTMG_BAD_ARG              ? XLA_FFI_Error_Code_INVALID_ARGUMENT
                                  : st == RRTMG_UNSUPPORTED_OPTION ? XLA_FFI_Error_Code_UNIMPLEMENTED
                                                                   : XLA_FFI_Error_Code_INTERNAL;
  return make_error(f, code, rrtmg_last_error(ctx));
}

static_assert(sizeof(rrtmg_lw_in) == 20 * sizeof(const float *), "rrtmg_lw_in is 20 array pointers");
static_assert(sizeof(rrtmg_sw_in) == 25 * sizeof(const float *), "rrtmg_sw_in is 25 array pointers");
static_assert(sizeof(rrtmg_lw_out) == 17 * sizeof(float *), "rrtmg_lw_out is 17 array pointers");
static_assert(sizeof(rrtmg_sw_out) == 23 * sizeof(float *), "rrtmg_sw_out is 23 array pointers");

size_t workspace_bytes(int device, const rrtmg_config *cfg, bool lw) {
  rrtmg_ctx *ctx = nullptr;
  std::string err;
  if (context_for(device, &ctx, err) != RRTMG_OK) {
    rrtmg::create_error(RRTMG_BAD_ARG, err);
    return 0;
  }
  return lw ? rrtmg_lw_workspace_bytes(ctx, cfg) : rrtmg_sw_workspace_bytes(ctx, cfg);
}

}  // namespace

extern "C" XLA_FFI_Error *rrtmg_ffi_lwrad(XLA_FFI_CallFrame *call_frame) { return run<rrtmg_lw_in>(call_frame, true); }
extern "C" XLA_FFI_Error *rrtmg_ffi_swrad(XLA_FFI_CallFrame *call_frame) { return run<rrtmg_sw_in>(call_frame, false); }

extern "C" rrtmg_status rrtmg_ffi_set_table_blob(const char *path) {
  if (!path || !*path) return rrtmg::create_error(RRTMG_BAD_ARG, "null or empty table blob path");
  std::lock_guard<std::mutex> lk(g_mutex);
  g_blob = path;
  return RRTMG_OK;
}

extern "C" size_t rrtmg_ffi_lw_workspace_bytes(int device, const rrtmg_config *cfg) {
  return workspace_bytes(device, cfg, true);
}

extern "C" size_t rrtmg_ffi_sw_workspace_bytes(int device, const rrtmg_config *cfg) {
  return workspace_bytes(device, cfg, false);
}

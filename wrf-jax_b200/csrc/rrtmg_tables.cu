// Native reader of the reference's RRTMG data files: RRTMG_LW_DATA and
// RRTMG_SW_DATA (Fortran unformatted sequential files, big-endian, one record
// per band) parsed and reduced from 16 to the compressed g-points per band in
// binary32 (WRF's cmbgb), replacing the absorption tables of a table blob.
// Host code only.  The record layouts are those the reference's loaders read
// (src/wrf_jax/physics/module_ra_rrtmg_lw.py:554-950,
// module_ra_rrtmg_sw.py:800-1170); the reduction follows
// module_ra_rrtmg_common.py:530-789.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "../../include/rrtmg_tables.h"
#include "rrtmg_kernels.h"

namespace {

constexpr int kMG = 16;  // original g-points per band

struct Field {
  const char *name;
  char kind;        // 'r' binary32, 'i' int32
  int ndim;         // 0: scalar
  int shape[4];     // Fortran dimension extents, first fastest
};

struct Band {
  int band;
  std::vector<Field> fields;
};

// Record layouts, in file order (the Fortran READ lists of the reference's loaders).
const std::vector<Band> &lw_layout() {
  static const std::vector<Band> b = {
      {1, {{"fracrefao", 'r', 1, {16}}, {"fracrefbo", 'r', 1, {16}}, {"kao", 'r', 3, {5, 13, 16}},
           {"kbo", 'r', 3, {5, 47, 16}}, {"kao_mn2", 'r', 2, {19, 16}}, {"kbo_mn2", 'r', 2, {19, 16}},
           {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {2, {{"fracrefao", 'r', 1, {16}}, {"fracrefbo", 'r', 1, {16}}, {"kao", 'r', 3, {5, 13, 16}},
           {"kbo", 'r', 3, {5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {3, {{"fracrefao", 'r', 2, {16, 9}}, {"fracrefbo", 'r', 2, {16, 5}}, {"kao", 'r', 4, {9, 5, 13, 16}},
           {"kbo", 'r', 4, {5, 5, 47, 16}}, {"kao_mn2o", 'r', 3, {9, 19, 16}}, {"kbo_mn2o", 'r', 3, {5, 19, 16}},
           {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {4, {{"fracrefao", 'r', 2, {16, 9}}, {"fracrefbo", 'r', 2, {16, 5}}, {"kao", 'r', 4, {9, 5, 13, 16}},
           {"kbo", 'r', 4, {5, 5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {5, {{"fracrefao", 'r', 2, {16, 9}}, {"fracrefbo", 'r', 2, {16, 5}}, {"kao", 'r', 4, {9, 5, 13, 16}},
           {"kbo", 'r', 4, {5, 5, 47, 16}}, {"kao_mo3", 'r', 3, {9, 19, 16}}, {"ccl4o", 'r', 1, {16}},
           {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {6, {{"fracrefao", 'r', 1, {16}}, {"kao", 'r', 3, {5, 13, 16}}, {"kao_mco2", 'r', 2, {19, 16}},
           {"cfc11adjo", 'r', 1, {16}}, {"cfc12o", 'r', 1, {16}}, {"selfrefo", 'r', 2, {10, 16}},
           {"forrefo", 'r', 2, {4, 16}}}},
      {7, {{"fracrefao", 'r', 2, {16, 9}}, {"fracrefbo", 'r', 1, {16}}, {"kao", 'r', 4, {9, 5, 13, 16}},
           {"kbo", 'r', 3, {5, 47, 16}}, {"kao_mco2", 'r', 3, {9, 19, 16}}, {"kbo_mco2", 'r', 2, {19, 16}},
           {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {8, {{"fracrefao", 'r', 1, {16}}, {"fracrefbo", 'r', 1, {16}}, {"kao", 'r', 3, {5, 13, 16}},
           {"kbo", 'r', 3, {5, 47, 16}}, {"kao_mco2", 'r', 2, {19, 16}}, {"kbo_mco2", 'r', 2, {19, 16}},
           {"kao_mn2o", 'r', 2, {19, 16}}, {"kbo_mn2o", 'r', 2, {19, 16}}, {"kao_mo3", 'r', 2, {19, 16}},
           {"cfc12o", 'r', 1, {16}}, {"cfc22adjo", 'r', 1, {16}}, {"selfrefo", 'r', 2, {10, 16}},
           {"forrefo", 'r', 2, {4, 16}}}},
      {9, {{"fracrefao", 'r', 2, {16, 9}}, {"fracrefbo", 'r', 1, {16}}, {"kao", 'r', 4, {9, 5, 13, 16}},
           {"kbo", 'r', 3, {5, 47, 16}}, {"kao_mn2o", 'r', 3, {9, 19, 16}}, {"kbo_mn2o", 'r', 2, {19, 16}},
           {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {10, {{"fracrefao", 'r', 1, {16}}, {"fracrefbo", 'r', 1, {16}}, {"kao", 'r', 3, {5, 13, 16}},
            {"kbo", 'r', 3, {5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {11, {{"fracrefao", 'r', 1, {16}}, {"fracrefbo", 'r', 1, {16}}, {"kao", 'r', 3, {5, 13, 16}},
            {"kbo", 'r', 3, {5, 47, 16}}, {"kao_mo2", 'r', 2, {19, 16}}, {"kbo_mo2", 'r', 2, {19, 16}},
            {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {12, {{"fracrefao", 'r', 2, {16, 9}}, {"kao", 'r', 4, {9, 5, 13, 16}}, {"selfrefo", 'r', 2, {10, 16}},
            {"forrefo", 'r', 2, {4, 16}}}},
      {13, {{"fracrefao", 'r', 2, {16, 9}}, {"fracrefbo", 'r', 1, {16}}, {"kao", 'r', 4, {9, 5, 13, 16}},
            {"kao_mco2", 'r', 3, {9, 19, 16}}, {"kao_mco", 'r', 3, {9, 19, 16}}, {"kbo_mo3", 'r', 2, {19, 16}},
            {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {14, {{"fracrefao", 'r', 1, {16}}, {"fracrefbo", 'r', 1, {16}}, {"kao", 'r', 3, {5, 13, 16}},
            {"kbo", 'r', 3, {5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {15, {{"fracrefao", 'r', 2, {16, 9}}, {"kao", 'r', 4, {9, 5, 13, 16}}, {"kao_mn2", 'r', 3, {9, 19, 16}},
            {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
      {16, {{"fracrefao", 'r', 2, {16, 9}}, {"fracrefbo", 'r', 1, {16}}, {"kao", 'r', 4, {9, 5, 13, 16}},
            {"kbo", 'r', 3, {5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}}}},
  };
  return b;
}

const std::vector<Band> &sw_layout() {
  static const std::vector<Band> b = {
      {16, {{"rayl", 'r', 0, {}}, {"strrat1", 'r', 0, {}}, {"layreffr", 'i', 0, {}}, {"kao", 'r', 4, {9, 5, 13, 16}},
            {"kbo", 'r', 3, {5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {3, 16}},
            {"sfluxrefo", 'r', 1, {16}}}},
      {17, {{"rayl", 'r', 0, {}}, {"strrat", 'r', 0, {}}, {"layreffr", 'i', 0, {}}, {"kao", 'r', 4, {9, 5, 13, 16}},
            {"kbo", 'r', 4, {5, 5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}},
            {"sfluxrefo", 'r', 2, {16, 5}}}},
      {18, {{"rayl", 'r', 0, {}}, {"strrat", 'r', 0, {}}, {"layreffr", 'i', 0, {}}, {"kao", 'r', 4, {9, 5, 13, 16}},
            {"kbo", 'r', 3, {5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {3, 16}},
            {"sfluxrefo", 'r', 2, {16, 9}}}},
      {19, {{"rayl", 'r', 0, {}}, {"strrat", 'r', 0, {}}, {"layreffr", 'i', 0, {}}, {"kao", 'r', 4, {9, 5, 13, 16}},
            {"kbo", 'r', 3, {5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {3, 16}},
            {"sfluxrefo", 'r', 2, {16, 9}}}},
      {20, {{"rayl", 'r', 0, {}}, {"layreffr", 'i', 0, {}}, {"absch4o", 'r', 1, {16}}, {"kao", 'r', 3, {5, 13, 16}},
            {"kbo", 'r', 3, {5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}},
            {"sfluxrefo", 'r', 1, {16}}}},
      {21, {{"rayl", 'r', 0, {}}, {"strrat", 'r', 0, {}}, {"layreffr", 'i', 0, {}}, {"kao", 'r', 4, {9, 5, 13, 16}},
            {"kbo", 'r', 4, {5, 5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {4, 16}},
            {"sfluxrefo", 'r', 2, {16, 9}}}},
      {22, {{"rayl", 'r', 0, {}}, {"strrat", 'r', 0, {}}, {"layreffr", 'i', 0, {}}, {"kao", 'r', 4, {9, 5, 13, 16}},
            {"kbo", 'r', 3, {5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {3, 16}},
            {"sfluxrefo", 'r', 2, {16, 9}}}},
      {23, {{"raylo", 'r', 1, {16}}, {"givfac", 'r', 0, {}}, {"layreffr", 'i', 0, {}}, {"kao", 'r', 3, {5, 13, 16}},
            {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {3, 16}}, {"sfluxrefo", 'r', 1, {16}}}},
      {24, {{"raylao", 'r', 2, {16, 9}}, {"raylbo", 'r', 1, {16}}, {"strrat", 'r', 0, {}}, {"layreffr", 'i', 0, {}},
            {"abso3ao", 'r', 1, {16}}, {"abso3bo", 'r', 1, {16}}, {"kao", 'r', 4, {9, 5, 13, 16}},
            {"kbo", 'r', 3, {5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}}, {"forrefo", 'r', 2, {3, 16}},
            {"sfluxrefo", 'r', 2, {16, 9}}}},
      {25, {{"raylo", 'r', 1, {16}}, {"layreffr", 'i', 0, {}}, {"abso3ao", 'r', 1, {16}}, {"abso3bo", 'r', 1, {16}},
            {"kao", 'r', 3, {5, 13, 16}}, {"sfluxrefo", 'r', 1, {16}}}},
      {26, {{"raylo", 'r', 1, {16}}, {"sfluxrefo", 'r', 1, {16}}}},
      {27, {{"raylo", 'r', 1, {16}}, {"scalekur", 'r', 0, {}}, {"layreffr", 'i', 0, {}}, {"kao", 'r', 3, {5, 13, 16}},
            {"kbo", 'r', 3, {5, 47, 16}}, {"sfluxrefo", 'r', 1, {16}}}},
      {28, {{"rayl", 'r', 0, {}}, {"strrat", 'r', 0, {}}, {"layreffr", 'i', 0, {}}, {"kao", 'r', 4, {9, 5, 13, 16}},
            {"kbo", 'r', 4, {5, 5, 47, 16}}, {"sfluxrefo", 'r', 2, {16, 5}}}},
      {29, {{"rayl", 'r', 0, {}}, {"layreffr", 'i', 0, {}}, {"absh2oo", 'r', 1, {16}}, {"absco2o", 'r', 1, {16}},
            {"kao", 'r', 3, {5, 13, 16}}, {"kbo", 'r', 3, {5, 47, 16}}, {"selfrefo", 'r', 2, {10, 16}},
            {"forrefo", 'r', 2, {4, 16}}, {"sfluxrefo", 'r', 1, {16}}}},
  };
  return b;
}

// One blob entry: dtype code (0 f32, 1 i32, 2 f64, 3 u64), shape, raw little-endian bytes.
struct Entry {
  uint32_t dtype = 0;
  std::vector<uint32_t> shape;
  std::vector<unsigned char> bytes;
};
using Blob = std::map<std::string, Entry>;

uint32_t be32(const unsigned char *p) {
  return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | uint32_t(p[3]);
}

bool read_file(const char *path, std::vector<unsigned char> &out, std::string &err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    err = std::string("cannot open ") + path;
    return false;
  }
  out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return true;
}

bool parse_blob(const std::vector<unsigned char> &raw, Blob &blob, std::string &err) {
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
  for (uint32_t i = 0; i < count; ++i) {
    const size_t pos = 16 + 88ull * i;
    if (pos + 88 > raw.size()) {
      err = "truncated table blob header";
      return false;
    }
    char name[49] = {0};
    std::memcpy(name, raw.data() + pos, 48);
    Entry e;
    uint32_t ndim, shape[4];
    uint64_t offset, nbytes;
    std::memcpy(&e.dtype, raw.data() + pos + 48, 4);
    std::memcpy(&ndim, raw.data() + pos + 52, 4);
    std::memcpy(shape, raw.data() + pos + 56, 16);
    std::memcpy(&offset, raw.data() + pos + 72, 8);
    std::memcpy(&nbytes, raw.data() + pos + 80, 8);
    if (ndim > 4 || e.dtype > 3 || offset > raw.size() || nbytes > raw.size() - offset) {
      err = std::string("bad table entry ") + name;
      return false;
    }
    // nbytes must equal the element size (f32, i32: 4; f64, u64: 8) times the extents
    uint64_t count = 1;
    bool overflow = false;
    for (uint32_t d = 0; d < ndim; ++d) {
      if (shape[d] != 0 && count > UINT64_MAX / 8 / shape[d]) overflow = true;
      count *= shape[d];
    }
    if (overflow || count * (e.dtype >= 2 ? 8u : 4u) != nbytes) {
      err = std::string("table entry size does not match its shape and type: ") + name;
      return false;
    }
    e.shape.assign(shape, shape + ndim);
    e.bytes.assign(raw.data() + offset, raw.data() + offset + nbytes);
    blob[name] = std::move(e);
  }
  return true;
}

// The blob layout of the package's table writer: header, 88-byte entries in
// name order, each array at a 256-byte boundary.
std::vector<unsigned char> write_blob(const Blob &blob) {
  const uint32_t count = static_cast<uint32_t>(blob.size());
  size_t data_start = 16 + 88ull * count;
  data_start = (data_start + 255) / 256 * 256;
  std::vector<unsigned char> body, head(16 + 88ull * count, 0);
  std::memcpy(head.data(), "RRTMGB2\0", 8);
  const uint32_t version = 1;
  std::memcpy(head.data() + 8, &version, 4);
  std::memcpy(head.data() + 12, &count, 4);
  size_t i = 0;
  for (const auto &kv : blob) {
    body.resize((body.size() + 255) / 256 * 256, 0);
    const uint64_t offset = data_start + body.size(), nbytes = kv.second.bytes.size();
    body.insert(body.end(), kv.second.bytes.begin(), kv.second.bytes.end());
    unsigned char *h = head.data() + 16 + 88 * i++;
    std::strncpy(reinterpret_cast<char *>(h), kv.first.c_str(), 47);
    const uint32_t ndim = static_cast<uint32_t>(kv.second.shape.size());
    uint32_t shape[4] = {1, 1, 1, 1};
    for (uint32_t d = 0; d < ndim; ++d) shape[d] = kv.second.shape[d];
    std::memcpy(h + 48, &kv.second.dtype, 4);
    std::memcpy(h + 52, &ndim, 4);
    std::memcpy(h + 56, shape, 16);
    std::memcpy(h + 72, &offset, 8);
    std::memcpy(h + 80, &nbytes, 8);
  }
  head.resize(data_start, 0);
  head.insert(head.end(), body.begin(), body.end());
  return head;
}

template <typename T>
Entry make_entry(uint32_t dtype, const std::vector<uint32_t> &shape, const std::vector<T> &v) {
  Entry e;
  e.dtype = dtype;
  e.shape = shape;
  e.bytes.resize(v.size() * sizeof(T));
  std::memcpy(e.bytes.data(), v.data(), e.bytes.size());
  return e;
}

template <typename T>
bool entry_values(const Blob &blob, const std::string &name, std::vector<T> &out, std::string &err) {
  auto it = blob.find(name);
  if (it == blob.end()) {
    err = "base blob has no " + name;
    return false;
  }
  out.resize(it->second.bytes.size() / sizeof(T));
  std::memcpy(out.data(), it->second.bytes.data(), out.size() * sizeof(T));
  return true;
}

// A raw record field: values in Fortran order.
struct Raw {
  const Field *f;
  std::vector<float> r;
  int32_t i = 0;
};

// g-point groups of one band: [a, b) ranges of original g-points per
// compressed g-point, with the binary32 weights (module_ra_rrtmg_common.py
// cmbgb).
struct Groups {
  std::vector<int> a, b;
  const float *w;  // 16 weights of the band
};

// Sequential binary32 sum over a group, weighted or not, of x(k) for k in [a, b).
template <typename Get>
float group_sum(const Groups &g, int igc, bool weighted, Get x) {
  float acc = 0.0f;
  for (int k = g.a[igc]; k < g.b[igc]; ++k) acc = acc + (weighted ? x(k) * g.w[k] : x(k));
  return acc;
}

void compress(const std::vector<Raw> &band, const Groups &g, const std::string &prefix, Blob &out) {
  const int ngc = static_cast<int>(g.a.size());
  for (const Raw &raw : band) {
    const Field &f = *raw.f;
    const std::string name = f.name;
    if (f.ndim == 0) {
      if (f.kind == 'i')
        out[prefix + "." + name] = make_entry<int32_t>(1, {1}, {raw.i});
      else
        out[prefix + "." + name] = make_entry<float>(0, {1}, {raw.r[0]});
      continue;
    }
    std::string base = name;
    if (name.rfind("kao_", 0) == 0 || name.rfind("kbo_", 0) == 0)
      base = name.substr(0, 2) + name.substr(3);
    else if (name.back() == 'o' && name != "raylo")
      base = name.substr(0, name.size() - 1);
    const bool gfirst_plain = name == "fracrefao" || name == "fracrefbo" || name == "sfluxrefo";
    static const char *kFirstWeighted[] = {"ccl4o",   "cfc11adjo", "cfc12o",  "cfc22adjo", "absch4o", "abso3ao",
                                           "abso3bo", "absh2oo",   "absco2o", "raylo",     "raylao",  "raylbo"};
    bool gfirst_weighted = false;
    for (const char *n : kFirstWeighted) gfirst_weighted |= name == n;
    if (gfirst_plain || gfirst_weighted) {
      // g-point is the first (fastest) Fortran index: out (ngc, rest) in C order
      const int rest = f.ndim == 2 ? f.shape[1] : 1;
      std::vector<float> v(static_cast<size_t>(ngc) * rest);
      for (int igc = 0; igc < ngc; ++igc)
        for (int r = 0; r < rest; ++r)
          v[static_cast<size_t>(igc) * rest + r] =
              group_sum(g, igc, gfirst_weighted, [&](int k) { return raw.r[k + kMG * r]; });
      std::vector<uint32_t> shape = {static_cast<uint32_t>(ngc)};
      if (f.ndim == 2) shape.push_back(static_cast<uint32_t>(rest));
      out[prefix + "." + (name == "raylo" ? std::string("rayl") : base)] = make_entry<float>(0, shape, v);
      continue;
    }
    // g-point is the last (slowest) Fortran index
    size_t inner = 1;
    for (int d = 0; d + 1 < f.ndim; ++d) inner *= f.shape[d];
    auto reduced = [&](size_t r, int igc) {
      return group_sum(g, igc, true, [&](int k) { return raw.r[r + inner * k]; });
    };
    if (name == "kao" || name == "kbo") {
      // (js, jt, jp, g) Fortran -> rows (jp * nt + jt) * ns + js, g columns
      const int ns = f.ndim == 4 ? f.shape[0] : 1;
      const int nt = f.shape[f.ndim - 3], np_ = f.shape[f.ndim - 2];
      std::vector<float> v(static_cast<size_t>(np_) * nt * ns * ngc);
      for (int jp = 0; jp < np_; ++jp)
        for (int jt = 0; jt < nt; ++jt)
          for (int js = 0; js < ns; ++js) {
            const size_t r = js + static_cast<size_t>(ns) * (jt + static_cast<size_t>(nt) * jp);
            const size_t row = (static_cast<size_t>(jp) * nt + jt) * ns + js;
            for (int igc = 0; igc < ngc; ++igc) v[row * ngc + igc] = reduced(r, igc);
          }
      out[prefix + "." + base] = make_entry<float>(0, {static_cast<uint32_t>(np_ * nt * ns), static_cast<uint32_t>(ngc)}, v);
      continue;
    }
    // minor / continuum tables: C order (d0, ..., ngc) of the Fortran extents
    std::vector<uint32_t> shape;
    for (int d = 0; d + 1 < f.ndim; ++d) shape.push_back(static_cast<uint32_t>(f.shape[d]));
    shape.push_back(static_cast<uint32_t>(ngc));
    std::vector<float> v(inner * ngc);
    // C-order index (i0, ..., i_{n-2}, igc) of the Fortran element (i0, ..., i_{n-2})
    const int nd = f.ndim - 1;
    std::vector<int> idx(nd, 0);
    for (size_t c = 0; c < inner; ++c) {
      size_t rem = c, r = 0, stride = 1;
      for (int d = nd - 1; d >= 0; --d) {
        idx[d] = static_cast<int>(rem % f.shape[d]);
        rem /= f.shape[d];
      }
      for (int d = 0; d < nd; ++d) {
        r += stride * idx[d];
        stride *= f.shape[d];
      }
      for (int igc = 0; igc < ngc; ++igc) v[c * ngc + igc] = reduced(r, igc);
    }
    out[prefix + "." + base] = make_entry<float>(0, shape, v);
  }
}

bool read_bands(const char *path, const std::vector<Band> &layout, const char *side, int first_band,
                const Blob &base, Blob &out, std::string &err) {
  std::vector<unsigned char> raw;
  if (!read_file(path, raw, err)) return false;
  std::vector<int32_t> ngc, ngs, ngn;
  std::vector<float> rwgt;
  const std::string s = side;
  if (!entry_values(base, s + ".ngc", ngc, err) || !entry_values(base, s + ".ngs", ngs, err) ||
      !entry_values(base, s + ".ngn", ngn, err) || !entry_values(base, s + ".rwgt", rwgt, err))
    return false;
  if (ngc.size() != layout.size() || ngs.size() != layout.size() || rwgt.size() != layout.size() * kMG) {
    err = "g-point maps of the base blob do not match the band count";
    return false;
  }
  size_t pos = 0;
  for (const Band &band : layout) {
    if (pos + 4 > raw.size()) {
      err = std::string(path) + ": truncated before band " + std::to_string(band.band);
      return false;
    }
    const uint32_t n = be32(raw.data() + pos);
    if (pos + 8 + static_cast<size_t>(n) > raw.size() || be32(raw.data() + pos + 4 + n) != n) {
      err = std::string(path) + ": bad record markers for band " + std::to_string(band.band);
      return false;
    }
    const unsigned char *body = raw.data() + pos + 4;
    size_t off = 0;
    std::vector<Raw> fields;
    for (const Field &f : band.fields) {
      size_t count = 1;
      for (int d = 0; d < f.ndim; ++d) count *= f.shape[d];
      if (off + 4 * count > n) {
        err = std::string(path) + ": band " + std::to_string(band.band) + " record too short";
        return false;
      }
      Raw r;
      r.f = &f;
      if (f.kind == 'i') {
        r.i = static_cast<int32_t>(be32(body + off));
      } else {
        r.r.resize(count);
        for (size_t e = 0; e < count; ++e) {
          const uint32_t u = be32(body + off + 4 * e);
          std::memcpy(&r.r[e], &u, 4);
        }
      }
      off += 4 * count;
      fields.push_back(std::move(r));
    }
    if (off != n) {
      err = std::string(path) + ": band " + std::to_string(band.band) + " record has extra bytes";
      return false;
    }
    pos += 8 + n;
    // groups of this band (ngs: cumulative compressed counts; ngn: originals per compressed point)
    const int ib = band.band - first_band;
    Groups g;
    g.w = rwgt.data() + ib * kMG;
    int start = ib == 0 ? 0 : ngs[ib - 1], k = 0;
    for (int igc = 0; igc < ngc[ib]; ++igc) {
      const int cnt = ngn[start + igc];
      g.a.push_back(k);
      g.b.push_back(k + cnt);
      k += cnt;
    }
    if (k != kMG) {
      err = "g-point groups of band " + std::to_string(band.band) + " do not cover 16 points";
      return false;
    }
    compress(fields, g, s + std::to_string(band.band), out);
  }
  if (pos != raw.size()) {
    err = std::string(path) + ": trailing bytes after the last band";
    return false;
  }
  return true;
}

bool blob_with_data(const char *base_path, const char *lw_path, const char *sw_path, std::vector<unsigned char> &out,
                    std::string &err) {
  std::vector<unsigned char> raw;
  Blob blob;
  if (!read_file(base_path, raw, err) || !parse_blob(raw, blob, err)) return false;
  Blob tables;
  if (!read_bands(lw_path, lw_layout(), "lw", 1, blob, tables, err)) return false;
  if (!read_bands(sw_path, sw_layout(), "sw", 16, blob, tables, err)) return false;
  for (auto &kv : tables) blob[kv.first] = std::move(kv.second);
  out = write_blob(blob);
  return true;
}

}  // namespace

extern "C" rrtmg_status rrtmg_blob_with_wrf_data(const char *base_blob_path, const char *lw_data_path,
                                                 const char *sw_data_path, const char *out_blob_path) {
  if (!base_blob_path || !lw_data_path || !sw_data_path || !out_blob_path)
    return rrtmg::create_error(RRTMG_BAD_ARG, "null path");
  std::vector<unsigned char> blob;
  std::string err;
  if (!blob_with_data(base_blob_path, lw_data_path, sw_data_path, blob, err))
    return rrtmg::create_error(RRTMG_BAD_ARG, err);
  std::ofstream f(out_blob_path, std::ios::binary);
  if (!f || !f.write(reinterpret_cast<const char *>(blob.data()), static_cast<std::streamsize>(blob.size())))
    return rrtmg::create_error(RRTMG_BAD_ARG, std::string("cannot write ") + out_blob_path);
  return RRTMG_OK;
}

extern "C" rrtmg_status rrtmg_create_with_wrf_data(const char *base_blob_path, const char *lw_data_path,
                                                   const char *sw_data_path, int device, rrtmg_ctx **out) {
  if (!base_blob_path || !lw_data_path || !sw_data_path || !out)
    return rrtmg::create_error(RRTMG_BAD_ARG, "null path or output pointer");
  std::vector<unsigned char> blob;
  std::string err;
  if (!blob_with_data(base_blob_path, lw_data_path, sw_data_path, blob, err))
    return rrtmg::create_error(RRTMG_BAD_ARG, err);
  return rrtmg_create_from_memory(blob.data(), blob.size(), device, out);
}

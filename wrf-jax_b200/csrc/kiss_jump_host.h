// Host-side construction of KISS jumps (include after the KissJump type).
//
// The McICA stream of a column (module_ra_rrtmg_common.py:964-1064) is
// consumed in (subcolumn, layer) order after `skip` discarded draws, so
// subcolumn g starts at draw skip + g * nlay.  kiss_jumps builds the jumps of
// all subcolumns by composition instead of stepping each one from zero: the
// LCG is an affine map of Z/2^32, the xorshift a linear map of GF(2)^32 (kept
// as the images of the 32 unit vectors), and both compose exactly, so
// J(skip + (g + 1) * nlay) = step^nlay o J(skip + g * nlay).  The
// multiply-with-carry generators jump by a^(k-2) mod (a * 2^16 - 1), a modular
// power per subcolumn.  Every result is integer arithmetic, identical to
// stepping the generators k times.
#pragma once

#include <cstdint>

namespace rrtmg {

namespace kiss_detail {

inline uint64_t powmod(uint64_t a, uint64_t e, uint64_t m) {
  uint64_t r = 1 % m, b = a % m;
  while (e) {
    if (e & 1) r = (r * b) % m;
    b = (b * b) % m;
    e >>= 1;
  }
  return r;
}

// One step of each of the two linear generators, as maps.
struct LinearMaps {
  uint32_t mul, add;  // LCG: x -> mul * x + add
  uint32_t xs[32];    // xorshift: images of the unit vectors
};

inline LinearMaps identity_maps() {
  LinearMaps m;
  m.mul = 1u;
  m.add = 0u;
  for (int b = 0; b < 32; ++b) m.xs[b] = 1u << b;
  return m;
}

inline uint32_t xs_apply(const uint32_t *images, uint32_t v) {
  uint32_t acc = 0;
  for (int b = 0; b < 32; ++b)
    if ((v >> b) & 1u) acc ^= images[b];
  return acc;
}

// a o b (apply b first)
inline LinearMaps compose(const LinearMaps &a, const LinearMaps &b) {
  LinearMaps c;
  c.mul = a.mul * b.mul;
  c.add = a.mul * b.add + a.add;
  for (int q = 0; q < 32; ++q) c.xs[q] = xs_apply(a.xs, b.xs[q]);
  return c;
}

inline LinearMaps one_step() {
  LinearMaps m;
  m.mul = 69069u;
  m.add = 1327217885u;
  for (int b = 0; b < 32; ++b) {
    uint32_t x = 1u << b;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    m.xs[b] = x;
  }
  return m;
}

inline LinearMaps power(uint64_t k) {
  LinearMaps result = identity_maps(), base = one_step();
  while (k) {
    if (k & 1) result = compose(base, result);
    base = compose(base, base);
    k >>= 1;
  }
  return result;
}

}  // namespace kiss_detail

// Jumps of nsub subcolumns of nlay draws each after `skip` draws.
inline void kiss_jumps(uint64_t skip, int nlay, int nsub, KissJump *out) {
  using namespace kiss_detail;
  const LinearMaps stride = power(static_cast<uint64_t>(nlay));
  LinearMaps cur = power(skip);
  for (int g = 0; g < nsub; ++g) {
    const uint64_t k = skip + static_cast<uint64_t>(g) * static_cast<uint64_t>(nlay);
    KissJump J{};
    J.lcg_mul = cur.mul;
    J.lcg_add = cur.add;
    for (int b = 0; b < 32; ++b) J.xs[b] = cur.xs[b];
    const uint64_t e = k >= 2 ? k - 2 : 0;
    J.mwc3_pow = static_cast<uint32_t>(powmod(18000, e, 18000ull * 65536 - 1));
    J.mwc4_pow = static_cast<uint32_t>(powmod(30903, e, 30903ull * 65536 - 1));
    J.steps = static_cast<uint32_t>(k);
    out[g] = J;
    cur = compose(stride, cur);
  }
}

}  // namespace rrtmg

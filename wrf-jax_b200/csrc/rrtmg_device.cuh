// Device-side data structures and numerics shared by the RRTMG kernels.
//
// Arithmetic contract: every statement is one IEEE binary32 operation with
// round-to-nearest, in the reference's order, and no fused multiply-add (the
// library is compiled with -fmad=false, -prec-div=true, -prec-sqrt=true).  This
// is the WRF default-REAL rounding WRF-JAX reproduces
// (src/wrf_jax/core/real_arithmetic.py:194-212,
// src/wrf_jax/physics/module_ra_rrtmg_lw.py:51-105).  logf/expf follow glibc
// 2.39's published binary64 algorithms so the device agrees bit for bit with
// the host libm the reference emulates (src/wrf_jax/core/wrf_math.py:120-280).
#pragma once

#include <cstdint>

namespace rrtmg {

constexpr int kLwBands = 16;
constexpr int kLwGpts = 140;
constexpr int kSwBands = 14;
constexpr int kSwGpts = 112;
constexpr int kMaxLay = 128;      // layers per column the kernels accept
constexpr int kMaxBuf = 40;       // LW buffer layers above the model top
constexpr int kLwMaskWords = 5;   // ceil(140 / 32)
constexpr int kSwMaskWords = 4;   // ceil(112 / 32)

struct LwBand {
  const float *fracrefa, *fracrefb, *ka, *kb, *selfref, *forref;
  const float *ka_mn2, *kb_mn2, *ka_mn2o, *kb_mn2o, *ka_mo3, *kb_mo3;
  const float *ka_mco2, *kb_mco2, *ka_mco, *ka_mo2, *kb_mo2;
  const float *ccl4, *cfc11adj, *cfc12, *cfc22adj;
  int ka_rows, kb_rows;
};

struct SwBand {
  const float *ka, *kb, *selfref, *forref, *sfluxref, *rayla, *raylb, *rayl_g;
  const float *absch4, *abso3a, *abso3b, *absh2o, *absco2;
  float rayl, strrat, strrat1, givfac, scalekur;
  int layreffr, forref_rows, sflux_cols;
};

// All lookup tables, as device pointers into one contiguous allocation.
struct Tables {
  LwBand lw[kLwBands];
  SwBand sw[kSwBands];
  // longwave reference atmosphere, Planck and cloud tables, Pade tables
  const float *lw_preflog, *lw_tref, *chi_mls, *totplnk;
  const float *absice3, *absliq1;
  const float *lw_pade_tau, *lw_pade_exp, *lw_pade_tfn;
  float lw_bpade;
  int lw_ntbl;
  // shortwave reference atmosphere, cloud optics, Pade table
  const float *sw_preflog, *sw_tref;
  const float *extliq1, *ssaliq1, *asyliq1, *extice3, *ssaice3, *asyice3, *fdlice3;
  const float *sw_pade_exp;
  float sw_bpade;
  int sw_ntbl;
  // shared
  const float *retab, *pprof, *tprof;
  int nprof;
  float o3wrk[31], ppwrkh[32];
  // glibc logf / expf data
  const double *logf_tab;           // (16, 2): 1/c, log c
  double logf_ln2, logf_a0, logf_a1, logf_a2;
  const unsigned long long *expf_tab;  // 32 entries
  double expf_invln2n, expf_c0, expf_c1, expf_c2;
};

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// JAX gather semantics for a computed row: a negative index wraps once, then
// the index is clamped into the table.
__device__ __forceinline__ int jrow(int r, int n) {
  if (r < 0) r += n;
  return clampi(r, 0, n - 1);
}

__device__ __forceinline__ float ld(const float *p) { return __ldg(p); }

__device__ __forceinline__ float interpf(float lo, float hi, float f) { return lo + f * (hi - lo); }

// Pa -> hPa: the reference's binary64 quotient rounded once to binary32
// (module_ra_rrtmg_common.py:70-82), identical to a binary32 division.
__device__ __forceinline__ float pa_to_hpa(float p) { return p / 100.0f; }

// First layer (bottom-up) whose heating rate the FP64 mode forms in binary64:
// the fifth-highest model layer (nk - 5) and every layer above it.
__host__ __device__ __forceinline__ int fp64_first_layer(int nk) { return nk > 5 ? nk - 5 : 0; }

// FP64 mode's heating rate of a layer (LW lw:5702-5712, SW sw:2285-2301):
// the net fluxes up - dn at the layer's bottom (0) and top (1), their
// difference and the division by the pressure thickness are binary64
// operations on the binary32 fluxes and level pressures, rounded once.
__device__ __forceinline__ float heating64(float heatfac, float up0, float dn0, float up1, float dn1, float plev0,
                                           float plev1) {
  const double f0 = static_cast<double>(up0) - static_cast<double>(dn0);
  const double f1 = static_cast<double>(up1) - static_cast<double>(dn1);
  const double dp = static_cast<double>(plev0) - static_cast<double>(plev1);
  return static_cast<float>(static_cast<double>(heatfac) * (f0 - f1) / dp);
}

// glibc 2.39 logf (e_logf.c, FMA build), including its special inputs.
__device__ __forceinline__ float glibc_logf(const Tables &T, float x) {
  uint32_t ix = __float_as_uint(x);
  if (ix == 0x3f800000u) return 0.0f;
  if (ix - 0x00800000u >= 0x7f800000u - 0x00800000u) {
    if (ix * 2u == 0u) return __int_as_float(0xff800000);          // log(+-0) = -inf
    if (ix == 0x7f800000u) return x;                                // log(inf) = inf
    if ((ix & 0x80000000u) || ix * 2u >= 0xff000000u) return __int_as_float(0x7fc00000);  // negative or NaN
    ix = __float_as_uint(x * 8388608.0f) - (23u << 23);             // subnormal: normalize
  }
  const uint32_t tmp = ix - 0x3f330000u;
  const int i = (tmp >> 19) & 15;
  const int k = static_cast<int32_t>(tmp) >> 23;
  const uint32_t iz = ix - (tmp & 0xff800000u);
  const double z = static_cast<double>(__uint_as_float(iz));
  const double invc = __ldg(T.logf_tab + 2 * i);
  const double logc = __ldg(T.logf_tab + 2 * i + 1);
  const double r = __fma_rn(z, invc, -1.0);
  const double y0 = __dadd_rn(logc, __dmul_rn(static_cast<double>(k), T.logf_ln2));
  const double r2 = __dmul_rn(r, r);
  double y = __fma_rn(T.logf_a1, r, T.logf_a2);
  y = __fma_rn(T.logf_a0, r2, y);
  y = __fma_rn(y, r2, __dadd_rn(y0, r));
  return __double2float_rn(y);
}

// glibc 2.39 expf (e_expf.c, FMA build), including its |x| >= 88 branch.
__device__ __forceinline__ float glibc_expf(const Tables &T, float x) {
  const uint32_t ux = __float_as_uint(x);
  if (((ux >> 20) & 0x7ffu) >= (0x42b00000u >> 20)) {   // |x| >= 88 or not finite
    if (ux == 0xff800000u) return 0.0f;                   // exp(-inf) = 0
    if (((ux >> 20) & 0x7ffu) >= (0x7f800000u >> 20)) return x + x;  // inf or NaN
    if (x > 88.7228317f) return __int_as_float(0x7f800000);         // overflow
    if (x < -103.972076f) return 0.0f;                               // underflow
  }
  const double xd = static_cast<double>(x);
  const double z = __dmul_rn(T.expf_invln2n, xd);
  const double kd = rint(z);
  const long long ki = static_cast<long long>(kd);
  const double r = __dsub_rn(z, kd);
  unsigned long long t = __ldg(T.expf_tab + (ki & 31));
  t += static_cast<unsigned long long>(ki) << 47;
  const double s = __longlong_as_double(static_cast<long long>(t));
  const double zz = __fma_rn(T.expf_c0, r, T.expf_c1);
  const double r2 = __dmul_rn(r, r);
  double y = __fma_rn(T.expf_c2, r, 1.0);
  y = __fma_rn(zz, r2, y);
  return __double2float_rn(__dmul_rn(y, s));
}

// KISS generator step (module_ra_rrtmg_common.py:976-997).
struct Kiss {
  uint32_t s1, s2, s3, s4;
  __device__ __forceinline__ float next() {
    s1 = 69069u * s1 + 1327217885u;
    uint32_t x = s2;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    s2 = x;
    s3 = 18000u * (s3 & 65535u) + (s3 >> 16);
    s4 = 30903u * (s4 & 65535u) + (s4 >> 16);
    const uint32_t kiss = s1 + s2 + (s3 << 16) + s4;
    const float k = static_cast<float>(static_cast<int32_t>(kiss));
    return k * 2.328306e-10f + 0.5f;
  }
};

// Jump of the four KISS recurrences by a fixed number of steps (computed on
// the host): LCG affine map, xorshift GF(2) matrix (column images of the 32
// unit vectors) and the multiply-with-carry powers a^(k-2) mod (a*2^16-1).
struct KissJump {
  uint32_t lcg_mul, lcg_add;
  uint32_t xs[32];
  uint32_t mwc3_pow, mwc4_pow;
  uint32_t steps;  // k
  uint32_t pad;
};

__device__ __forceinline__ uint32_t mwc_step(uint32_t v, uint32_t a) { return a * (v & 65535u) + (v >> 16); }

__device__ __forceinline__ uint32_t mwc_jump(uint32_t v, uint32_t a, uint32_t pw, uint32_t k) {
  if (k == 0) return v;
  const uint32_t once = mwc_step(v, a);
  if (k == 1) return once;
  const uint32_t twice = mwc_step(once, a);
  const uint64_t m = static_cast<uint64_t>(a) * 65536ull - 1ull;
  if (twice == static_cast<uint32_t>(m)) return twice;
  return static_cast<uint32_t>((static_cast<uint64_t>(twice) * pw) % m);
}

__device__ __forceinline__ Kiss kiss_jump(Kiss s, const KissJump &J) {
  Kiss o;
  o.s1 = J.lcg_mul * s.s1 + J.lcg_add;
  uint32_t acc = 0;
#pragma unroll
  for (int b = 0; b < 32; ++b)
    if ((s.s2 >> b) & 1u) acc ^= J.xs[b];
  o.s2 = acc;
  o.s3 = mwc_jump(s.s3, 18000u, J.mwc3_pow, J.steps);
  o.s4 = mwc_jump(s.s4, 30903u, J.mwc4_pow, J.steps);
  return o;
}

__device__ __forceinline__ uint32_t kiss_seed(float pmid) {
  const float frac = pmid - truncf(pmid);
  return static_cast<uint32_t>(static_cast<int32_t>(frac * 1000000000.0f));
}

}  // namespace rrtmg

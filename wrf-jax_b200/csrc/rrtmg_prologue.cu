// Radiation prologue on the GPU: WRF cal_cldfra1 cloud fraction, the cosine
// of the solar zenith angle and the CAM ozone climatology, one thread per
// column walking its levels (src/wrf_jax/runtime.py:7733-7766 computes them
// before its RRTMG calls).  Plus the host helpers for the per-step scalars.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "../../include/rrtmg_prologue.h"
#include "rrtmg_kernels.h"

namespace rrtmg {
namespace {

constexpr int kPrologueThreads = 256;

// ---------------------------------------------------------------------------
// sin / cos as the reference's zenith-angle code evaluates them
// ---------------------------------------------------------------------------

// Intel SVML's four-lane single-precision sin/cos, as WRF's vectorised loop
// computes them and runtime.py:6027-6096 restates them: 1/pi scaling, a
// round-to-integer by adding 1.5 * 2^23, a 4-part Cody-Waite reduction by
// pi, the quadrant parity as a sign flip and an odd degree-9 polynomial.
// Every step is one binary32 operation (explicit _rn intrinsics: never
// contracted).  Constants come from the table blob (svml.sinf, svml.cosf) in
// the order the reference's code lists them.
__device__ __forceinline__ float svml_reduce_poly(const float *k, float src, float y, uint32_t octant) {
  float x = __fsub_rn(src, __fmul_rn(y, k[0]));
  x = __fsub_rn(x, __fmul_rn(y, k[1]));
  x = __fsub_rn(x, __fmul_rn(y, k[2]));
  x = __fsub_rn(x, __fmul_rn(y, k[3]));
  const float x2 = __fmul_rn(x, x);
  const float sx = __uint_as_float(__float_as_uint(x) ^ octant);
  float q = __fmul_rn(k[4], x2);
  q = __fadd_rn(q, k[5]);
  q = __fmul_rn(q, x2);
  q = __fadd_rn(q, k[6]);
  q = __fmul_rn(q, x2);
  q = __fadd_rn(q, k[7]);
  float corr = __fmul_rn(x2, q);
  corr = __fmul_rn(sx, corr);
  return __fadd_rn(sx, corr);
}

// K.s: 1/pi, 1.5*2^23 (twice), pi in 4 parts, 4 polynomial terms, |x| limit.
__device__ __forceinline__ float svml_sinf(const SvmlConsts &K, float src) {
  const uint32_t bits = __float_as_uint(src);
  const float a = __uint_as_float(bits & 0x7fffffffu);
  float y = __fmul_rn(a, K.s[0]);
  y = __fadd_rn(y, K.s[1]);
  const uint32_t octant = __float_as_uint(y) << 31;
  y = __fsub_rn(y, K.s[2]);
  float r = svml_reduce_poly(K.s + 3, a, y, octant);
  r = __uint_as_float(__float_as_uint(r) ^ (bits & 0x80000000u));
  // beyond |x| = 1e4 the reference switches to the library sin; no zenith
  // input gets there (|latitude| <= pi/2, |hour angle| < 13 rad)
  return fabsf(src) > K.s[11] ? sinf(src) : r;
}

// K.c: pi/2, 1/pi, 1.5*2^23 (twice), 1/2, pi in 4 parts, 4 polynomial terms, |x| limit.
__device__ __forceinline__ float svml_cosf(const SvmlConsts &K, float src) {
  float y = __fadd_rn(K.c[0], src);
  y = __fmul_rn(y, K.c[1]);
  y = __fadd_rn(y, K.c[2]);
  const uint32_t octant = __float_as_uint(y) << 31;
  y = __fsub_rn(y, K.c[3]);
  y = __fsub_rn(y, K.c[4]);
  const float r = svml_reduce_poly(K.c + 5, src, y, octant);
  return fabsf(src) > K.c[13] ? cosf(src) : r;
}

// glibc 2.39 sinf/cosf (sysdeps/ieee754/flt-32/s_sinf.c, s_cosf.c with the
// data of sincosf_data.c; the x86-64 FMA build that the reference's libm
// calls reach), for |x| < 120: the argument in binary64, |x| < 0.75 straight
// into the polynomials, otherwise reduced by n * pi/2 with n rounded from
// x * 2^24 * 2/pi; the quadrant picks sin or cos and their signs.
struct GlibcSinCos {
  double hpi_inv = 0x1.45F306DC9C883p+23;
  double hpi = 0x1.921FB54442D18p0;
  double c0 = 0x1p0, c1 = -0x1.ffffffd0c621cp-2, c2 = 0x1.55553e1068f19p-5,
         c3 = -0x1.6c087e89a359dp-10, c4 = 0x1.99343027bf8c3p-16;
  double s1 = -0x1.555545995a603p-3, s2 = 0x1.1107605230bc4p-7, s3 = -0x1.994eb3774cf24p-13;
};

__device__ __forceinline__ float glibc_sincos_poly(double x, double x2, int n, double neg_cos) {
  const GlibcSinCos p;
  if ((n & 1) == 0) {
    const double x3 = __dmul_rn(x, x2);
    const double s1 = __fma_rn(x2, p.s3, p.s2);
    const double x7 = __dmul_rn(x3, x2);
    const double s = __fma_rn(x3, p.s1, x);
    return __double2float_rn(__fma_rn(x7, s1, s));
  }
  const double x4 = __dmul_rn(x2, x2);
  const double c2 = __fma_rn(x2, neg_cos * p.c4, neg_cos * p.c3);
  const double c1 = __fma_rn(x2, neg_cos * p.c1, neg_cos * p.c0);
  const double x6 = __dmul_rn(x4, x2);
  const double c = __fma_rn(x4, neg_cos * p.c2, c1);
  return __double2float_rn(__fma_rn(x6, c2, c));
}

__device__ __forceinline__ uint32_t abstop12(float y) { return (__float_as_uint(y) >> 20) & 0x7ffu; }

// cosine = false: sinf, true: cosf
__device__ float glibc_sinf_cosf(float y, bool cosine) {
  const GlibcSinCos p;
  const double x = static_cast<double>(y);
  if (abstop12(y) < abstop12(0x1.921FB6p-1f)) {
    if (abstop12(y) < abstop12(0x1p-12f)) return cosine ? 1.0f : y;
    return glibc_sincos_poly(x, __dmul_rn(x, x), cosine ? 1 : 0, 1.0);
  }
  if (abstop12(y) < abstop12(120.0f)) {
    const double r = __dmul_rn(x, p.hpi_inv);
    const int n = (static_cast<int32_t>(r) + 0x800000) >> 24;
    const double xr = __fma_rn(-static_cast<double>(n), p.hpi, x);
    const double s = ((n & 3) == 1 || (n & 3) == 2) ? -1.0 : 1.0;
    const double neg_cos = (n & 2) ? -1.0 : 1.0;
    return glibc_sincos_poly(__dmul_rn(xr, s), __dmul_rn(xr, xr), cosine ? (n ^ 1) : n, neg_cos);
  }
  // large arguments: beyond every zenith input (see svml_sinf)
  return cosine ? cosf(y) : sinf(y);
}

// ---------------------------------------------------------------------------
// per-level pieces
// ---------------------------------------------------------------------------

// WRF cal_cldfra1 for one level (runtime.py:5896-5964): saturation over
// water and ice from Tetens-type fits, the ice-weighted saturation mixing
// ratio, relative humidity, and the Xu-Randall fraction
// RH^0.25 * (1 - exp(-100 qcld / (qvs - qv)^0.49)), cut below 0.01, 1 when
// saturated.  One binary32 operation per reference operation; exp and power
// are CUDA's expf/powf.
__device__ __forceinline__ float cal_cldfra1(float qv, float qc, float qi, float qs, float t, float p) {
  const float es0 = __fmul_rn(1000.0f, 0.61078f);
  const float ep_2 = static_cast<float>(287.0 / 461.6);
  // the reference's final mask first: every other element is 0 whatever the
  // intermediate values (the saturation terms of invalid T or p are never used)
  const bool valid = (t > 100.0f) & (p > 100.0f);
  const float qcld = __fadd_rn(__fadd_rn(qi, qc), qs);
  if (!(valid & (qcld >= 1.0e-12f))) return 0.0f;
  const float tc = __fsub_rn(t, 273.15f);
  const float esw = __fmul_rn(es0, expf(__fdiv_rn(__fmul_rn(17.2693882f, tc), __fsub_rn(t, 35.86f))));
  const float esi = __fmul_rn(es0, expf(__fdiv_rn(__fmul_rn(21.8745584f, tc), __fsub_rn(t, 7.66f))));
  const float dw = __fsub_rn(p, esw), di = __fsub_rn(p, esi);
  const float qvsw = (dw > 1.0f) ? __fdiv_rn(__fmul_rn(ep_2, esw), dw) : 0.0f;
  const float qvsi = (di > 1.0f) ? __fdiv_rn(__fmul_rn(ep_2, esi), di) : 0.0f;
  const float w = __fdiv_rn(__fadd_rn(qi, qs), qcld);
  const float qvs = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, w), qvsw), __fmul_rn(w, qvsi));
  const float rhum = (qvs > 0.0f) ? __fdiv_rn(qv, qvs) : 0.0f;
  if (rhum >= 1.0f) return 1.0f;
  // numpy maximum keeps NaN; so do these selects
  float subsat = __fsub_rn(qvs, qv);
  subsat = (subsat < 1.0e-10f) ? 1.0e-10f : subsat;
  float arg = __fdiv_rn(__fmul_rn(-100.0f, qcld), powf(subsat, 0.49f));
  arg = (arg < -6.9f) ? -6.9f : arg;
  const float rpos = (rhum < 1.0e-10f) ? 1.0e-10f : rhum;
  const float partial = __fmul_rn(powf(rpos, 0.25f), __fsub_rn(1.0f, expf(arg)));
  return (partial < 0.01f) ? 0.0f : partial;
}

// Index of the last entry < v in an ascending table (numpy searchsorted
// 'left' minus one), clamped to [0, n-2].
__device__ __forceinline__ int bracket(const float *tab, int n, float v) {
  int lo = 0, hi = n;  // count of entries < v lies in [lo, hi]
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (tab[mid] < v) lo = mid + 1; else hi = mid;
  }
  const int i = lo - 1;
  return i < 0 ? 0 : (i > n - 2 ? n - 2 : i);
}

struct OzoneColumn {
  const float *lo0, *hi0, *lo1, *hi1;  // the two months' rows at the bracketing latitudes
  float span, dlat, f1, f2;
  // runtime.py:5775-5782: per month lower + (upper - lower) / span * dlat,
  // then the two months weighted; every statement rounded to binary32
  __device__ __forceinline__ float at(int l) const {
    const float a = __fadd_rn(lo0[l], __fmul_rn(__fdiv_rn(__fsub_rn(hi0[l], lo0[l]), span), dlat));
    const float b = __fadd_rn(lo1[l], __fmul_rn(__fdiv_rn(__fsub_rn(hi1[l], lo1[l]), span), dlat));
    return __fadd_rn(__fmul_rn(a, f1), __fmul_rn(b, f2));
  }
};

template <bool kCld, bool kOz, bool kCz, bool kFlag>
__global__ void __launch_bounds__(kPrologueThreads, 5)
prologue_kernel(const PrologueArgs a) {
  extern __shared__ float smem[];
  float *s_plev = smem;                       // levsiz
  float *s_lat = s_plev + a.levsiz;           // latsiz
  float *s_oz = s_lat + a.latsiz;             // (2, latsiz, levsiz): month_lo, month_hi
  if (kOz) {
    const int tab = a.latsiz * a.levsiz;
    for (int e = threadIdx.x; e < a.levsiz; e += blockDim.x) s_plev[e] = __ldg(a.oz_plev + e);
    for (int e = threadIdx.x; e < a.latsiz; e += blockDim.x) s_lat[e] = __ldg(a.oz_lat + e);
    for (int e = threadIdx.x; e < tab; e += blockDim.x) {
      s_oz[e] = __ldg(a.oz_tab + static_cast<size_t>(a.month_lo) * tab + e);
      s_oz[tab + e] = __ldg(a.oz_tab + static_cast<size_t>(a.month_hi) * tab + e);
    }
    __syncthreads();
  }
  const int ncol = a.nx * a.ny;
  const float degrad = static_cast<float>(3.14159265358979323846 / 180.0);
  const int vec_rows = (a.nx / 4) * 4;
  const int lane = threadIdx.x & 31;
  bool any_condensate = false;
  // Cloudy levels (the only ones whose cloud fraction is not 0 by the final
  // mask) are queued per warp and evaluated 32 at a time with every lane
  // busy, instead of in place with most lanes idle: up to 63 element indices
  // per warp (31 left over plus one level's 32).
  __shared__ unsigned long long s_queue[kPrologueThreads / 32][64];
  unsigned long long *q = s_queue[threadIdx.x >> 5];
  int qn = 0;  // warp-uniform
  auto drain = [&](int n) {
    if (lane < n) {
      const size_t e = q[lane];
      a.cldfra[e] = cal_cldfra1(__ldg(a.qv + e), __ldg(a.qc + e), __ldg(a.qi + e), __ldg(a.qs + e),
                                __ldg(a.t + e), __ldg(a.p + e));
    }
  };
  // whole warps take the same columns' iterations (the queue is warp-synchronous)
  for (int c0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); c0 < ncol; c0 += gridDim.x * blockDim.x) {
    const int c = c0 + lane;
    const bool live = c < ncol;
    const int cc = live ? c : ncol - 1;  // in-range addresses for idle lanes; nothing stored for them
    const int i = cc / a.ny, j = cc - i * a.ny;
    if (kCz && live) {
      // runtime.py:6233-6243
      const float lat = __ldg(a.xlat + c), lon = __ldg(a.xlong + c);
      const float tloc = __fadd_rn(a.tloctm0, __fdiv_rn(lon, 15.0f));
      const float hrang = __fmul_rn(__fmul_rn(15.0f, __fsub_rn(tloc, 12.0f)), degrad);
      const float xxlat = __fmul_rn(lat, degrad);
      float s_la, c_la, c_hr;
      if (i < vec_rows) {
        s_la = svml_sinf(a.svml, xxlat);
        c_la = svml_cosf(a.svml, xxlat);
        c_hr = svml_cosf(a.svml, hrang);
      } else {
        s_la = glibc_sinf_cosf(xxlat, false);
        c_la = glibc_sinf_cosf(xxlat, true);
        c_hr = glibc_sinf_cosf(hrang, true);
      }
      const float st = __fmul_rn(s_la, a.sin_declin);
      float ct = __fmul_rn(c_la, a.cos_declin);
      ct = __fmul_rn(ct, c_hr);
      float cz = __fadd_rn(st, ct);
      cz = (cz < -1.0f) ? -1.0f : cz;
      cz = (cz > 1.0f) ? 1.0f : cz;
      a.coszr[c] = cz;
    }
    OzoneColumn oz;
    if (kOz) {
      // runtime.py:5767-5773: latitude bracket and offsets
      const float lat = __ldg(a.xlat + cc);
      const int li = bracket(s_lat, a.latsiz, lat);
      oz.dlat = __fsub_rn(lat, s_lat[li]);
      oz.span = __fsub_rn(s_lat[li + 1], s_lat[li]);
      const float *m0 = s_oz, *m1 = s_oz + a.latsiz * a.levsiz;
      oz.lo0 = m0 + li * a.levsiz;
      oz.hi0 = oz.lo0 + a.levsiz;
      oz.lo1 = m1 + li * a.levsiz;
      oz.hi1 = oz.lo1 + a.levsiz;
      oz.f1 = a.fact_lo;
      oz.f2 = a.fact_hi;
    }
    if (!(kCld || kOz || kFlag)) continue;
    const size_t base = static_cast<size_t>(i) * a.nk * a.ny + j;
    const float ptop = kOz ? s_plev[0] : 0.0f;
    const float pbot = kOz ? s_plev[a.levsiz - 1] : 0.0f;
    // pressure bracket, walked from the previous level's (levels go up, so
    // it mostly stays or steps down), and the climatology at its two ends
    int kk = kOz ? a.levsiz - 2 : 0, cached = -1;
    float v_lo = 0.0f, v_hi = 0.0f;
    constexpr bool kQ = kCld || kFlag, kP = kCld || kOz;
    float n_qc = 0.0f, n_qi = 0.0f, n_qs = 0.0f, n_t = 0.0f, n_p = 0.0f;
    auto load = [&](size_t e) {
      if (kQ) {
        n_qc = __ldg(a.qc + e);
        n_qi = __ldg(a.qi + e);
        n_qs = __ldg(a.qs + e);
      }
      if (kCld) n_t = __ldg(a.t + e);
      if (kP) n_p = __ldg(a.p + e);
    };
    load(base);
    for (int k = 0; k < a.nk; ++k) {
      const size_t e = base + static_cast<size_t>(k) * a.ny;
      const float qc = n_qc, qi = n_qi, qs = n_qs, t = n_t, p = n_p;
      if (k + 1 < a.nk) load(e + a.ny);
      if (kFlag)
        any_condensate |= live && ((__float_as_uint(qc) | __float_as_uint(qi) | __float_as_uint(qs)) & 0x7fffffffu) != 0u;
      if (kCld) {
        // the final mask of runtime.py:5964 first: valid T and p, condensate >= 1e-12
        bool heavy = false;
        if (live) {
          heavy = ((t > 100.0f) & (p > 100.0f)) && __fadd_rn(__fadd_rn(qi, qc), qs) >= 1.0e-12f;
          if (!heavy) a.cldfra[e] = 0.0f;
        }
        const unsigned m = __ballot_sync(0xffffffffu, heavy);
        if (heavy) q[qn + __popc(m & ((1u << lane) - 1u))] = e;
        qn += __popc(m);
        if (qn >= 32) {
          __syncwarp();
          drain(32);
          __syncwarp();
          if (lane < qn - 32) q[lane] = q[32 + lane];
          qn -= 32;
          __syncwarp();
        }
      }
      if (kOz && live) {
        // runtime.py:5788-5801: pressure bracket, linear in pressure; above
        // the top level scaled by p / plev[0], below the bottom the last value
        float v;
        if (p < ptop) {
          v = __fdiv_rn(__fmul_rn(oz.at(0), p), ptop);
        } else if (p > pbot) {
          v = oz.at(a.levsiz - 1);
        } else {
          // largest kk with plev[kk] < p, clamped to [0, levsiz-2]
          while (kk > 0 && !(s_plev[kk] < p)) --kk;
          while (kk < a.levsiz - 2 && s_plev[kk + 1] < p) ++kk;
          if (kk != cached) {
            if (kk == cached - 1) {
              v_hi = v_lo;
              v_lo = oz.at(kk);
            } else {
              v_lo = oz.at(kk);
              v_hi = oz.at(kk + 1);
            }
            cached = kk;
          }
          const float dpu = __fsub_rn(p, s_plev[kk]);
          const float dpl = __fsub_rn(s_plev[kk + 1], p);
          const float num = __fadd_rn(__fmul_rn(v_lo, dpl), __fmul_rn(v_hi, dpu));
          v = __fdiv_rn(num, __fadd_rn(dpl, dpu));
        }
        a.o33d[e] = v;
      }
    }
  }
  if (kCld) {
    __syncwarp();
    drain(qn);
  }
  if (kFlag && __any_sync(0xffffffffu, any_condensate) && lane == 0) atomicOr(a.condensate, 1);
}

template <bool kCld, bool kOz, bool kCz, bool kFlag>
cudaError_t launch_variant(const PrologueArgs &a, int blocks, size_t smem, cudaStream_t stream) {
  auto kern = prologue_kernel<kCld, kOz, kCz, kFlag>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
  }
  kern<<<blocks, kPrologueThreads, smem, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace

size_t prologue_smem_bytes(int levsiz, int latsiz) {
  return sizeof(float) * (static_cast<size_t>(levsiz) + latsiz + 2 * static_cast<size_t>(latsiz) * levsiz);
}

cudaError_t launch_prologue(const PrologueArgs &a, cudaStream_t stream) {
  const bool cld = a.cldfra != nullptr, oz = a.o33d != nullptr, cz = a.coszr != nullptr;
  const bool flag = a.condensate != nullptr;
  const int ncol = a.nx * a.ny;
  if (ncol <= 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = oz ? prologue_smem_bytes(a.levsiz, a.latsiz) : 0;
  // the ozone tables are staged once per block: a persistent grid of a few
  // blocks per SM when they are needed, one thread per column otherwise
  const int need = (ncol + kPrologueThreads - 1) / kPrologueThreads;
  const int blocks = oz ? std::min(need, sms * 5) : need;
  const int key = (cld ? 8 : 0) | (oz ? 4 : 0) | (cz ? 2 : 0) | (flag ? 1 : 0);
  switch (key) {
#define RRTMG_PROLOGUE_CASE(K)                                                              \
  case K:                                                                                   \
    return launch_variant<((K) & 8) != 0, ((K) & 4) != 0, ((K) & 2) != 0, ((K) & 1) != 0>( \
        a, blocks, smem, stream);
    RRTMG_PROLOGUE_CASE(1) RRTMG_PROLOGUE_CASE(2) RRTMG_PROLOGUE_CASE(3) RRTMG_PROLOGUE_CASE(4)
    RRTMG_PROLOGUE_CASE(5) RRTMG_PROLOGUE_CASE(6) RRTMG_PROLOGUE_CASE(7) RRTMG_PROLOGUE_CASE(8)
    RRTMG_PROLOGUE_CASE(9) RRTMG_PROLOGUE_CASE(10) RRTMG_PROLOGUE_CASE(11) RRTMG_PROLOGUE_CASE(12)
    RRTMG_PROLOGUE_CASE(13) RRTMG_PROLOGUE_CASE(14) RRTMG_PROLOGUE_CASE(15)
#undef RRTMG_PROLOGUE_CASE
    default:
      return cudaSuccess;
  }
}

}  // namespace rrtmg

// ---------------------------------------------------------------------------
// host helpers for the per-step scalars
// ---------------------------------------------------------------------------
namespace {

// mid-month days of the CAM ozone cycle (runtime.py:5718)
constexpr float kOzoneMidMonth[12] = {16, 45, 75, 105, 136, 166, 197, 228, 258, 289, 319, 350};

// Every line is one binary32 operation: volatile stores keep the host
// compiler from fusing or reordering them.
inline float r32(float v) {
  volatile float s = v;
  return s;
}

}  // namespace

extern "C" rrtmg_status rrtmg_radconst(double julian, float *declin, float *solcon) {
  if (!declin || !solcon) return RRTMG_BAD_ARG;
  // runtime.py:5667-5690
  const float degrad = static_cast<float>(3.14159265358979323846 / 180.0);
  const float dpd = r32(360.0f / 365.0f);
  const float jr = static_cast<float>(julian);
  const float obecl = r32(23.5f * degrad);
  const float sinob = std::sin(obecl);
  float sxlong = jr >= 80.0f ? r32(dpd * r32(jr - 80.0f)) : r32(dpd * r32(jr + 285.0f));
  sxlong = r32(sxlong * degrad);
  *declin = std::asin(r32(sinob * std::sin(sxlong)));
  const float djul = r32(r32(jr * 360.0f) / 365.0f);
  const float rjul = r32(djul * degrad);
  const float twice = r32(2.0f * rjul);
  float ecc = 1.000110f;
  ecc = r32(ecc + r32(0.034221f * std::cos(rjul)));
  ecc = r32(ecc + r32(0.001280f * std::sin(rjul)));
  ecc = r32(ecc + r32(0.000719f * std::cos(twice)));
  ecc = r32(ecc + r32(0.000077f * std::sin(twice)));
  *solcon = r32(1370.0f * ecc);
  return RRTMG_OK;
}

extern "C" rrtmg_status rrtmg_prologue_scalars_from_calendar(double julian, double xtime, double gmt, double declin,
                                                             rrtmg_prologue_scalars *out) {
  if (!out || !std::isfinite(julian) || !std::isfinite(xtime) || !std::isfinite(gmt) || !std::isfinite(declin))
    return RRTMG_BAD_ARG;
  // equation of time and local-time offset (runtime.py:6220-6234)
  const float jr = static_cast<float>(julian);
  const float da = r32(r32(static_cast<float>(6.2831853071795862) * r32(jr - 1.0f)) / 365.0f);
  const float da2 = r32(2.0f * da);
  float eot = 0.000075f;
  eot = r32(eot + r32(0.001868f * std::cos(da)));
  eot = r32(eot - r32(0.032077f * std::sin(da)));
  eot = r32(eot - r32(0.014615f * std::cos(da2)));
  eot = r32(eot - r32(0.04089f * std::sin(da2)));
  eot = r32(eot * 229.18f);
  const float xt24 = r32(std::fmod(static_cast<float>(xtime), 1440.0f) + eot);
  out->tloctm0 = r32(static_cast<float>(gmt) + r32(xt24 / 60.0f));
  out->sin_declin = std::sin(static_cast<float>(declin));
  out->cos_declin = std::cos(static_cast<float>(declin));
  // ozone months (runtime.py:5717-5750)
  float t = r32(jr + 1.0f);
  int whole = static_cast<int>(t);
  const float frac = r32(t - static_cast<float>(whole));
  whole %= 365;
  if (whole == 0) whole = 365;
  t = r32(frac + static_cast<float>(whole));
  int nxt = 0;
  while (nxt < 12 && !(kOzoneMidMonth[nxt] > t)) ++nxt;
  if (nxt == 12) nxt = 0;
  if (nxt > 0) {
    const int prv = nxt - 1;
    const float span = r32(kOzoneMidMonth[nxt] - kOzoneMidMonth[prv]);
    out->month_lo = prv;
    out->month_hi = nxt;
    out->fact_lo = r32(r32(kOzoneMidMonth[nxt] - t) / span);
    out->fact_hi = r32(r32(t - kOzoneMidMonth[prv]) / span);
  } else {
    const float first = kOzoneMidMonth[0], last = kOzoneMidMonth[11];
    const float span = r32(r32(first + 365.0f) - last);
    out->month_lo = 11;
    out->month_hi = 0;
    if (t > first) {
      out->fact_lo = r32(r32(r32(first + 365.0f) - t) / span);
      out->fact_hi = r32(r32(t - last) / span);
    } else {
      out->fact_lo = r32(r32(first - t) / span);
      out->fact_hi = r32(r32(r32(t + 365.0f) - last) / span);
    }
  }
  return RRTMG_OK;
}

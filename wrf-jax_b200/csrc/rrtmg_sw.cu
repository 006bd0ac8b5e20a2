// RRTMG shortwave on the GPU: one thread per column, fused from the WRF adapter
// to the theta tendencies and the 2-D surface/TOA fields.
//
// Reference call: rrtmg_swrad_wrf_columns (src/wrf_jax/physics/module_ra_rrtmg_sw.py:2386)
// and below it: inatm_sw (sw:1250), cldprmc_sw (sw:1409), setcoef_sw (sw:7101),
// taumol16..29 (sw:4043-6675), spcvmc (sw:6788-7094) with reftra (sw:3490-3601)
// and vrtqdr (sw:3604-3720), heating (sw:2285-2301), day mask (sw:2667-2719).
// The adapter passes rounding_token=None, so every statement is one binary32
// operation in the order written.
//
// Schedule.  Night columns (coszr <= 0) write zeros and exit: the reference
// masks every output of such columns.  For a day column the thread walks the
// 14 bands; per band it evaluates the band's gas optics for all layers once
// (thread-local tables of taug/taur and the band's cloud optics), then for each
// g-point runs a top-down pass (delta-Eddington layer reflectance and
// transmittance, direct beam, downward adding recurrence) and a bottom-up pass
// (upward adding recurrence, level fluxes) that accumulates the spectral sums
// in g-point order.
#include <atomic>

#include "rrtmg_device.cuh"
#include "rrtmg_kernels.h"

namespace rrtmg {
namespace {

constexpr int kNgc[kSwBands] = {6, 12, 8, 8, 10, 10, 2, 10, 8, 6, 6, 8, 6, 12};
constexpr int kGofs[kSwBands] = {0, 6, 18, 26, 34, 44, 54, 56, 66, 74, 80, 86, 94, 100};
constexpr int kMaxLev = kMaxLay + 1;
constexpr float kOneMinus = 1.0f - 1.0e-6f;

struct Col {
  int i, j, nk, nlay, ny;
  float o3top, adjflux, mu, coszen, albedo;
  int laytrop;
  int inflg, iceflg, has_reqc, has_reqi, has_reqs, icloud;
  float co2, n2o, ch4;
};

struct SLayer {
  float pavel, tavel, pdp;
  int jp, jt, jt1, indself, indfor, trop;
  float fac00, fac01, fac10, fac11;
  float colh2o, colco2, colo3, colch4, colo2, colmol;
  float selffac, selffrac, forfac, forfrac;
  float cldfrac, clwp, ciwp, cswp, rel, rei, res;
};

// The fields of SLayer, as the sweep schedule's layer kernel stores them
// (one array per field, (layer, chunk slot) with slots fastest) for the
// band-parallel optics kernel.
#define RRTMG_SW_LAYER_FLOATS(X)                                                                           \
  X(pavel) X(tavel) X(pdp) X(fac00) X(fac01) X(fac10) X(fac11) X(colh2o) X(colco2) X(colo3) X(colch4)      \
  X(colo2) X(colmol) X(selffac) X(selffrac) X(forfac) X(forfrac) X(cldfrac) X(clwp) X(ciwp) X(cswp) X(rel) \
  X(rei) X(res)
#define RRTMG_SW_LAYER_INTS(X) X(jp) X(jt) X(jt1) X(indself) X(indfor) X(trop)
#define RRTMG_SW_COUNT(name) +1
constexpr int kSwLayerFields = 1 RRTMG_SW_LAYER_FLOATS(RRTMG_SW_COUNT) RRTMG_SW_LAYER_INTS(RRTMG_SW_COUNT);  // + cloud-water flag
#undef RRTMG_SW_COUNT

__device__ __forceinline__ float in3(const float *p, const Col &C, int k) {
  return ld(p + (static_cast<size_t>(C.i) * C.nk + k) * C.ny + C.j);
}
__device__ __forceinline__ float in3w(const float *p, const Col &C, int k) {
  return ld(p + (static_cast<size_t>(C.i) * (C.nk + 1) + k) * C.ny + C.j);
}

__device__ float o3data_layer(const Tables &T, float pa, float pb) {
  float total = 0.0f;
#pragma unroll 4
  for (int b = 0; b < 31; ++b) {
    const float pb1 = fmaxf(pa - T.ppwrkh[b], 0.0f);
    const float pb2 = fmaxf(pa - T.ppwrkh[b + 1], 0.0f);
    const float pt1 = fmaxf(pb - T.ppwrkh[b], 0.0f);
    const float pt2 = fmaxf(pb - T.ppwrkh[b + 1], 0.0f);
    const float overlap = ((pb2 - pb1) - pt2) + pt1;
    total = total + overlap * T.o3wrk[b];
  }
  return total / (pa - pb);
}

__device__ float retab_interp(const Tables &T, float temp, int hi) {
  const int tint = static_cast<int>(temp);
  const int index = clampi(static_cast<int>(temp - 179.0f), 1, hi);
  const float corr = temp - static_cast<float>(tint);
  return ld(T.retab + index - 1) * (1.0f - corr) + ld(T.retab + index) * corr;
}

// Layer quantities: adapter extension, inatm_sw, cloud paths, setcoef_sw.
__device__ SLayer make_layer(const Tables &T, const SwArgs &a, const Col &C, int l) {
  SLayer L;
  const int nk = C.nk;
  const float plev0 = pa_to_hpa(in3w(a.in.p8w, C, l));
  const float plev1 = l + 1 <= nk ? pa_to_hpa(in3w(a.in.p8w, C, l + 1)) : 1.0e-5f;
  L.pavel = l < nk ? pa_to_hpa(in3(a.in.p3d, C, l)) : 0.5f * pa_to_hpa(in3w(a.in.p8w, C, nk));
  L.tavel = l < nk ? in3(a.in.t3d, C, l) : in3w(a.in.t8w, C, nk);
  const int kq = l < nk ? l : nk - 1;
  const float h2o = fmaxf(in3(a.in.qv, C, kq), 1.0e-12f) * 1.607793f;
  const float o3 = l < nk ? in3(a.in.o3, C, l) : C.o3top;
  // inatm_sw (sw:1286-1320)
  const float amd = 28.9660f, amw = 18.0160f, avogad = 6.02214199e23f, grav = 9.8066f;
  L.pdp = plev0 - plev1;
  const float amm = (1.0f - h2o) * amd + h2o * amw;
  const float num = (L.pdp * 1.0e3f) * avogad;
  const float den = ((1.0e2f * grav) * amm) * (1.0f + h2o);
  const float coldry = num / den;
  const float wk0 = h2o * coldry, wk1 = C.co2 * coldry, wk2 = o3 * coldry, wk3 = C.n2o * coldry;
  const float wk5 = C.ch4 * coldry, wk6 = 0.209488f * coldry;
  // setcoef_sw (sw:7101-7306)
  const float stpfac = 296.0f / 1013.0f;
  const float plog = glibc_logf(T, L.pavel);
  const int jp = clampi(static_cast<int>(36.0f - 5.0f * (plog + 0.04f)), 1, 58);
  const float fp = 5.0f * (ld(T.sw_preflog + jp - 1) - plog);
  const float tf = (L.tavel - ld(T.sw_tref + jp - 1)) / 15.0f;
  const int jt = clampi(static_cast<int>(3.0f + tf), 1, 4);
  const float ft = tf - static_cast<float>(jt - 3);
  const float tf1 = (L.tavel - ld(T.sw_tref + jp)) / 15.0f;
  const int jt1 = clampi(static_cast<int>(3.0f + tf1), 1, 4);
  const float ft1 = tf1 - static_cast<float>(jt1 - 3);
  const float water = wk0 / coldry;
  const float scalefac = (L.pavel * stpfac) / L.tavel;
  const int trop = plog > 4.56f;
  L.trop = l < C.laytrop;
  const float forfac = scalefac / (1.0f + water);
  const float ftf = (332.0f - L.tavel) / 36.0f;
  const int indfor_t = clampi(static_cast<int>(ftf), 1, 2);
  const float forfrac_t = ftf - static_cast<float>(indfor_t);
  const float fsf = (L.tavel - 188.0f) / 36.0f;
  L.indfor = trop ? indfor_t : 3;
  L.forfrac = trop ? forfrac_t : fsf - 1.0f;
  const float selffac_t = water * forfac;
  const float fself = (L.tavel - 188.0f) / 7.2f;
  const int indself_t = clampi(static_cast<int>(fself) - 7, 1, 9);
  const float selffrac_t = fself - static_cast<float>(indself_t + 7);
  L.indself = trop ? indself_t : 0;
  L.selffac = trop ? selffac_t : 0.0f;
  L.selffrac = trop ? selffrac_t : 0.0f;
  L.forfac = forfac;
  const float cs = 1.0e-20f;
  L.colh2o = cs * wk0;
  L.colco2 = cs * wk1;
  L.colo3 = cs * wk2;
  const float coln2o0 = cs * wk3;
  L.colch4 = cs * wk5;
  L.colo2 = cs * wk6;
  L.colmol = cs * coldry + L.colh2o;
  const float fallback = 1.0e-32f * coldry;
  if (L.colco2 == 0.0f) L.colco2 = fallback;
  (void)coln2o0;
  if (L.colch4 == 0.0f) L.colch4 = fallback;
  if (L.colo2 == 0.0f) L.colo2 = fallback;
  const float compfp = 1.0f - fp;
  L.fac10 = compfp * ft;
  L.fac00 = compfp * (1.0f - ft);
  L.fac11 = fp * ft1;
  L.fac01 = fp * (1.0f - ft1);
  L.jp = jp;
  L.jt = jt;
  L.jt1 = jt1;
  // cloud radii and paths (common:801-961); zero in the extra top layer
  L.cldfrac = 0.0f; L.clwp = 0.0f; L.ciwp = 0.0f; L.cswp = 0.0f;
  L.rel = 10.0f; L.rei = 10.0f; L.res = 10.0f;
  if (l < nk) {
    const float t = L.tavel;
    const float cldfra = in3(a.in.cldfra, C, l);
    float qc = fmaxf(in3(a.in.qc, C, l), 0.0f), qi = fmaxf(in3(a.in.qi, C, l), 0.0f);
    float qs = fmaxf(in3(a.in.qs, C, l), 0.0f);
    const int c2 = C.i * C.ny + C.j;
    const float xland = ld(a.in.xland + c2);
    float recloud = 5.0f, reice = 10.0f, resnow = 10.0f;
    if (C.icloud != 0) {
      if (C.has_reqc) {
        recloud = fmaxf(2.5f, in3(a.in.re_cloud, C, l) * 1.0e6f);
        const int cloudy_min = (recloud <= 2.5f) && (cldfra > 0.0f);
        if (cloudy_min && (xland - 1.5f > 0.0f)) recloud = 10.5f;
        if (cloudy_min && (xland - 1.5f < 0.0f)) recloud = 7.5f;
      }
      if (C.has_reqi) {
        reice = fmaxf(5.0f, in3(a.in.re_ice, C, l) * 1.0e6f);
        if ((reice <= 5.0f) && (cldfra > 0.0f)) reice = fmaxf(retab_interp(T, t, 75), 5.0f);
      }
      if (C.has_reqs) resnow = fmaxf(10.0f, in3(a.in.re_snow, C, l) * 1.0e6f);
      if (!C.has_reqs && C.has_reqi && C.has_reqc) {
        resnow = fmaxf(10.0f, in3(a.in.re_ice, C, l) * 1.0e6f);
        qs = qi;
        qi = 0.0f;
        reice = 10.0f;
      }
    }
    const float dp = L.pdp;
    const float denom = fmaxf(0.01f, cldfra);
    float gicewp = (qi + qs) * dp * 100.0f / grav * 1000.0f;
    const float gliqwp = qc * dp * 100.0f / grav * 1000.0f;
    float cicewp = gicewp / denom;
    const float cliqwp = gliqwp / denom;
    if (C.iceflg >= 4) {
      gicewp = qi * dp * 100.0f / grav * 1000.0f;
      cicewp = gicewp / denom;
    }
    float csnowp = 0.0f, res_adj = resnow;
    if (C.iceflg == 5) {
      float smf = 0.99f;
      if (res_adj > 130.0f) {
        const float lim = (130.0f / res_adj) * (130.0f / res_adj);
        smf = fminf(0.99f, lim);
        res_adj = 130.0f;
      }
      const float gsnowp = qs * smf * dp * 100.0f / grav * 1000.0f;
      csnowp = gsnowp / denom;
    }
    const float xice = ld(a.in.xice + c2), snow = ld(a.in.snow + c2);
    const float landm = 2.0f - xland, snowh = 0.001f * snow;
    const float rocean = 14.0f, rland = 8.0f, rice = 14.0f;
    float rel = rland + (rocean - rland) * fminf(1.0f, fmaxf(0.0f, (273.16f - t) * 0.05f));
    rel = rel + (rocean - rel) * fminf(1.0f, fmaxf(0.0f, snowh * 10.0f));
    rel = rel + (rocean - rel) * fminf(1.0f, fmaxf(0.0f, 1.0f - landm));
    rel = rel + (rice - rel) * fminf(1.0f, fmaxf(0.0f, xice));
    float rei = retab_interp(T, t, 94);
    if (C.inflg >= 3) rel = recloud;
    if (C.iceflg >= 4) rei = reice;
    if (C.iceflg == 3) rei = fminf(140.0f, rei * 1.0315f);
    L.cldfrac = cldfra;
    L.clwp = cliqwp;
    L.ciwp = cicewp;
    L.cswp = (C.inflg == 5) ? csnowp : 0.0f;
    L.rel = rel;
    L.rei = rei;
    L.res = (C.inflg == 5) ? res_adj : 10.0f;
  }
  return L;
}

// ---------------------------------------------------------------------------
// taumol16..29 helpers
// ---------------------------------------------------------------------------
struct SwSpec {
  float sc, fs, f[8];
  int js0;
};

__device__ __forceinline__ SwSpec sw_species(float primary, float ratio_secondary, const SLayer &L, float scale, int cap) {
  SwSpec s;
  s.sc = primary + ratio_secondary;
  const float q = primary / s.sc;
  const float sp = q > kOneMinus ? kOneMinus : q;
  const float sm = scale * sp;
  const int js = 1 + static_cast<int>(sm);
  s.fs = sm - floorf(sm);
  const float comp = 1.0f - s.fs;
  s.js0 = clampi(js - 1, 0, cap);
  s.f[0] = comp * L.fac00;
  s.f[1] = s.fs * L.fac00;
  s.f[2] = comp * L.fac10;
  s.f[3] = s.fs * L.fac10;
  s.f[4] = comp * L.fac01;
  s.f[5] = s.fs * L.fac01;
  s.f[6] = comp * L.fac11;
  s.f[7] = s.fs * L.fac11;
  return s;
}

__device__ __forceinline__ float k8(const float *tab, int ngc, int ns, int js0, int jt0, int jt10, int jp0, int jp1,
                                    const float *f, int g) {
  auto R = [&](int js, int jt, int jp) { return ld(tab + (((jp) * 5 + (jt)) * ns + (js)) * ngc + g); };
  float s = f[0] * R(js0, jt0, jp0);
  s = s + f[1] * R(js0 + 1, jt0, jp0);
  s = s + f[2] * R(js0, jt0 + 1, jp0);
  s = s + f[3] * R(js0 + 1, jt0 + 1, jp0);
  s = s + f[4] * R(js0, jt10, jp1);
  s = s + f[5] * R(js0 + 1, jt10, jp1);
  s = s + f[6] * R(js0, jt10 + 1, jp1);
  s = s + f[7] * R(js0 + 1, jt10 + 1, jp1);
  return s;
}

__device__ __forceinline__ float k4(const float *tab, int ngc, int jt0, int jt10, int jp0, int jp1, const SLayer &L, int g) {
  float s = L.fac00 * ld(tab + (jp0 * 5 + jt0) * ngc + g);
  s = s + L.fac10 * ld(tab + (jp0 * 5 + jt0 + 1) * ngc + g);
  s = s + L.fac01 * ld(tab + (jp1 * 5 + jt10) * ngc + g);
  s = s + L.fac11 * ld(tab + (jp1 * 5 + jt10 + 1) * ngc + g);
  return s;
}

__device__ __forceinline__ float self_interp(const SwBand &B, int ngc, const SLayer &L, int g) {
  const int i0 = clampi(L.indself - 1, 0, 8);
  const float s0 = ld(B.selfref + i0 * ngc + g);
  return s0 + L.selffrac * (ld(B.selfref + (i0 + 1) * ngc + g) - s0);
}

__device__ __forceinline__ float for_interp(const SwBand &B, int ngc, const SLayer &L, int g, int cap) {
  const int i0 = clampi(L.indfor - 1, 0, cap);
  const int i1 = jrow(i0 + 1, B.forref_rows);
  const float f0 = ld(B.forref + i0 * ngc + g);
  return f0 + L.forfrac * (ld(B.forref + i1 * ngc + g) - f0);
}

// Gas optical depth and Rayleigh depth of band B (0 = band 16) at one layer.
// The species weights returned in sp8/sp4 feed the solar-source rules.
template <int B>
__device__ __forceinline__ void sw_taumol(const Tables &T, const SLayer &L, float *taug, float *taur, SwSpec &sp8, SwSpec &sp4) {
  constexpr int ngc = kNgc[B];
  constexpr int bn = B + 16;
  const SwBand &K = T.sw[B];
  const bool trop = L.trop;
  const int jp = L.jp;
  const int jt0 = clampi(L.jt - 1, 0, 3), jt10 = clampi(L.jt1 - 1, 0, 3);
  const int jp0 = clampi(jp - 1, 0, 11), jp1 = jp0 + 1;
  const int kjp0 = clampi(jp - 13, 0, 45), kjp1 = clampi(jp - 12, 0, 46);
  const float colh2o = L.colh2o, colmol = L.colmol;
  if constexpr (bn == 16) sp8 = sw_species(colh2o, K.strrat1 * L.colch4, L, 8.0f, 7);
  if constexpr (bn == 17 || bn == 19 || bn == 21) sp8 = sw_species(colh2o, K.strrat * L.colco2, L, 8.0f, 7);
  if constexpr (bn == 18) sp8 = sw_species(colh2o, K.strrat * L.colch4, L, 8.0f, 7);
  if constexpr (bn == 22) sp8 = sw_species(colh2o, (1.6f * K.strrat) * L.colo2, L, 8.0f, 7);
  if constexpr (bn == 24) sp8 = sw_species(colh2o, K.strrat * L.colo2, L, 8.0f, 7);
  if constexpr (bn == 28) sp8 = sw_species(L.colo3, K.strrat * L.colo2, L, 8.0f, 7);
  if constexpr (bn == 17 || bn == 21) sp4 = sw_species(colh2o, K.strrat * L.colco2, L, 4.0f, 3);
  if constexpr (bn == 28) sp4 = sw_species(L.colo3, K.strrat * L.colo2, L, 4.0f, 3);
#pragma unroll
  for (int g = 0; g < ngc; ++g) {
    float tg = 0.0f, tr = 0.0f;
    if constexpr (bn == 16) {
      if (trop) {
        const float ta = k8(K.ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
        const float cont = colh2o * (L.selffac * self_interp(K, ngc, L, g) + L.forfac * for_interp(K, ngc, L, g, 1));
        tg = sp8.sc * ta + cont;
      } else {
        tg = L.colch4 * k4(K.kb, ngc, jt0, jt10, kjp0, kjp1, L, g);
      }
      tr = colmol * K.rayl;
    } else if constexpr (bn == 17 || bn == 21) {
      if (trop) {
        const float ta = k8(K.ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
        const float cont = colh2o * (L.selffac * self_interp(K, ngc, L, g) + L.forfac * for_interp(K, ngc, L, g, 2));
        tg = sp8.sc * ta + cont;
      } else {
        const float sa = k8(K.kb, ngc, 5, sp4.js0, jt0, jt10, kjp0, kjp1, sp4.f, g);
        const float cont = (colh2o * L.forfac) * for_interp(K, ngc, L, g, 2);
        tg = sp8.sc * sa + cont;
      }
      tr = colmol * K.rayl;
    } else if constexpr (bn == 18 || bn == 19) {
      if (trop) {
        const float ta = k8(K.ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
        const float cont = colh2o * (L.selffac * self_interp(K, ngc, L, g) + L.forfac * for_interp(K, ngc, L, g, 2));
        tg = sp8.sc * ta + cont;
      } else {
        const float col = bn == 18 ? L.colch4 : L.colco2;
        tg = col * k4(K.kb, ngc, jt0, jt10, kjp0, kjp1, L, g);
      }
      tr = colmol * K.rayl;
    } else if constexpr (bn == 20) {
      if (trop) {
        const float ta = k4(K.ka, ngc, jt0, jt10, jp0, jp1, L, g);
        const float inner = (ta + L.selffac * self_interp(K, ngc, L, g)) + L.forfac * for_interp(K, ngc, L, g, 2);
        tg = colh2o * inner + L.colch4 * ld(K.absch4 + g);
      } else {
        const float sa = k4(K.kb, ngc, jt0, jt10, kjp0, kjp1, L, g);
        const float inner = sa + L.forfac * for_interp(K, ngc, L, g, 2);
        tg = colh2o * inner + L.colch4 * ld(K.absch4 + g);
      }
      tr = colmol * K.rayl;
    } else if constexpr (bn == 22) {
      const float o2cont = (4.35e-4f * L.colo2) / (350.0f * 2.0f);
      if (trop) {
        const float ta = k8(K.ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
        const float cont = colh2o * (L.selffac * self_interp(K, ngc, L, g) + L.forfac * for_interp(K, ngc, L, g, 2));
        tg = (sp8.sc * ta + cont) + o2cont;
      } else {
        const float sa = k4(K.kb, ngc, jt0, jt10, kjp0, kjp1, L, g);
        tg = (L.colo2 * 1.6f) * sa + o2cont;
      }
      tr = colmol * K.rayl;
    } else if constexpr (bn == 23) {
      if (trop) {
        const float ta = k4(K.ka, ngc, jt0, jt10, jp0, jp1, L, g);
        const float sum = (K.givfac * ta + L.selffac * self_interp(K, ngc, L, g)) + L.forfac * for_interp(K, ngc, L, g, 1);
        tg = colh2o * sum;
      }
      tr = colmol * ld(K.rayl_g + g);
    } else if constexpr (bn == 24) {
      if (trop) {
        const float ta = k8(K.ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
        const float cont = colh2o * (L.selffac * self_interp(K, ngc, L, g) + L.forfac * for_interp(K, ngc, L, g, 1));
        tg = (sp8.sc * ta + L.colo3 * ld(K.abso3a + g)) + cont;
        const float r0 = ld(K.rayla + g * 9 + sp8.js0), r1 = ld(K.rayla + g * 9 + sp8.js0 + 1);
        tr = colmol * (r0 + sp8.fs * (r1 - r0));
      } else {
        const float sa = k4(K.kb, ngc, jt0, jt10, kjp0, kjp1, L, g);
        tg = L.colo2 * sa + L.colo3 * ld(K.abso3b + g);
        tr = colmol * ld(K.raylb + g);
      }
    } else if constexpr (bn == 25) {
      if (trop) {
        const float ta = k4(K.ka, ngc, jt0, jt10, jp0, jp1, L, g);
        tg = colh2o * ta + L.colo3 * ld(K.abso3a + g);
      } else {
        tg = L.colo3 * ld(K.abso3b + g);
      }
      tr = colmol * ld(K.rayl_g + g);
    } else if constexpr (bn == 26) {
      tg = 0.0f;
      tr = colmol * ld(K.rayl_g + g);
    } else if constexpr (bn == 27) {
      const float ab = trop ? k4(K.ka, ngc, jt0, jt10, jp0, jp1, L, g) : k4(K.kb, ngc, jt0, jt10, kjp0, kjp1, L, g);
      tg = L.colo3 * ab;
      tr = colmol * ld(K.rayl_g + g);
    } else if constexpr (bn == 28) {
      if (trop) tg = sp8.sc * k8(K.ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
      else tg = sp8.sc * k8(K.kb, ngc, 5, sp4.js0, jt0, jt10, kjp0, kjp1, sp4.f, g);
      tr = colmol * K.rayl;
    } else {  // 29
      if (trop) {
        const float ta = k4(K.ka, ngc, jt0, jt10, jp0, jp1, L, g);
        const float wat = (ta + L.selffac * self_interp(K, ngc, L, g)) + L.forfac * for_interp(K, ngc, L, g, 2);
        tg = colh2o * wat + L.colco2 * ld(K.absco2 + g);
      } else {
        const float sa = k4(K.kb, ngc, jt0, jt10, kjp0, kjp1, L, g);
        tg = L.colco2 * sa + colh2o * ld(K.absh2o + g);
      }
      tr = colmol * K.rayl;
    }
    taug[g] = tg;
    taur[g] = tr;
  }
}

// cldprmc_sw for one cloudy (band, layer) (sw:1409-1626; ice >= 3, liquid 1)
struct CloudOpt {
  float tau, ssa, asm_, taor;
  bool active;
};

__device__ CloudOpt sw_cloud(const Tables &T, const SLayer &L, int band, int iceflag) {
  CloudOpt o;
  const float cldmin = 1.0e-20f;
  const float ciwp = L.ciwp, clwp = L.clwp, cswp = iceflag == 5 ? L.cswp : 0.0f;
  const float cwp = (ciwp + clwp) + cswp;
  o.active = cwp >= cldmin;
  const float radice = L.rei, radliq = L.rel, radsno = iceflag == 5 ? L.res : 0.0f;
  const float factor = (radice - 2.0f) / 3.0f;
  int index = static_cast<int>(factor);
  if (index == 46) index = 45;
  const float fint = factor - static_cast<float>(index);
  const int r0 = jrow(index - 1, 46), r1 = jrow(index, 46);
  float extice = interpf(ld(T.extice3 + r0 * 14 + band), ld(T.extice3 + r1 * 14 + band), fint);
  float ssaice = interpf(ld(T.ssaice3 + r0 * 14 + band), ld(T.ssaice3 + r1 * 14 + band), fint);
  float gice = interpf(ld(T.asyice3 + r0 * 14 + band), ld(T.asyice3 + r1 * 14 + band), fint);
  const float fdelta = interpf(ld(T.fdlice3 + r0 * 14 + band), ld(T.fdlice3 + r1 * 14 + band), fint);
  const float fw = fdelta + 0.5f / ssaice;
  float forwice = fw > gice ? gice : fw;
  if ((ciwp + cswp) == 0.0f) { extice = 0.0f; ssaice = 0.0f; gice = 0.0f; forwice = 0.0f; }
  float extsno = 0.0f, ssasno = 0.0f, gsno = 0.0f, forwsno = 0.0f;
  if (iceflag == 5 && cswp > 0.0f) {
    const float fs = (radsno - 2.0f) / 3.0f;
    int is = static_cast<int>(fs);
    if (is == 46) is = 45;
    const float fints = fs - static_cast<float>(is);
    const int s0 = jrow(is - 1, 46), s1 = jrow(is, 46);
    extsno = interpf(ld(T.extice3 + s0 * 14 + band), ld(T.extice3 + s1 * 14 + band), fints);
    ssasno = interpf(ld(T.ssaice3 + s0 * 14 + band), ld(T.ssaice3 + s1 * 14 + band), fints);
    gsno = interpf(ld(T.asyice3 + s0 * 14 + band), ld(T.asyice3 + s1 * 14 + band), fints);
    const float fds = interpf(ld(T.fdlice3 + s0 * 14 + band), ld(T.fdlice3 + s1 * 14 + band), fints);
    const float fw2 = fds + 0.5f / ssasno;
    forwsno = fw2 > gsno ? gsno : fw2;
  }
  int il = static_cast<int>(radliq - 1.5f);
  if (il == 0) il = 1;
  if (il == 58) il = 57;
  const float fint_liq = (radliq - 1.5f) - static_cast<float>(il);
  const int q0 = jrow(il - 1, 58), q1 = jrow(il, 58);
  float extliq = interpf(ld(T.extliq1 + q0 * 14 + band), ld(T.extliq1 + q1 * 14 + band), fint_liq);
  float ssaliq = interpf(ld(T.ssaliq1 + q0 * 14 + band), ld(T.ssaliq1 + q1 * 14 + band), fint_liq);
  if (fint_liq < 0.0f && ssaliq > 1.0f) ssaliq = ld(T.ssaliq1 + q0 * 14 + band);
  float gliq = interpf(ld(T.asyliq1 + q0 * 14 + band), ld(T.asyliq1 + q1 * 14 + band), fint_liq);
  if (clwp == 0.0f) { extliq = 0.0f; ssaliq = 0.0f; gliq = 0.0f; }
  const float forwliq = gliq * gliq;
  const float tauliqorig = clwp * extliq;
  const float tauiceorig = ciwp * extice;
  const float ssaliq_d = ssaliq * (1.0f - forwliq) / (1.0f - forwliq * ssaliq);
  const float tauliq = (1.0f - forwliq * ssaliq) * tauliqorig;
  const float ssaice_d = ssaice * (1.0f - forwice) / (1.0f - forwice * ssaice);
  const float tauice = (1.0f - forwice * ssaice) * tauiceorig;
  const float scatliq = ssaliq_d * tauliq;
  float scatice = ssaice_d * tauice;
  float tau_new, taor_new, scatsno = 0.0f;
  if (iceflag == 5) {
    const float tausnoorig = cswp * extsno;
    const float ssasno_d = ssasno * (1.0f - forwsno) / (1.0f - forwsno * ssasno);
    const float tausno = (1.0f - forwsno * ssasno) * tausnoorig;
    scatsno = ssasno_d * tausno;
    tau_new = (tauliq + tauice) + tausno;
    taor_new = (tauliqorig + tauiceorig) + tausnoorig;
  } else {
    tau_new = tauliq + tauice;
    taor_new = tauliqorig + tauiceorig;
  }
  if (tau_new == 0.0f) tau_new = cldmin;
  if (scatice == 0.0f) scatice = cldmin;
  if (scatsno == 0.0f) scatsno = cldmin;
  if (iceflag == 5) {
    const float ssum = (scatliq + scatice) + scatsno;
    o.ssa = ssum / tau_new;
    const float num = (scatliq * (gliq - forwliq) / (1.0f - forwliq) + scatice * (gice - forwice) / (1.0f - forwice)) +
                      scatsno * (gsno - forwsno) / (1.0f - forwsno);
    o.asm_ = num / ssum;
  } else {
    const float ssum = scatliq + scatice;
    o.ssa = ssum / tau_new;
    const float num = scatliq * (gliq - forwliq) / (1.0f - forwliq) + scatice * (gice - forwice) / (1.0f - forwice);
    o.asm_ = num / ssum;
  }
  o.tau = tau_new;
  o.taor = taor_new;
  if (!o.active) { o.tau = 0.0f; o.ssa = 1.0f; o.asm_ = 0.0f; o.taor = 0.0f; }
  return o;
}

__device__ __forceinline__ float exp_lookup(const Tables &T, float v) {
  if (v <= 0.06f) return (1.0f - v) + (0.5f * v) * v;
  const float tblind = v / (T.sw_bpade + v);
  const int it = clampi(static_cast<int>(static_cast<float>(T.sw_ntbl) * tblind + 0.5f), 0, T.sw_ntbl);
  return ld(T.sw_pade_exp + it);
}

struct RT4 {
  float ref, refd, tra, trad;
};

// exp_lookup of min(v, 500) given ex_v = exp_lookup(v) (reftra's clamp of
// its exponent arguments, sw:3530-3545)
__device__ __forceinline__ float lookup_clamped(const Tables &T, float v, float ex_v) {
  return v > 500.0f ? exp_lookup(T, 500.0f) : ex_v;
}

// x / d, or x itself when d is exactly 1 (then the quotient is x exactly).
__device__ __forceinline__ float div_or_same(float x, float d) { return d == 1.0f ? x : x / d; }

// 0 / x as IEEE binary32 division computes it: a zero with the sign of x, or
// the canonical NaN when x is zero or NaN.
__device__ __forceinline__ float zero_over(float x) {
  if (x == 0.0f || x != x) return __int_as_float(0x7fffffff);
  return __int_as_float(__float_as_int(x) & static_cast<int>(0x80000000u));
}

// The four components of x and y have the same bit patterns.
__device__ __forceinline__ bool same_bits(float4 x, float4 y) {
  return ((__float_as_uint(x.x) ^ __float_as_uint(y.x)) | (__float_as_uint(x.y) ^ __float_as_uint(y.y)) |
          (__float_as_uint(x.z) ^ __float_as_uint(y.z)) | (__float_as_uint(x.w) ^ __float_as_uint(y.w))) == 0u;
}

// FP64 mode: the Pade lookup of exp(-v) (sw:2722-2760) with binary64
// arithmetic; the table is the same binary32 data.
__device__ __forceinline__ double exp_lookup64(const Tables &T, double v) {
  if (v <= 0.06) return (1.0 - v) + (0.5 * v) * v;
  const double tblind = v / (static_cast<double>(T.sw_bpade) + v);
  const int it = clampi(static_cast<int>(static_cast<double>(T.sw_ntbl) * tblind + 0.5), 0, T.sw_ntbl);
  return static_cast<double>(ld(T.sw_pade_exp + it));
}

// FP64 mode's reftra (sw:3490-3601) for a layer whose delta-scaled
// single-scattering albedo zwo is >= 0.999 or whose optical depth zto1 is
// below 0.1: both branches in binary64 on the binary32 inputs, the four
// results rounded once.  Near zwo = 1 the general branch's g1 * g1 - g2 * g2
// cancels (its binary32 relative error grows as 1 / (1 - zw)); for a thin
// layer the O(1) terms of the reflectance and transmittance numerators cancel
// to O(zto1), and in binary32 a layer of optical depth 5e-4 can come out with
// a negative reflectance and 70% transmittance instead of 99.96%.
__device__ __noinline__ RT4 reftra64(const Tables &T, float zg_in, float mu_in, float zto1_in, float zw_in) {
  const double zg = zg_in, mu = mu_in, zto1 = zto1_in, zw = zw_in;
  const double eps = 1.0e-8, zwcrit = 0.9999995;
  double ref, refd, tra, trad;
  const double zg3 = 3.0 * zg;
  const double g1 = (8.0 - zw * (5.0 + zg3)) * 0.25;
  const double g2 = 3.0 * (zw * (1.0 - zg)) * 0.25;
  const double g3 = (2.0 - zg3 * mu) * 0.25;
  const double g4 = 1.0 - g3;
  const double sr = zg != 1.0 ? zg / (1.0 - zg) : 0.0;
  const double denom = zg != 1.0 ? 1.0 - (1.0 - zw) * sr * sr : 1.0;
  const double zwo = (zw > 0.0 && denom != 0.0) ? zw / denom : 0.0;
  double ze2 = zto1 / mu;
  if (ze2 > 500.0) ze2 = 500.0;
  const double zem2 = exp_lookup64(T, ze2);
  if (zwo >= zwcrit) {
    const double za = g1 * mu;
    const double za1 = za - g3;
    const double zgt = g1 * zto1;
    ref = (zgt - za1 * (1.0 - zem2)) / (1.0 + zgt);
    tra = 1.0 - ref;
    refd = zgt / (1.0 + zgt);
    trad = 1.0 - refd;
    if (zem2 == 1.0) { ref = 0.0; tra = 1.0; refd = 0.0; trad = 1.0; }
  } else {
    const double za1 = g1 * g4 + g2 * g3;
    const double za2 = g1 * g3 + g2 * g4;
    const double rad = g1 * g1 - g2 * g2;
    const double zrk = sqrt(rad > 0.0 ? rad : 0.0);
    const double zrp = zrk * mu;
    const double zrp1 = 1.0 + zrp, zrm1 = 1.0 - zrp, zrk2 = 2.0 * zrk;
    const double zrpp = 1.0 - zrp * zrp;
    const double zrkg = zrk + g1;
    const double zr1 = zrm1 * (za2 + zrk * g3);
    const double zr2 = zrp1 * (za2 - zrk * g3);
    const double zr3 = zrk2 * (g3 - za2 * mu);
    const double zr4 = zrpp * zrkg;
    const double zr5 = zrpp * (zrk - g1);
    const double zt1 = zrp1 * (za1 + zrk * g4);
    const double zt2 = zrm1 * (za1 - zrk * g4);
    const double zt3 = zrk2 * (g4 + za1 * mu);
    const double zbeta = (g1 - zrk) / zrkg;
    double ze1 = zrk * zto1;
    if (ze1 > 500.0) ze1 = 500.0;
    const double zem1 = exp_lookup64(T, ze1);
    const double zep1 = 1.0 / zem1;
    const double zep2 = 1.0 / zem2;
    const double zdenr = zr4 * zep1 + zr5 * zem1;
    const double zdent = zr4 * zep1 + zr5 * zem1;
    if (zdenr >= -eps && zdenr <= eps) {
      ref = eps;
      tra = zem2;
    } else {
      ref = zw * (zr1 * zep1 - zr2 * zem1 - zr3 * zem2) / zdenr;
      tra = zem2 - zem2 * zw * (zt1 * zep1 - zt2 * zem1 - zt3 * zep2) / zdent;
    }
    const double zemm = zem1 * zem1;
    const double zdend = 1.0 / ((1.0 - zbeta * zemm) * zrkg);
    refd = g2 * (1.0 - zemm) * zdend;
    trad = zrk2 * zem1 * zdend;
  }
  RT4 r;
  r.ref = static_cast<float>(ref);
  r.refd = static_cast<float>(refd);
  r.tra = static_cast<float>(tra);
  r.trad = static_cast<float>(trad);
  return r;
}

// Delta-Eddington layer reflectance/transmittance (reftra_sw_columns,
// sw:3490-3601) of a layer that scatters (the reference's lrt = true).
// zto1_mu = zto1 / mu and ex_zto1_mu = exp_lookup(zto1_mu) come from the
// caller, which needs the same quotient and lookup for its direct beam.
// Divisions whose divisor is exactly 1 are skipped: their quotient is the
// dividend, bit for bit.
// kFp64: the FP64 mode, which hands layers with zwo >= 0.999 or zto1 < 0.1
// to reftra64.
template <bool kFp64>
__device__ __forceinline__ RT4 reftra(const Tables &T, float zg, float mu, float zto1, float zw, float zto1_mu,
                                      float ex_zto1_mu) {
  RT4 r;
  const float eps = 1.0e-8f, zwcrit = 0.9999995f;
  const float zg3 = 3.0f * zg;
  const float g1 = (8.0f - zw * (5.0f + zg3)) * 0.25f;
  const float g2 = 3.0f * (zw * (1.0f - zg)) * 0.25f;
  const float g3 = (2.0f - zg3 * mu) * 0.25f;
  const float g4 = 1.0f - g3;
  const float sr = zg != 1.0f ? div_or_same(zg, 1.0f - zg) : 0.0f;
  const float denom = zg != 1.0f ? 1.0f - (1.0f - zw) * sr * sr : 1.0f;
  const float zwo = (zw > 0.0f && denom != 0.0f) ? div_or_same(zw, denom) : 0.0f;
  if constexpr (kFp64) {
    if (zwo >= 0.999f || zto1 < 0.1f) return reftra64(T, zg, mu, zto1, zw);
  }
  if (zwo >= zwcrit) {
    const float za = g1 * mu;
    const float za1 = za - g3;
    const float zgt = g1 * zto1;
    const float ex = lookup_clamped(T, zto1_mu, ex_zto1_mu);
    r.ref = (zgt - za1 * (1.0f - ex)) / (1.0f + zgt);
    r.tra = 1.0f - r.ref;
    r.refd = zgt / (1.0f + zgt);
    r.trad = 1.0f - r.refd;
    if (ex == 1.0f) { r.ref = 0.0f; r.tra = 1.0f; r.refd = 0.0f; r.trad = 1.0f; }
    return r;
  }
  const float za1 = g1 * g4 + g2 * g3;
  const float za2 = g1 * g3 + g2 * g4;
  const float rad = g1 * g1 - g2 * g2;
  const float zrk = sqrtf(rad > 0.0f ? rad : 0.0f);
  const float zrp = zrk * mu;
  const float zrp1 = 1.0f + zrp, zrm1 = 1.0f - zrp, zrk2 = 2.0f * zrk;
  const float zrpp = 1.0f - zrp * zrp;
  const float zrkg = zrk + g1;
  const float zr1 = zrm1 * (za2 + zrk * g3);
  const float zr2 = zrp1 * (za2 - zrk * g3);
  const float zr3 = zrk2 * (g3 - za2 * mu);
  const float zr4 = zrpp * zrkg;
  const float zr5 = zrpp * (zrk - g1);
  const float zt1 = zrp1 * (za1 + zrk * g4);
  const float zt2 = zrm1 * (za1 - zrk * g4);
  const float zt3 = zrk2 * (g4 + za1 * mu);
  const float zbeta = (g1 - zrk) / zrkg;
  float ze1 = zrk * zto1;
  if (ze1 > 500.0f) ze1 = 500.0f;
  const float zem1 = exp_lookup(T, ze1);
  const float zep1 = 1.0f / zem1;
  const float zem2 = lookup_clamped(T, zto1_mu, ex_zto1_mu);
  const float zep2 = 1.0f / zem2;
  const float zdenr = zr4 * zep1 + zr5 * zem1;
  const float zdent = zr4 * zep1 + zr5 * zem1;
  if ((zdenr >= -eps) && (zdenr <= eps)) {
    r.ref = eps;
    r.tra = zem2;
  } else {
    r.ref = zw * (zr1 * zep1 - zr2 * zem1 - zr3 * zem2) / zdenr;
    r.tra = zem2 - zem2 * zw * (zt1 * zep1 - zt2 * zem1 - zt3 * zep2) / zdent;
  }
  const float zemm = zem1 * zem1;
  const float zdend = 1.0f / ((1.0f - zbeta * zemm) * zrkg);
  r.refd = g2 * (1.0f - zemm) * zdend;
  r.trad = zrk2 * zem1 * zdend;
  return r;
}

// Solar source of band B (the per-band rules of sw:4430-4450): the source
// layer from the layers' jp (jp(l)), the spectral interpolation (js0, fs) of
// the layer (spec(ls, js0, fs), asked only when the band uses it), and the
// source of each g-point.
template <int B, class JpFn, class SpecFn>
__device__ __forceinline__ void sw_source(const Tables &T, const Col &C, JpFn jp, SpecFn spec, float *sflux) {
  constexpr int ngc = kNgc[B];
  constexpr int bn = B + 16;
  const int n = C.nlay;
  const SwBand &K = T.sw[B];
  const int layreffr = K.layreffr;
  int ls = -1;
  bool found = false;
  // The searches read jp in batches of kJpBatch layers so that the record
  // loads overlap; each stops where its condition can no longer hold (below
  // laytrop for the lower-atmosphere bands, from laytrop up for 17 and 28).
  constexpr int kJpBatch = 8;
  if constexpr (bn == 18 || bn == 19 || bn == 21 || bn == 22 || bn == 24) {
    // first troposphere crossing of layreffr, one layer up, capped at laytrop-1
    const int lend = C.laytrop < n ? C.laytrop : n;
    for (int l0 = 0; l0 < lend && !found; l0 += kJpBatch) {
      int jb[kJpBatch + 1];
#pragma unroll
      for (int q = 0; q <= kJpBatch; ++q) jb[q] = l0 + q < n ? jp(l0 + q) : 0;
#pragma unroll
      for (int q = 0; q < kJpBatch; ++q) {
        const int l = l0 + q;
        if (l < lend && !found) {
          const int jl = jb[q];
          const int next = l + 1 < n ? jb[q + 1] : jl;
          if (jl < layreffr && next >= layreffr) {
            found = true;
            ls = (l + 1 < C.laytrop - 1) ? l + 1 : C.laytrop - 1;
          }
        }
      }
    }
    if (!found) ls = C.laytrop - 1;
  }
  if constexpr (bn == 17 || bn == 28) {
    const int lbeg = C.laytrop > 1 ? C.laytrop : 1;
    for (int l0 = lbeg; l0 < n && !found; l0 += kJpBatch) {
      int jb[kJpBatch + 1];  // jp(l0 - 1 + q)
#pragma unroll
      for (int q = 0; q <= kJpBatch; ++q) jb[q] = l0 - 1 + q < n ? jp(l0 - 1 + q) : 0;
#pragma unroll
      for (int q = 0; q < kJpBatch; ++q) {
        const int l = l0 + q;
        if (l < n && !found && jb[q] < layreffr && jb[q + 1] >= layreffr) {
          found = true;
          ls = l;
        }
      }
    }
    if (!found) ls = n - 1;
  }
  bool have = false;
  if constexpr (bn == 17 || bn == 28) have = C.laytrop < n;
  if constexpr (bn == 18 || bn == 19 || bn == 21 || bn == 22 || bn == 24) have = C.laytrop > 0;
  float src_fs = 0.0f;
  int src_js0 = 0;
  if (have && ls >= 0) spec(ls, src_js0, src_fs);
#pragma unroll
  for (int g = 0; g < ngc; ++g) {
    float sz = 0.0f;
    if constexpr (bn == 16 || bn == 29) sz = C.laytrop < n ? ld(K.sfluxref + g) : 0.0f;
    if constexpr (bn == 20 || bn == 23 || bn == 25 || bn == 26) sz = C.laytrop > 0 ? ld(K.sfluxref + g) : 0.0f;
    if constexpr (bn == 27) sz = C.laytrop < n ? K.scalekur * ld(K.sfluxref + g) : 0.0f;
    if constexpr (bn == 17 || bn == 28 || bn == 18 || bn == 19 || bn == 21 || bn == 22 || bn == 24) {
      if (have) {
        const int c = K.sflux_cols;
        const float s0 = ld(K.sfluxref + g * c + src_js0), s1 = ld(K.sfluxref + g * c + src_js0 + 1);
        sz = s0 + src_fs * (s1 - s0);
      }
    }
    sflux[g] = sz;
  }
}

// Day-column compaction: a warp ballots its columns' coszr > 0 and appends the
// day columns to a.daylist (one atomic per warp, ascending within a warp); the
// night columns' outputs (sw:2536-2557 masks them to zero) and every column's
// coszr / *cln outputs are written here.
__global__ void __launch_bounds__(256) sw_daylist_kernel(SwArgs a) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool inside = col < a.ncol && !dead_column(a.live, col);
  const float coszen = inside ? ld(a.in.coszr + col) : 0.0f;
  const bool day = coszen > 0.0f;
  const unsigned ballot = __ballot_sync(0xffffffffu, inside && day);
  int base = 0;
  if (lane == 0 && ballot) base = atomicAdd(a.nday, __popc(ballot));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (!inside) return;
  a.coszr_out[col] = coszen;
#pragma unroll
  for (int q = 0; q < 4; ++q) a.zero2[q][col] = 0.0f;
  if (day) {
    a.daylist[base + __popc(ballot & ((1u << lane) - 1u))] = col;
    return;
  }
  const int i = col / a.ny, j = col - i * a.ny;
  const size_t rbase = static_cast<size_t>(i) * a.nk * a.ny + j;
  for (int k = 0; k < a.nk; ++k) {
    a.rthraten[rbase + static_cast<size_t>(k) * a.ny] = 0.0f;
    a.rthratenc[rbase + static_cast<size_t>(k) * a.ny] = 0.0f;
  }
  a.upt[col] = 0.0f; a.uptc[col] = 0.0f; a.dnt[col] = 0.0f; a.dntc[col] = 0.0f;
  a.upb[col] = 0.0f; a.upbc[col] = 0.0f; a.dnb[col] = 0.0f; a.dnbc[col] = 0.0f;
  a.swcf[col] = 0.0f; a.gsw[col] = 0.0f; a.swddir[col] = 0.0f; a.swddni[col] = 0.0f;
  a.swddif[col] = 0.0f; a.swdownc[col] = 0.0f; a.swddnic[col] = 0.0f; a.swddirc[col] = 0.0f;
}

__device__ __forceinline__ float sw_pavel(const SwArgs &a, const Col &C, int l) {
  return l < C.nk ? pa_to_hpa(in3(a.in.p3d, C, l)) : 0.5f * pa_to_hpa(in3w(a.in.p8w, C, C.nk));
}

// Column set-up of a day column without laytrop (buffer ozone; sw:2491-2508).
__device__ __forceinline__ void sw_setup_head(const Tables &T, const SwArgs &a, int col, Col &C) {
  C.i = col / a.ny;
  C.j = col - C.i * a.ny;
  C.nk = a.nk;
  C.ny = a.ny;
  C.nlay = a.nk + 1;
  const int nk = C.nk, n = C.nlay;
  const float coszen = ld(a.in.coszr + col);
  C.coszen = coszen;
  C.mu = fmaxf(coszen, 1.0e-10f);
  C.albedo = ld(a.in.albedo + col);
  C.co2 = a.co2; C.n2o = a.n2o; C.ch4 = a.ch4;
  C.inflg = a.inflg; C.iceflg = a.iceflg;
  C.has_reqc = a.has_reqc; C.has_reqi = a.has_reqi; C.has_reqs = a.has_reqs; C.icloud = a.icloud;
  C.adjflux = 1.0f * (a.solcon / 1.36822e3f);
  // ozone in the extra top layer (sw:2491-2508)
  {
    const float amdo = 0.603461f;
    const float pnk1 = pa_to_hpa(in3w(a.in.p8w, C, nk - 1)), pnk = pa_to_hpa(in3w(a.in.p8w, C, nk));
    const float mmr_k = o3data_layer(T, pnk1, pnk);
    const float mmr_t = o3data_layer(T, pnk, 1.0e-5f);
    float top = (in3(a.in.o3, C, nk - 1) - mmr_k * amdo) + mmr_t * amdo;
    if (top <= 0.0f) top = mmr_t * amdo;
    C.o3top = top;
  }
  (void)n;
}

// Heating rate and theta tendency of layer l of a day column from its level
// sums accs (six arrays of stride `stride`, top-down; sw:2285-2301).
__device__ __forceinline__ void sw_layer_output(const SwArgs &a, const Col &C, int l, const float *accs,
                                                int stride) {
  const int nk = C.nk, n = C.nlay;
  const size_t rbase = static_cast<size_t>(C.i) * nk * C.ny + C.j;
  const float *fu = accs, *fd = accs + stride, *cu = accs + 2 * stride, *cd = accs + 3 * stride;
  const float heatfac = (9.8066f * 8.6400e4f) / (1004.5f * 1.0e2f);
  // bottom-up level l is top-down index n - l
  const float n1 = fd[n - (l + 1)] - fu[n - (l + 1)], n0 = fd[n - l] - fu[n - l];
  const float c1 = cd[n - (l + 1)] - cu[n - (l + 1)], c0 = cd[n - l] - cu[n - l];
  const float plev0 = pa_to_hpa(in3w(a.in.p8w, C, l));
  const float plev1 = pa_to_hpa(in3w(a.in.p8w, C, l + 1));
  const float zdpgcp = heatfac / (plev0 - plev1);
  float hr = (n1 - n0) * zdpgcp;
  float hrc = (c1 - c0) * zdpgcp;
  if (l >= a.fp64_from) {  // FP64 mode
    hr = heating64(heatfac, fu[n - l], fd[n - l], fu[n - (l + 1)], fd[n - (l + 1)], plev0, plev1);
    hrc = heating64(heatfac, cu[n - l], cd[n - l], cu[n - (l + 1)], cd[n - (l + 1)], plev0, plev1);
  }
  const float pi3d = ld(a.in.pi3d + rbase + static_cast<size_t>(l) * C.ny);
  a.rthraten[rbase + static_cast<size_t>(l) * C.ny] = (hr / 86400.0f) / pi3d;
  a.rthratenc[rbase + static_cast<size_t>(l) * C.ny] = (hrc / 86400.0f) / pi3d;
}

// 2-D outputs of a day column from its level sums (sw:2536-2719).
__device__ __forceinline__ void sw_column_outputs(const SwArgs &a, const Col &C, int col, const float *accs,
                                                  int stride) {
  const int n = C.nlay;
  const float coszen = C.coszen;
  const float *fu = accs, *fd = accs + stride, *cu = accs + 2 * stride, *cd = accs + 3 * stride;
  const float *fdir = accs + 4 * stride, *cdir = accs + 5 * stride;
  a.upt[col] = fu[0];
  a.uptc[col] = cu[0];
  a.dnt[col] = fd[0];
  a.dntc[col] = cd[0];
  a.upb[col] = fu[n];
  a.upbc[col] = cu[n];
  a.dnb[col] = fd[n];
  a.dnbc[col] = cd[n];
  a.swcf[col] = (fd[0] - fu[0]) - (cd[0] - cu[0]);
  a.gsw[col] = fd[n] - fu[n];
  a.swddir[col] = fdir[n];
  a.swddni[col] = fdir[n] / coszen;
  a.swddif[col] = fd[n] - fdir[n];
  a.swdownc[col] = cd[n];
  a.swddirc[col] = cdir[n];
  a.swddnic[col] = cdir[n] / coszen;
}

// ---------------------------------------------------------------------------
// Sweep schedule, every domain size.  Day-list slots are processed in chunks;
// per chunk:
//   sw_colprep_kernel  warp = day slot: the column set-up once (laytrop by a
//                      warp vote over the layers);
//   sw_layer_kernel    thread = (day slot, layer): the layer set-up into
//                      layer fields, and jp into the layer record;
//   sw_optics_kernel   thread = (day slot, layer), block = one band: the
//                      band's gas and Rayleigh depths of every g-point, its
//                      cloud optics and the spectral interpolation its solar
//                      source uses, into the layer record;
//   sw_source_kernel   thread = (day slot, band): the band's solar source;
//   sw_sweep_kernel    block = kSweepCols day slots x 112 g-points, thread =
//                      one g-point: the top-down pass (delta-Eddington layers,
//                      direct beam, downward adding) and the bottom-up pass
//                      (upward adding, level fluxes) of spcvmc, the
//                      per-level spectral sums in g-point order in shared
//                      memory, then heating and the 2-D outputs.
// Records: per chunk slot a column record, then nlay layer records of kSwRec
// floats (1,376 bytes per layer, 70 KB per day column at nk = 50), then the
// kSwLayerFields layer fields (124 bytes per layer).  Each
// band's g-points start on a 16-byte boundary (kPadOfs) so the optics kernel
// writes whole float4s: taug at [0, 128), taur at [128, 256), the cloud optics
// (tau, ssa, asm, unscaled tau) of band B at 256 + 4 B, the solar-source
// interpolation (js0, fs) of band B at 312 + 2 B, jp at 340.
constexpr int kSwRec = 344;
constexpr int kSwRecTaur = 128, kSwRecCloud = 256, kSwRecSpec = 312, kSwRecJp = 340;
constexpr int kPadOfs[kSwBands] = {0, 8, 20, 28, 36, 48, 60, 64, 76, 84, 92, 100, 108, 116};
static_assert(kSwRecJp < kSwRec && kSwRec % 4 == 0, "record layout");
__constant__ int kPadOfsDev[kSwBands] = {0, 8, 20, 28, 36, 48, 60, 64, 76, 84, 92, 100, 108, 116};

struct SwColRec {
  Col C;
  float sflux[kSwGpts];
};
constexpr size_t kSwColRecFloats = (sizeof(SwColRec) + 15) / 16 * 4;

// chunk-relative slot u = t - a.chunk_first
__device__ __forceinline__ SwColRec *sw_colrecs(const SwArgs &a) { return reinterpret_cast<SwColRec *>(a.records); }
__device__ __forceinline__ float *sw_layrecs(const SwArgs &a) {
  return a.records + kSwColRecFloats * static_cast<size_t>(a.chunk_capacity);
}
// the layer fields of the chunk: field f of (layer l, slot u) at
// [(f * (nk + 1) + l) * chunk_capacity + u]
__device__ __forceinline__ float *sw_layfields(const SwArgs &a) {
  return sw_layrecs(a) + static_cast<size_t>(kSwRec) * (a.nk + 1) * a.chunk_capacity;
}

// A warp per day column; the lanes take the layers of the laytrop count.
__global__ void __launch_bounds__(128) sw_colprep_kernel(Tables T, SwArgs a) {
  const int lane = threadIdx.x & 31;
  const int u = blockIdx.x * 4 + (threadIdx.x >> 5);
  const int t = a.chunk_first + u;
  if (u >= a.chunk_count || t >= *a.nday) return;  // whole warps
  Col C;
  sw_setup_head(T, a, a.daylist[t], C);
  int count = 0;
  for (int l = lane; l < C.nlay; l += 32) count += glibc_logf(T, sw_pavel(a, C, l)) > 4.56f;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(0xffffffffu, count, o);
  C.laytrop = count;
  if (lane == 0) sw_colrecs(a)[u].C = C;
}

// ngc values of v to float4s at dst (the tail padded with zeros).
template <int NGC>
__device__ __forceinline__ void store_padded(float4 *dst, const float *v) {
#pragma unroll
  for (int q = 0; q < (NGC + 3) / 4; ++q) {
    const int g = 4 * q;
    dst[q] = make_float4(v[g], g + 1 < NGC ? v[g + 1] : 0.0f, g + 2 < NGC ? v[g + 2] : 0.0f,
                         g + 3 < NGC ? v[g + 3] : 0.0f);
  }
}

// Band B of one layer record: gas and Rayleigh depths of every g-point, the
// band's cloud optics (cldprmc_sw only where the layer holds cloud water; a
// layer without any has the reference's inactive values 0, 1, 0, 0), and the
// spectral interpolation its solar source uses (into spec[2 B], spec[2 B + 1]).
template <int B>
__device__ __forceinline__ void sw_band_record(const Tables &T, const SLayer &L, bool cloud_water, int iceflg,
                                               float4 *rec, float *spec) {
  constexpr int ngc = kNgc[B], bn = B + 16, pofs = kPadOfs[B];
  SwSpec sp8, sp4;
  sp8.sc = 0.0f; sp8.fs = 0.0f; sp8.js0 = 0;
  sp4 = sp8;
  float tg[ngc], tr[ngc];
  sw_taumol<B>(T, L, tg, tr, sp8, sp4);
  store_padded<ngc>(rec + pofs / 4, tg);
  store_padded<ngc>(rec + (kSwRecTaur + pofs) / 4, tr);
  float4 cq = make_float4(0.0f, 1.0f, 0.0f, 0.0f);
  if (cloud_water) {
    const CloudOpt o = sw_cloud(T, L, B, iceflg);
    cq = make_float4(o.tau, o.ssa, o.asm_, o.taor);
  }
  rec[kSwRecCloud / 4 + B] = cq;
  const SwSpec &sp = (bn == 17 || bn == 28) ? sp4 : sp8;
  spec[2 * B] = __int_as_float(sp.js0);
  spec[2 * B + 1] = sp.fs;
}

// sw_layer_kernel: thread = (layer, chunk slot), slots fastest: the layer
// set-up (make_layer) and cldprmc_sw's activity test once, stored as layer
// fields, and the layer's jp into its record.
__global__ void __launch_bounds__(128) sw_layer_kernel(Tables T, SwArgs a) {
  const int n = a.nk + 1;
  const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int l = static_cast<int>(idx / a.chunk_count);
  const int u = static_cast<int>(idx - static_cast<long long>(l) * a.chunk_count);
  if (l >= n || a.chunk_first + u >= *a.nday) return;
  const Col C = sw_colrecs(a)[u].C;
  const SLayer L = make_layer(T, a, C, l);
  // the activity test of cldprmc_sw (sw:1409-1440), the same for every band
  const float cswp = C.iceflg == 5 ? L.cswp : 0.0f;
  const bool cloud_water = a.icld != 0 && ((L.ciwp + L.clwp) + cswp) >= 1.0e-20f;
  float *fld = sw_layfields(a) + static_cast<size_t>(l) * a.chunk_capacity + u;
  const size_t fstride = static_cast<size_t>(n) * a.chunk_capacity;
  int f = 0;
#define RRTMG_SW_PUT(name) fld[static_cast<size_t>(f++) * fstride] = L.name;
#define RRTMG_SW_PUTI(name) fld[static_cast<size_t>(f++) * fstride] = __int_as_float(L.name);
  RRTMG_SW_LAYER_FLOATS(RRTMG_SW_PUT)
  RRTMG_SW_LAYER_INTS(RRTMG_SW_PUTI)
#undef RRTMG_SW_PUT
#undef RRTMG_SW_PUTI
  fld[static_cast<size_t>(f) * fstride] = __int_as_float(cloud_water ? 1 : 0);
  float4 *rec = reinterpret_cast<float4 *>(sw_layrecs(a) + (static_cast<size_t>(u) * n + l) * kSwRec);
  rec[kSwRecJp / 4] = make_float4(__int_as_float(L.jp), 0.0f, 0.0f, 0.0f);
}

// sw_optics_kernel: one band per block.  Blocks of (layer, chunk slot) pairs
// are taken kSwOpticsGroup at a time through all 14 bands, so that a group's
// layer fields (about 8 MB) are read from L2 by the later bands; each block
// runs one band's code only.
// Resident blocks per SM the register allocation must allow: 6 (80
// registers); at 8 (64 registers, with spills) the 425 x 425 x 50 step took
// 118 ms instead of 103.
constexpr int kSwOpticsGroup = 512;
constexpr int kSwOpticsMinBlocks = 6;
constexpr int kSwSweepMinBlocks = 4;
__global__ void __launch_bounds__(128, kSwOpticsMinBlocks) sw_optics_kernel(Tables T, SwArgs a, int nblk) {
  const int group = blockIdx.x / (kSwOpticsGroup * kSwBands);
  const int g0 = group * kSwOpticsGroup;
  const int gsize = nblk - g0 < kSwOpticsGroup ? nblk - g0 : kSwOpticsGroup;
  const int within = blockIdx.x - group * kSwOpticsGroup * kSwBands;
  const int band = within / gsize;
  const int blk = g0 + (within - band * gsize);
  const int n = a.nk + 1;
  const long long idx = static_cast<long long>(blk) * blockDim.x + threadIdx.x;
  const int l = static_cast<int>(idx / a.chunk_count);
  const int u = static_cast<int>(idx - static_cast<long long>(l) * a.chunk_count);
  if (l >= n || a.chunk_first + u >= *a.nday) return;
  const float *fld = sw_layfields(a) + static_cast<size_t>(l) * a.chunk_capacity + u;
  const size_t fstride = static_cast<size_t>(n) * a.chunk_capacity;
  SLayer L;
  int f = 0;
#define RRTMG_SW_GET(name) L.name = fld[static_cast<size_t>(f++) * fstride];
#define RRTMG_SW_GETI(name) L.name = __float_as_int(fld[static_cast<size_t>(f++) * fstride]);
  RRTMG_SW_LAYER_FLOATS(RRTMG_SW_GET)
  RRTMG_SW_LAYER_INTS(RRTMG_SW_GETI)
#undef RRTMG_SW_GET
#undef RRTMG_SW_GETI
  const bool cloud_water = __float_as_int(fld[static_cast<size_t>(f) * fstride]) != 0;
  const int iceflg = sw_colrecs(a)[u].C.iceflg;
  float *rec = sw_layrecs(a) + (static_cast<size_t>(u) * n + l) * kSwRec;
  float spec[2 * kSwBands];
#define RRTMG_SW_OPT(B)                                                                                    \
  {                                                                                                        \
    sw_band_record<B>(T, L, cloud_water, iceflg, reinterpret_cast<float4 *>(rec), spec);                   \
    *reinterpret_cast<float2 *>(rec + kSwRecSpec + 2 * (B)) = make_float2(spec[2 * (B)], spec[2 * (B) + 1]); \
  }
  switch (band) {
    case 0: RRTMG_SW_OPT(0); break;
    case 1: RRTMG_SW_OPT(1); break;
    case 2: RRTMG_SW_OPT(2); break;
    case 3: RRTMG_SW_OPT(3); break;
    case 4: RRTMG_SW_OPT(4); break;
    case 5: RRTMG_SW_OPT(5); break;
    case 6: RRTMG_SW_OPT(6); break;
    case 7: RRTMG_SW_OPT(7); break;
    case 8: RRTMG_SW_OPT(8); break;
    case 9: RRTMG_SW_OPT(9); break;
    case 10: RRTMG_SW_OPT(10); break;
    case 11: RRTMG_SW_OPT(11); break;
    case 12: RRTMG_SW_OPT(12); break;
    default: RRTMG_SW_OPT(13); break;
  }
#undef RRTMG_SW_OPT
}

#define RRTMG_SW_BAND_SWITCH(band, CALL) \
  switch (band) {                        \
    case 0: CALL(0); break;              \
    case 1: CALL(1); break;              \
    case 2: CALL(2); break;              \
    case 3: CALL(3); break;              \
    case 4: CALL(4); break;              \
    case 5: CALL(5); break;              \
    case 6: CALL(6); break;              \
    case 7: CALL(7); break;              \
    case 8: CALL(8); break;              \
    case 9: CALL(9); break;              \
    case 10: CALL(10); break;            \
    case 11: CALL(11); break;            \
    case 12: CALL(12); break;            \
    default: CALL(13); break;            \
  }

__global__ void __launch_bounds__(128) sw_source_kernel(Tables T, SwArgs a) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= a.chunk_count || a.chunk_first + u >= *a.nday) return;
  const int n = a.nk + 1;
  SwColRec &R = sw_colrecs(a)[u];
  const float *recs = sw_layrecs(a) + static_cast<size_t>(u) * n * kSwRec;
  const int band = blockIdx.y;
  auto jp = [&](int l) { return __float_as_int(recs[static_cast<size_t>(l) * kSwRec + kSwRecJp]); };
  auto spec = [&](int ls, int &js0, float &fs) {
    const float *q = recs + static_cast<size_t>(ls) * kSwRec + kSwRecSpec + 2 * band;
    js0 = __float_as_int(q[0]);
    fs = q[1];
  };
#define RRTMG_SW_SRC(B)                                 \
  {                                                     \
    constexpr int gofs_ = kGofs[B];                     \
    sw_source<B>(T, R.C, jp, spec, R.sflux + gofs_);    \
  }
  RRTMG_SW_BAND_SWITCH(band, RRTMG_SW_SRC)
#undef RRTMG_SW_SRC
}
#undef RRTMG_SW_BAND_SWITCH

__constant__ int kSwGofsDev[kSwBands] = {0, 6, 18, 26, 34, 44, 54, 56, 66, 74, 80, 86, 94, 100};

constexpr int kSweepCols = 2;                         // day columns per block
constexpr int kSweepThreads = kSweepCols * kSwGpts;   // 224: one thread per g-point
constexpr int kRing = 8;                              // levels of terms per ordered-sum round

// Shared memory of a sweep block: the level terms of the last kRing levels of
// the current pass, awaiting their g-ordered sums, and the sums themselves.
struct SweepShared {
  float ring[kRing][kSweepCols][4][kSwGpts];
  float sums[kSweepCols][6][kMaxLev];  // type: fu, fd, cu, cd, fdir, cdir; level top-down
  uint32_t slotbits[2][kMaxLay / 32][kSweepThreads];  // per thread: cloudy slots, total = clear slots
};

// One level of one adding path, as the bottom-up pass reads it back: the
// layer's reflectances/transmittances and direct-beam transmittance, and the
// level's cumulative direct beam and downward recurrence (vrtqdr, sw:3655-3702).
struct SwLevel {
  float4 rt;   // ref, refd, tra, trad
  float4 dn;   // dbt, tdbt, tdn, rdnd
};

// Adds ring rounds into the sums: chain (column, type, level) adds the 112
// terms of its level in g-point order, starting from zero as the
// reference's ordered sums do (sw:153-177).  `levels[j]` is the level of ring
// slot j, `types` the sums' type indices of the pass's ring types.
__device__ __forceinline__ void sweep_flush(SweepShared &S, int count, int ntypes, const int *types, int level0,
                                            int dir) {
  __syncthreads();
  const int chains = kSweepCols * ntypes * count;
  for (int ch = threadIdx.x; ch < chains; ch += kSweepThreads) {
    const int j = ch % count;
    const int rest = ch / count;
    const int q = rest % ntypes;
    const int c = rest / ntypes;
    const float *v = S.ring[j][c][q];
    float acc = 0.0f;
#pragma unroll 16
    for (int G = 0; G < kSwGpts; ++G) acc = acc + v[G];
    S.sums[c][types[q]][level0 + dir * j] = acc;
  }
  __syncthreads();
}

// Block = kSweepCols consecutive slots of the chunk; thread = (slot, g-point).
// A slot past the day count repeats the block's first slot so that every
// thread takes the same barriers; its results are not written.
//
// Work per g-point layer follows spcvmc (sw:6887-7041) statement by statement;
// three kinds of operation are shared or skipped where the result is known
// bit for bit: the quotient tau / mu and its Pade lookup, computed once for
// the direct beam and reftra's exponent; divisions by a divisor that is
// exactly 1; and, in a g-point layer without cloud, the cloudy
// reflectance/transmittance inputs, whose only consumer is a reftra call the
// reference skips (lrt = false).  The total-sky stack slot of such a layer is
// not stored: the bottom-up pass re-forms it from the clear-sky slot with the
// reference's mixing expression.
template <bool kFp64>
__global__ void __launch_bounds__(kSweepThreads, kSwSweepMinBlocks) sw_sweep_kernel(Tables T, SwArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SweepShared &S = *reinterpret_cast<SweepShared *>(smem_raw);
  const int nday = *a.nday;
  const int u0 = blockIdx.x * kSweepCols;
  if (u0 >= a.chunk_count || a.chunk_first + u0 >= nday) return;  // whole block
  const int cslot = threadIdx.x / kSwGpts;
  const int G = threadIdx.x - cslot * kSwGpts;
  const int u_own = u0 + cslot;
  const bool live = u_own < a.chunk_count && a.chunk_first + u_own < nday;
  const int u = live ? u_own : u0;
  const int col = a.daylist[a.chunk_first + u];
  const SwColRec &R = sw_colrecs(a)[u];
  const Col C = R.C;
  const float sflux_g = R.sflux[G];
  const int n = C.nlay;
  const float mu = C.mu;
  const int clear_only = a.icld == 0;
  int band = kSwBands - 1;
  while (G < kSwGofsDev[band]) --band;
  const int P = kPadOfsDev[band] + (G - kSwGofsDev[band]);  // record position of the g-point
  const float *recs = sw_layrecs(a) + static_cast<size_t>(u) * n * kSwRec;
  const float *crec = recs + kSwRecCloud + 4 * band;
  const uint32_t *maskbase = a.mask + col + static_cast<size_t>(G >> 5) * a.ncol;
  const size_t mstride = static_cast<size_t>(kSwMaskWords) * a.ncol;
  const uint32_t bit = 1u << (G & 31);

  // per-thread stack of the top-down pass, read back bottom-up
  SwLevel stc[kMaxLev], stt[kMaxLev];
  // per stack slot r, bit r & 31 of word r >> 5 (gathered in registers, 32
  // slots at a time, then kept in shared memory): the g-point layer is cloudy
  // (its total-sky reftra results are stored), and the slot's total-sky
  // values equal the clear-sky ones bit for bit (no total-sky slot is stored;
  // the bottom-up pass reuses the clear-sky slot and reads no mask word)
  uint32_t cloudy_bits = 0, same_word = 0;

  // ---- top-down pass: layer optics, direct beam, downward adding (sw:6887-7041)
  const int dtypes[2] = {4, 5};
  float tdbtc_nd = 1.0f, tdbt_nd = 1.0f;
  const float zincflx = ((C.adjflux * sflux_g) * mu) * 1.0f;
  S.ring[0][cslot][0][G] = tdbt_nd * zincflx;
  S.ring[0][cslot][1][G] = tdbtc_nd * zincflx;
  int filled = 1, level0 = 0;
  // carry of the downward recurrence: level r values of each path
  float c_tdbt = 1.0f, c_tdn = 1.0f, c_rdnd = 0.0f;
  float t_tdbt = 1.0f, t_tdn = 1.0f, t_rdnd = 0.0f;
  // layer values are loaded one layer ahead
  const float *rl = recs + static_cast<size_t>(n - 1) * kSwRec;
  float nx_tg = rl[P], nx_tr = rl[kSwRecTaur + P];
  float4 nx_cld = *reinterpret_cast<const float4 *>(crec + static_cast<size_t>(n - 1) * kSwRec);
  uint32_t nx_word = maskbase[static_cast<size_t>(n - 1) * mstride];
  for (int r = 0; r < n; ++r) {
    const int l = n - 1 - r;
    const uint32_t word = nx_word;
    const float tr = nx_tr, tg = nx_tg;
    const float4 cld = nx_cld;
    if (l > 0) {
      const float *q = recs + static_cast<size_t>(l - 1) * kSwRec;
      nx_tg = q[P];
      nx_tr = q[kSwRecTaur + P];
      nx_cld = *reinterpret_cast<const float4 *>(crec + static_cast<size_t>(l - 1) * kSwRec);
      nx_word = maskbase[static_cast<size_t>(l - 1) * mstride];
    }
    const bool cldb = !clear_only && (word & bit) != 0u;
    const float cloud = cldb ? 1.0f : 0.0f;
    const float clear = 1.0f - cloud;
    // clear sky: gas + Rayleigh, no aerosol (sw:6923-6927)
    const float ztau = (tr + tg) + 0.0f;
    const float zom0 = tr + 0.0f * 1.0f;
    const float zgr = zero_over(zom0);  // 0 * 1 * 0 / zom
    const float zom = zom0 / ztau;
    const float v_nd = ztau / mu;
    const float dbtc_nd = exp_lookup(T, v_nd);
    tdbtc_nd = tdbtc_nd * dbtc_nd;
    const float zf = zgr * zgr;
    const float zwf = zom * zf;
    const float d_w = 1.0f - zwf;
    const float ztauc = d_w * ztau;
    const float zomcc = div_or_same(zom - zwf, d_w);
    const float zgcc = div_or_same(zgr - zf, 1.0f - zf);
    // ztauc is ztau exactly when d_w == 1
    const float v_c = d_w == 1.0f ? v_nd : ztauc / mu;
    const float dbtc = d_w == 1.0f ? dbtc_nd : exp_lookup(T, v_c);
    const RT4 c = reftra<kFp64>(T, zgcc, mu, ztauc, zomcc, v_c, dbtc);
    const float4 c_rt = make_float4(c.ref, c.refd, c.tra, c.trad);
    stc[r].rt = c_rt;
    stc[r].dn = make_float4(dbtc, c_tdbt, c_tdn, c_rdnd);
    // the total-sky carry equals the clear-sky one bit for bit (first half of
    // the test whether this slot's total-sky values need storing)
    const bool carry_same =
        same_bits(make_float4(0.0f, t_tdbt, t_tdn, t_rdnd), make_float4(0.0f, c_tdbt, c_tdn, c_rdnd));
    // downward recurrence of vrtqdr (sw:3681-3702) for level r + 1
    {
      const float tdbt_next = c_tdbt * dbtc;
      float tdn_next, rdnd_next;
      if (r == 0) {
        tdn_next = c.tra;
        rdnd_next = c.refd;
      } else {
        const float zreflect = 1.0f / (1.0f - c.refd * c_rdnd);
        tdn_next = c_tdbt * c.tra + c.trad * ((c_tdn - c_tdbt) + c_tdbt * c.ref * c_rdnd) * zreflect;
        rdnd_next = c.refd + c.trad * c.trad * c_rdnd * zreflect;
      }
      c_tdbt = tdbt_next;
      c_tdn = tdn_next;
      c_rdnd = rdnd_next;
    }
    if (!clear_only) {
      float ref, refd, tra, trad, dbt;
      if (cldb) {
        const float tcld = cld.x, wcld = cld.y, gcld = cld.z, taor = cld.w;
        const float tauorig = ztau + taor;
        const float dbtmo_nd = exp_lookup(T, tauorig / mu);
        const float dbt_nd = clear * dbtc_nd + cloud * dbtmo_nd;
        tdbt_nd = tdbt_nd * dbt_nd;
        const float ztauo = ztauc + tcld;
        float zomco = ztauc * zomcc + tcld * wcld;
        const float zgco = (tcld * wcld * gcld + ztauc * zomcc * zgcc) / zomco;
        zomco = zomco / ztauo;
        const float v_o = ztauo / mu;
        const float dbtmo = exp_lookup(T, v_o);
        const RT4 o = reftra<kFp64>(T, zgco, mu, ztauo, zomco, v_o, dbtmo);
        ref = clear * c.ref + cloud * o.ref;
        refd = clear * c.refd + cloud * o.refd;
        tra = clear * c.tra + cloud * o.tra;
        trad = clear * c.trad + cloud * o.trad;
        dbt = clear * dbtc + cloud * dbtmo;
        stt[r].rt = make_float4(ref, refd, tra, trad);
        cloudy_bits |= 1u << (r & 31);
      } else {
        // no cloud in this g-point layer: taor = tcld = 0, so tauorig and
        // ztauo are ztau and ztauc plus zero, and the cloudy reftra is the
        // reference's lrt = false constant set (0, 0, 1, 1)
        const float tauorig = ztau + 0.0f;
        const float dbtmo_nd = __float_as_uint(tauorig) == __float_as_uint(ztau) ? dbtc_nd
                                                                                 : exp_lookup(T, tauorig / mu);
        const float dbt_nd = clear * dbtc_nd + cloud * dbtmo_nd;
        tdbt_nd = tdbt_nd * dbt_nd;
        const float ztauo = ztauc + 0.0f;
        const float dbtmo = __float_as_uint(ztauo) == __float_as_uint(ztauc) ? dbtc : exp_lookup(T, ztauo / mu);
        ref = clear * c.ref + cloud * 0.0f;
        refd = clear * c.refd + cloud * 0.0f;
        tra = clear * c.tra + cloud * 1.0f;
        trad = clear * c.trad + cloud * 1.0f;
        dbt = clear * dbtc + cloud * dbtmo;
      }
      const float4 t_dn = make_float4(dbt, t_tdbt, t_tdn, t_rdnd);
      if (!cldb && carry_same && __float_as_uint(dbt) == __float_as_uint(dbtc) &&
          same_bits(make_float4(ref, refd, tra, trad), c_rt)) {
        same_word |= 1u << (r & 31);
      } else {
        stt[r].dn = t_dn;
      }
      const float tdbt_next = t_tdbt * dbt;
      float tdn_next, rdnd_next;
      if (r == 0) {
        tdn_next = tra;
        rdnd_next = refd;
      } else {
        const float zreflect = 1.0f / (1.0f - refd * t_rdnd);
        tdn_next = t_tdbt * tra + trad * ((t_tdn - t_tdbt) + t_tdbt * ref * t_rdnd) * zreflect;
        rdnd_next = refd + trad * trad * t_rdnd * zreflect;
      }
      t_tdbt = tdbt_next;
      t_tdn = tdn_next;
      t_rdnd = rdnd_next;
    } else {
      tdbt_nd = tdbtc_nd;
    }
    if ((r & 31) == 31 || r == n - 1) {
      S.slotbits[0][r >> 5][threadIdx.x] = cloudy_bits;
      S.slotbits[1][r >> 5][threadIdx.x] = same_word;
      cloudy_bits = 0;
      same_word = 0;
    }
    S.ring[filled][cslot][0][G] = tdbt_nd * zincflx;
    S.ring[filled][cslot][1][G] = tdbtc_nd * zincflx;
    if (++filled == kRing || r == n - 1) {
      sweep_flush(S, filled, 2, dtypes, level0, 1);
      level0 += filled;
      filled = 0;
    }
  }

  // ---- bottom-up pass: upward adding and level fluxes (vrtqdr, sw:3655-3720)
  const int utypes[4] = {0, 1, 2, 3};
  // surface albedos of this g-point's band: direct (albp) and diffuse (albd);
  // the Noah-MP fields, when given, for columns with xland < 1.5 (sw:2519-2530):
  // visible in bands 25-28, near infrared in 16-24 and 29 (sw:2120-2127)
  float albp = C.albedo, albd = C.albedo;
  if (a.in.alswvisdir && ld(a.in.xland + col) < 1.5f) {
    const bool vis = band >= 9 && band <= 12;
    albp = ld((vis ? a.in.alswvisdir : a.in.alswnirdir) + col);
    albd = ld((vis ? a.in.alswvisdif : a.in.alswnirdif) + col);
  }
  float rupc = albp, rupdc = albd;
  float rupt = albp, rupdt = albd;
  level0 = n;
  // surface level n: albedo reflection, no transmission; the recurrence's level-n values
  SwLevel c = {make_float4(albp, albd, 0.0f, 0.0f), make_float4(0.0f, c_tdbt, c_tdn, c_rdnd)};
  SwLevel t = {make_float4(albp, albd, 0.0f, 0.0f), make_float4(0.0f, t_tdbt, t_tdn, t_rdnd)};
  if (clear_only) t = c;
  // stack slot j (layer n - 1 - j) of both paths; a layer without cloud in
  // this g-point has the total-sky mix clear * c + cloud * (0, 0, 1, 1)
  auto load_slot = [&](int j, SwLevel &lc, SwLevel &lt) {
    lc = stc[j];
    if (clear_only || ((S.slotbits[1][j >> 5][threadIdx.x] >> (j & 31)) & 1u) != 0u) {
      lt = lc;
      return;
    }
    lt.dn = stt[j].dn;
    if (((S.slotbits[0][j >> 5][threadIdx.x] >> (j & 31)) & 1u) != 0u) {
      lt.rt = stt[j].rt;
    } else {
      const float clear = 1.0f, cloud = 0.0f;
      lt.rt = make_float4(clear * lc.rt.x + cloud * 0.0f, clear * lc.rt.y + cloud * 0.0f,
                          clear * lc.rt.z + cloud * 1.0f, clear * lc.rt.w + cloud * 1.0f);
    }
  };
  for (int k = n; k >= 0; --k) {
    SwLevel nc = c, nt = t;
    if (k > 0) load_slot(k - 1, nc, nt);
    if (k < n) {
      const float zrc = 1.0f / (1.0f - rupdc * c.rt.y);
      const float nrupc = c.rt.x + c.rt.w * ((c.rt.z - c.dn.x) * rupdc + c.dn.x * rupc) * zrc;
      const float nrupdc = c.rt.y + c.rt.w * c.rt.w * rupdc * zrc;
      rupc = nrupc;
      rupdc = nrupdc;
      if (!clear_only) {
        const float zrt = 1.0f / (1.0f - rupdt * t.rt.y);
        const float nrupt = t.rt.x + t.rt.w * ((t.rt.z - t.dn.x) * rupdt + t.dn.x * rupt) * zrt;
        const float nrupdt = t.rt.y + t.rt.w * t.rt.w * rupdt * zrt;
        rupt = nrupt;
        rupdt = nrupdt;
      }
    }
    // level fluxes; tdbt = dn.y, tdn = dn.z, rdnd = dn.w
    const float zrefc = 1.0f / (1.0f - c.dn.w * rupdc);
    const float fuc = (c.dn.y * rupc + (c.dn.z - c.dn.y) * rupdc) * zrefc;
    const float fdc = c.dn.y + (c.dn.z - c.dn.y + c.dn.y * rupc * c.dn.w) * zrefc;
    float fut = fuc, fdt = fdc;
    if (!clear_only) {
      const float zreft = 1.0f / (1.0f - t.dn.w * rupdt);
      fut = (t.dn.y * rupt + (t.dn.z - t.dn.y) * rupdt) * zreft;
      fdt = t.dn.y + (t.dn.z - t.dn.y + t.dn.y * rupt * t.dn.w) * zreft;
    }
    S.ring[filled][cslot][0][G] = fut * zincflx;
    S.ring[filled][cslot][1][G] = fdt * zincflx;
    S.ring[filled][cslot][2][G] = fuc * zincflx;
    S.ring[filled][cslot][3][G] = fdc * zincflx;
    if (++filled == kRing || k == 0) {
      sweep_flush(S, filled, 4, utypes, level0, -1);
      level0 -= filled;
      filled = 0;
    }
    c = nc;
    t = nt;
  }

  // ---- outputs of the block's live columns (sw:2285-2301, 2536-2719)
  for (int q = threadIdx.x; q < kSweepCols * kMaxLay; q += kSweepThreads) {
    const int cs = q / kMaxLay, l = q - cs * kMaxLay;
    const int uq = u0 + cs;
    if (l >= a.nk || uq >= a.chunk_count || a.chunk_first + uq >= nday) continue;
    sw_layer_output(a, sw_colrecs(a)[uq].C, l, &S.sums[cs][0][0], kMaxLev);
  }
  if (G == 0 && live) sw_column_outputs(a, C, col, &S.sums[cslot][0][0], kMaxLev);
}

}  // namespace

cudaError_t launch_sw_daylist(const SwArgs &a, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(a.nday, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  sw_daylist_kernel<<<(a.ncol + 255) / 256, 256, 0, stream>>>(a);
  return cudaGetLastError();
}

size_t sw_record_floats(int nk, int chunk) {
  return (kSwColRecFloats + static_cast<size_t>(kSwRec + kSwLayerFields) * (nk + 1)) * static_cast<size_t>(chunk);
}

cudaError_t launch_sw_chunk_optics(const Tables &T, const SwArgs &a, cudaStream_t stream) {
  const int threads = 128;
  const int n = a.nk + 1;
  sw_colprep_kernel<<<(a.chunk_count + 3) / 4, threads, 0, stream>>>(T, a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long long layers = static_cast<long long>(a.chunk_count) * n;
  const long long blocks = (layers + threads - 1) / threads;
  sw_layer_kernel<<<static_cast<unsigned>(blocks), threads, 0, stream>>>(T, a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  sw_optics_kernel<<<static_cast<unsigned>(blocks * kSwBands), threads, 0, stream>>>(T, a, static_cast<int>(blocks));
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  sw_source_kernel<<<dim3((a.chunk_count + threads - 1) / threads, kSwBands), threads, 0, stream>>>(T, a);
  return cudaGetLastError();
}

template <bool kFp64>
static cudaError_t launch_sweep(const Tables &T, const SwArgs &a, cudaStream_t stream) {
  if (sizeof(SweepShared) > 48 * 1024) {  // a ring of more levels needs the opt-in
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && !((configured.load() >> dev) & 1ull)) {
      e = cudaFuncSetAttribute(sw_sweep_kernel<kFp64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(sizeof(SweepShared)));
      if (e != cudaSuccess) return e;
      configured.fetch_or(1ull << dev);
    }
  }
  sw_sweep_kernel<kFp64><<<(a.chunk_count + kSweepCols - 1) / kSweepCols, kSweepThreads, sizeof(SweepShared),
                           stream>>>(T, a);
  return cudaGetLastError();
}

cudaError_t launch_sw_chunk_sweep(const Tables &T, const SwArgs &a, cudaStream_t stream) {
  return a.fp64_reftra ? launch_sweep<true>(T, a, stream) : launch_sweep<false>(T, a, stream);
}

}  // namespace rrtmg

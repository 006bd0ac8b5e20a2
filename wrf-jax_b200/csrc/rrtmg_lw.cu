// RRTMG longwave on the GPU: one thread per column, fused from the WRF adapter
// to the theta tendencies.
//
// Reference call: rrtmg_lwrad_wrf_columns (src/wrf_jax/physics/module_ra_rrtmg_lw.py:6789)
// and everything below it: buffer layers (lw:6633-6786), cloud radii and paths
// (common:801-961), inatm (lw:953), setcoef (lw:1175), taumol1..16
// (lw:1597-4684), cldprmc (lw:5725), rtrnmc (lw:5476-5722), broadband sums
// (lw:170-199) and the theta tendency (lw:7040-7057).  McICA masks come from
// rrtmg_mcica.cu.
//
// Layout and schedule.  Inputs are read in place from WRF's (x, z, y) layout,
// where neighbouring columns of a row are adjacent in memory at every level, so
// a warp's loads are coalesced.  Each thread sweeps its column layer by layer:
// the downward sweep visits layers top to bottom and, per layer, evaluates the
// band gas optics for all 140 g-points, advances their radiances and forms the
// level flux as the reference's ordered g-point/band sum; the upward sweep
// re-derives the layer optics bottom to top.  Only the 2 x 140 radiances, the
// downward level fluxes and the buffer-layer profile live in thread-local
// memory; per-layer coefficients stay in registers.
#include "rrtmg_device.cuh"
#include "rrtmg_kernels.h"

namespace rrtmg {
namespace {

constexpr int kNgc[kLwBands] = {10, 12, 16, 14, 16, 8, 12, 8, 12, 6, 8, 8, 4, 2, 2, 2};
constexpr int kGofs[kLwBands] = {0, 10, 22, 38, 52, 68, 76, 88, 96, 108, 114, 122, 130, 134, 136, 138};
// lwdatinit delwave (module_ra_rrtmg_common.py:736-738)
__constant__ float kDelwave[kLwBands] = {340.0f, 150.0f, 130.0f, 70.0f, 120.0f, 160.0f, 100.0f, 100.0f,
                                      210.0f, 90.0f, 320.0f, 280.0f, 170.0f, 130.0f, 220.0f, 650.0f};
// diffusivity fit (lw:5520-5531)
__constant__ float kA0[kLwBands] = {1.66f, 1.55f, 1.58f, 1.66f, 1.54f, 1.454f, 1.89f, 1.33f,
                                 1.668f, 1.66f, 1.66f, 1.66f, 1.66f, 1.66f, 1.66f, 1.66f};
__constant__ float kA1[kLwBands] = {0.0f, 0.25f, 0.22f, 0.0f, 0.13f, 0.446f, -0.10f, 0.40f,
                                 -0.006f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
__constant__ float kA2[kLwBands] = {0.0f, -12.0f, -11.7f, 0.0f, -0.72f, -0.243f, 0.19f, -0.062f,
                                 0.414f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
constexpr float kOneMinus = 1.0f - 1.0e-6f;

// ---------------------------------------------------------------------------
// per-column context
// ---------------------------------------------------------------------------
struct Col {
  int i, j, nk, nlay, ny, nbuf;
  int laytrop;
  float tsfc, semiss, pwvcm;
  float co2, n2o, ch4, cfc11, cfc12;
  int inflg, iceflg, has_reqc, has_reqi, has_reqs, icloud;
  float plev_b[kMaxBuf + 1];   // levels nk .. nlay
  float play_b[kMaxBuf];       // layers nk .. nlay-1
  float tlev_b[kMaxBuf + 1];   // levels nk .. nlay
  float tlay_b[kMaxBuf + 1];   // layers nk-1 .. nlay-1
  float o3_b[kMaxBuf];         // layers nk .. nlay-1
};

struct Layer {
  float pavel, tavel, plev0, plev1, coldry;
  float wx0, wx1, wx2, wx3;
  int jp, jt, jt1, indself, indfor, indminor;
  int trop;  // l < laytrop
  float colh2o, colco2, colo3, coln2o, colco, colch4, colo2, colbrd;
  float fac00, fac01, fac10, fac11;
  float rat_h2oco2, rat_h2oco2_1, rat_h2oo3, rat_h2oo3_1, rat_h2on2o, rat_h2on2o_1;
  float rat_h2och4, rat_h2och4_1, rat_n2oco2, rat_n2oco2_1, rat_o3co2, rat_o3co2_1;
  float selffac, selffrac, forfac, forfrac, minorfrac, scaleminor, scaleminorn2;
  // Planck interpolation (lw:1210-1233): layer, lower and upper level
  int indlay, indlev0, indlev1;
  float tlayfrac, tlev0frac, tlev1frac;
  // cloud path inputs of the layer (common:877-961), zero above the model top
  float cldfrac, clwp, ciwp, cswp, rel, rei, res;
};

__device__ __forceinline__ float in3(const float *p, const Col &C, int k) {
  return ld(p + (static_cast<size_t>(C.i) * C.nk + k) * C.ny + C.j);
}
__device__ __forceinline__ float in3w(const float *p, const Col &C, int k) {
  return ld(p + (static_cast<size_t>(C.i) * (C.nk + 1) + k) * C.ny + C.j);
}

__device__ __forceinline__ float plev_at(const LwArgs &a, const Col &C, int l) {
  return l < C.nk ? pa_to_hpa(in3w(a.in.p8w, C, l)) : C.plev_b[l - C.nk];
}
__device__ __forceinline__ float play_at(const LwArgs &a, const Col &C, int l) {
  return l < C.nk ? pa_to_hpa(in3(a.in.p3d, C, l)) : C.play_b[l - C.nk];
}
__device__ __forceinline__ float tlev_at(const LwArgs &a, const Col &C, int l) {
  return l < C.nk ? in3w(a.in.t8w, C, l) : C.tlev_b[l - C.nk];
}
__device__ __forceinline__ float tlay_at(const LwArgs &a, const Col &C, int l) {
  return l < C.nk - 1 ? in3(a.in.t3d, C, l) : C.tlay_b[l - (C.nk - 1)];
}
__device__ __forceinline__ float h2o_at(const LwArgs &a, const Col &C, int l) {
  const int k = l < C.nk ? l : C.nk - 1;
  return fmaxf(in3(a.in.qv, C, k), 1.0e-12f) * 1.607793f;
}
__device__ __forceinline__ float o3_at(const LwArgs &a, const Col &C, int l) {
  return l < C.nk ? in3(a.in.o3, C, l) : C.o3_b[l - C.nk];
}

// o3data (common:357-404) for one layer bounded by pressures pa > pb
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

// Column set-up: buffer layers above the model top (lw:6633-6786).
// kWarp: called by the 32 lanes of a warp for one column, each lane taking
// every 32nd buffer level (temperature) and buffer layer (ozone) into the
// warp's shared arrays s_tlev / s_o3, which every lane then reads back; the
// values are those of the one-thread form.
template <bool kWarp = false>
__device__ void column_setup(const Tables &T, const LwArgs &a, Col &C, int lane = 0, float *s_tlev = nullptr,
                             float *s_o3 = nullptr) {
  const int nk = C.nk, nlay = C.nlay, nbuf = C.nbuf;
  C.plev_b[0] = pa_to_hpa(in3w(a.in.p8w, C, nk));
  for (int m = 1; m <= nbuf; ++m) C.plev_b[m] = C.plev_b[m - 1] - 4.0f;
  C.plev_b[nbuf] = 0.0f;
  for (int m = 0; m < nbuf; ++m) C.play_b[m] = 0.5f * (C.plev_b[m] + C.plev_b[m + 1]);
  // interface temperatures from the standard profile plus the model-top offset
  auto varint = [&](float p) {
    int count = 0;
    for (int q = 0; q < T.nprof; ++q) count += (ld(T.pprof + q) >= p);
    const int idx = clampi(count - 1, 0, T.nprof - 1);
    const int idx1 = idx + 1 < T.nprof - 1 ? idx + 1 : T.nprof - 1;
    const float p0 = ld(T.pprof + idx), p1 = ld(T.pprof + idx1);
    const float t0 = ld(T.tprof + idx), t1 = ld(T.tprof + idx1);
    const float w = (idx == T.nprof - 1) ? 0.0f : (p - p0) / (p1 - p0);
    return w * (t1 - t0) + t0;
  };
  const float offset = in3w(a.in.t8w, C, nk - 1) - varint(pa_to_hpa(in3w(a.in.p8w, C, nk - 1)));
  if constexpr (kWarp) {
    for (int m = lane; m <= nbuf; m += 32) s_tlev[m] = varint(C.plev_b[m]) + offset;
  } else {
    for (int m = 0; m <= nbuf; ++m) C.tlev_b[m] = varint(C.plev_b[m]) + offset;
  }
  // ozone above the model top (lw:6766-6786)
  const float amdo = 0.603461f;
  const float o3base = in3(a.in.o3, C, nk - 1) -
                       o3data_layer(T, pa_to_hpa(in3w(a.in.p8w, C, nk - 1)), C.plev_b[0]) * amdo;
  auto o3_layer = [&](int m) {
    const float mmr = o3data_layer(T, C.plev_b[m], C.plev_b[m + 1]) * amdo;
    float top = o3base + mmr;
    if (top <= 0.0f) top = mmr;
    return top;
  };
  if constexpr (kWarp) {
    for (int m = lane; m < nbuf; m += 32) s_o3[m] = o3_layer(m);
    __syncwarp();
    for (int m = 0; m <= nbuf; ++m) C.tlev_b[m] = s_tlev[m];
    for (int m = 0; m < nbuf; ++m) C.o3_b[m] = s_o3[m];
  } else {
    for (int m = 0; m < nbuf; ++m) C.o3_b[m] = o3_layer(m);
  }
  // tlay[lev-1] = (tlev[lev] + tlev[lev-1]) / 2 for lev = nk .. nlay
  C.tlay_b[0] = 0.5f * (C.tlev_b[0] + in3w(a.in.t8w, C, nk - 1));
  for (int m = 1; m <= nbuf; ++m) C.tlay_b[m] = 0.5f * (C.tlev_b[m] + C.tlev_b[m - 1]);
  (void)nlay;
}

// Layer coefficients: inatm (lw:953-1035), cloud paths, setcoef (lw:1175-1441).
__device__ __forceinline__ Layer make_layer(const Tables &T, const LwArgs &a, const Col &C, int l) {
  Layer L;
  L.pavel = play_at(a, C, l);
  L.tavel = tlay_at(a, C, l);
  L.plev0 = plev_at(a, C, l);
  L.plev1 = plev_at(a, C, l + 1);
  const float h2o = h2o_at(a, C, l);
  const float o3 = o3_at(a, C, l);
  const float amd = 28.9660f, amw = 18.0160f, avogad = 6.02214199e23f, grav = 9.8066f;
  const float amm = (1.0f - h2o) * amd + h2o * amw;
  const float pm = ((L.plev0 - L.plev1) * 1.0e3f) * avogad;
  float md = 1.0e2f * grav;
  md = md * amm;
  md = md * (1.0f + h2o);
  const float coldry = pm / md;
  L.coldry = coldry;
  const float o2 = 0.209488f;
  float summol = 0.0f;
  summol = summol + C.co2;
  summol = summol + o3;
  summol = summol + C.n2o;
  summol = summol + 0.0f;
  summol = summol + C.ch4;
  summol = summol + o2;
  const float wbrodl = coldry * (1.0f - summol);
  const float wk0 = h2o * coldry, wk1 = C.co2 * coldry, wk2 = o3 * coldry, wk3 = C.n2o * coldry;
  const float wk4 = 0.0f * coldry, wk5 = C.ch4 * coldry, wk6 = o2 * coldry;
  L.wx0 = (0.093e-9f * coldry) * 1.0e-20f;
  L.wx1 = (C.cfc11 * coldry) * 1.0e-20f;
  L.wx2 = (C.cfc12 * coldry) * 1.0e-20f;
  L.wx3 = (0.169e-9f * coldry) * 1.0e-20f;

  // Planck indices
  {
    const float tl = L.tavel - 159.0f;
    L.indlay = clampi(static_cast<int>(tl), 1, 180);
    L.tlayfrac = tl - static_cast<float>(L.indlay);
    const float t0 = tlev_at(a, C, l) - 159.0f;
    L.indlev0 = clampi(static_cast<int>(t0), 1, 180);
    L.tlev0frac = t0 - static_cast<float>(L.indlev0);
    const float t1 = tlev_at(a, C, l + 1) - 159.0f;
    L.indlev1 = clampi(static_cast<int>(t1), 1, 180);
    L.tlev1frac = t1 - static_cast<float>(L.indlev1);
  }
  const float stpfac = 296.0f / 1013.0f;
  const float plog = glibc_logf(T, L.pavel);
  const int jp = clampi(static_cast<int>(36.0f - 5.0f * (plog + 0.04f)), 1, 58);
  const float fp = 5.0f * (ld(T.lw_preflog + jp - 1) - plog);
  const float tf = (L.tavel - ld(T.lw_tref + jp - 1)) / 15.0f;
  const int jt = clampi(static_cast<int>(3.0f + tf), 1, 4);
  const float ft = tf - static_cast<float>(jt - 3);
  const float tf1 = (L.tavel - ld(T.lw_tref + jp)) / 15.0f;
  const int jt1 = clampi(static_cast<int>(3.0f + tf1), 1, 4);
  const float ft1 = tf1 - static_cast<float>(jt1 - 3);
  const float water = wk0 / coldry;
  const float scalefac = (L.pavel * stpfac) / L.tavel;
  const int trop = plog > 4.56f;
  L.trop = l < C.laytrop;
  const float forfac_base = scalefac / (1.0f + water);
  const float ftf = (332.0f - L.tavel) / 36.0f;
  const int indfor_t = clampi(static_cast<int>(ftf), 1, 2);
  const float forfrac_t = ftf - static_cast<float>(indfor_t);
  const float fsf = (L.tavel - 188.0f) / 36.0f;
  L.indfor = trop ? indfor_t : 3;
  L.forfrac = trop ? forfrac_t : fsf - 1.0f;
  const float fself = (L.tavel - 188.0f) / 7.2f;
  const int indself_t = clampi(static_cast<int>(fself) - 7, 1, 9);
  const float selffrac_t = fself - static_cast<float>(indself_t + 7);
  L.indself = trop ? indself_t : 0;
  L.selffrac = trop ? selffrac_t : 0.0f;
  L.scaleminor = L.pavel / L.tavel;
  L.scaleminorn2 = L.scaleminor * (wbrodl / (coldry + wk0));
  const float fminor = (L.tavel - 180.8f) / 7.2f;
  L.indminor = clampi(static_cast<int>(fminor), 1, 18);
  L.minorfrac = fminor - static_cast<float>(L.indminor);
  const float tiny = 1.0e-20f;
  const float fallback = 1.0e-32f * coldry;
  L.colh2o = tiny * wk0;
  L.colco2 = tiny * wk1;
  L.colo3 = tiny * wk2;
  L.coln2o = tiny * wk3;
  L.colco = tiny * wk4;
  L.colch4 = tiny * wk5;
  L.colo2 = tiny * wk6;
  if (L.colco2 == 0.0f) L.colco2 = fallback;
  if (L.colo3 == 0.0f) L.colo3 = fallback;
  if (L.coln2o == 0.0f) L.coln2o = fallback;
  if (L.colco == 0.0f) L.colco = fallback;
  if (L.colch4 == 0.0f) L.colch4 = fallback;
  L.colbrd = tiny * wbrodl;
  const float *chi = T.chi_mls;
  const int j0 = jp - 1, j1 = jp;
  auto CHI = [&](int gas, int lev) { return ld(chi + gas * 59 + lev); };
  L.rat_h2oco2 = CHI(0, j0) / CHI(1, j0);
  L.rat_h2oco2_1 = CHI(0, j1) / CHI(1, j1);
  L.rat_h2oo3 = trop ? CHI(0, j0) / CHI(2, j0) : 0.0f;
  L.rat_h2oo3_1 = trop ? CHI(0, j1) / CHI(2, j1) : 0.0f;
  L.rat_h2on2o = trop ? CHI(0, j0) / CHI(3, j0) : 0.0f;
  L.rat_h2on2o_1 = trop ? CHI(0, j1) / CHI(3, j1) : 0.0f;
  L.rat_h2och4 = trop ? CHI(0, j0) / CHI(5, j0) : 0.0f;
  L.rat_h2och4_1 = trop ? CHI(0, j1) / CHI(5, j1) : 0.0f;
  L.rat_n2oco2 = trop ? CHI(3, j0) / CHI(1, j0) : 0.0f;
  L.rat_n2oco2_1 = trop ? CHI(3, j1) / CHI(1, j1) : 0.0f;
  L.rat_o3co2 = trop ? 0.0f : CHI(2, j0) / CHI(1, j0);
  L.rat_o3co2_1 = trop ? 0.0f : CHI(2, j1) / CHI(1, j1);
  const float compfp = 1.0f - fp;
  L.fac10 = compfp * ft;
  L.fac00 = compfp * (1.0f - ft);
  L.fac11 = fp * ft1;
  L.fac01 = fp * (1.0f - ft1);
  L.selffac = L.colh2o * (water * forfac_base);
  L.forfac = L.colh2o * forfac_base;
  L.jp = jp;
  L.jt = jt;
  L.jt1 = jt1;

  // cloud radii and in-cloud paths (common:801-961); zero above the model top
  L.cldfrac = 0.0f; L.clwp = 0.0f; L.ciwp = 0.0f; L.cswp = 0.0f;
  L.rel = 10.0f; L.rei = 10.0f; L.res = 10.0f;
  if (l < C.nk) {
    const float t = in3(a.in.t3d, C, l);
    const float cldfra = in3(a.in.cldfra, C, l);
    float qc = fmaxf(in3(a.in.qc, C, l), 0.0f), qi = fmaxf(in3(a.in.qi, C, l), 0.0f);
    float qs = fmaxf(in3(a.in.qs, C, l), 0.0f);
    const float xland = ld(a.in.xland + C.i * C.ny + C.j);
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
    const float temp = L.tavel;
    const float dp = L.plev0 - L.plev1;
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
    const float xice = ld(a.in.xice + C.i * C.ny + C.j), snow = ld(a.in.snow + C.i * C.ny + C.j);
    const float landm = 2.0f - xland, snowh = 0.001f * snow;
    const float rocean = 14.0f, rland = 8.0f, rice = 14.0f;
    float rel = rland + (rocean - rland) * fminf(1.0f, fmaxf(0.0f, (273.16f - temp) * 0.05f));
    rel = rel + (rocean - rel) * fminf(1.0f, fmaxf(0.0f, snowh * 10.0f));
    rel = rel + (rocean - rel) * fminf(1.0f, fmaxf(0.0f, 1.0f - landm));
    rel = rel + (rice - rel) * fminf(1.0f, fmaxf(0.0f, xice));
    float rei = retab_interp(T, temp, 94);
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
// taumol helpers (lw:108-168, 1444-1594)
// ---------------------------------------------------------------------------
struct Spec {
  float sc, sp, fs;
  int js;
};

__device__ __forceinline__ Spec specint(float primary, float ratio, float secondary, float scale) {
  Spec s;
  s.sc = primary + ratio * secondary;
  const float q = primary / s.sc;
  s.sp = q > kOneMinus ? kOneMinus : q;
  const float sm = scale * s.sp;
  s.js = 1 + static_cast<int>(sm);
  s.fs = sm - floorf(sm);
  return s;
}

struct Edge {
  float f000, f100, f200, f010, f110, f210;
  int mode;  // 0 mid, 1 low, 2 high
};

__device__ __forceinline__ Edge edge_factors(float specparm, float fs, float fa, float fb) {
  Edge e;
  if (specparm < 0.125f || specparm > 0.875f) {
    e.mode = specparm < 0.125f ? 1 : 2;
    const float p = e.mode == 1 ? fs - 1.0f : 0.0f - fs;
    const float p2 = p * p, p4 = p2 * p2;
    const float fk0 = p4, fk1 = (1.0f - p) - 2.0f * p4, fk2 = p + p4;
    e.f000 = fk0 * fa; e.f100 = fk1 * fa; e.f200 = fk2 * fa;
    e.f010 = fk0 * fb; e.f110 = fk1 * fb; e.f210 = fk2 * fb;
  } else {
    e.mode = 0;
    e.f000 = (1.0f - fs) * fa; e.f100 = fs * fa; e.f200 = 0.0f;
    e.f010 = (1.0f - fs) * fb; e.f110 = fs * fb; e.f210 = 0.0f;
  }
  return e;
}

__device__ __forceinline__ float safe(const float *tab, int rows, int ngc, int r, int g) {
  return ld(tab + clampi(r, 0, rows - 1) * ngc + g);
}

__device__ __forceinline__ float edge_major(const float *tab, int rows, int ngc, int base, const Edge &e, int g) {
  float s;
  if (e.mode == 1) {
    s = e.f000 * safe(tab, rows, ngc, base, g);
    s = s + e.f100 * safe(tab, rows, ngc, base + 1, g);
    s = s + e.f200 * safe(tab, rows, ngc, base + 2, g);
    s = s + e.f010 * safe(tab, rows, ngc, base + 9, g);
    s = s + e.f110 * safe(tab, rows, ngc, base + 10, g);
    s = s + e.f210 * safe(tab, rows, ngc, base + 11, g);
  } else if (e.mode == 2) {
    s = e.f200 * safe(tab, rows, ngc, base - 1, g);
    s = s + e.f100 * safe(tab, rows, ngc, base, g);
    s = s + e.f000 * safe(tab, rows, ngc, base + 1, g);
    s = s + e.f210 * safe(tab, rows, ngc, base + 8, g);
    s = s + e.f110 * safe(tab, rows, ngc, base + 9, g);
    s = s + e.f010 * safe(tab, rows, ngc, base + 10, g);
  } else {
    s = e.f000 * safe(tab, rows, ngc, base, g);
    s = s + e.f100 * safe(tab, rows, ngc, base + 1, g);
    s = s + e.f010 * safe(tab, rows, ngc, base + 9, g);
    s = s + e.f110 * safe(tab, rows, ngc, base + 10, g);
  }
  return s;
}

__device__ __forceinline__ float major4(const float *tab, int ngc, int i0, int i1, int g, const Layer &L) {
  float s = L.fac00 * ld(tab + i0 * ngc + g);
  s = s + L.fac10 * ld(tab + (i0 + 1) * ngc + g);
  s = s + L.fac01 * ld(tab + i1 * ngc + g);
  s = s + L.fac11 * ld(tab + (i1 + 1) * ngc + g);
  return s;
}

__device__ __forceinline__ float strat_binary(const float *tab, int rows, int ngc, int ind, int g, float fs, float fa, float fb) {
  const float comp = 1.0f - fs;
  const float s000 = comp * fa, s100 = fs * fa, s010 = comp * fb, s110 = fs * fb;
  float s = s000 * safe(tab, rows, ngc, ind, g);
  s = s + s100 * safe(tab, rows, ngc, ind + 1, g);
  s = s + s010 * safe(tab, rows, ngc, ind + 5, g);
  s = s + s110 * safe(tab, rows, ngc, ind + 6, g);
  return s;
}

__device__ __forceinline__ int ind5(int v, int rows) { return clampi(v, 0, rows - 2); }

__device__ __forceinline__ float lin_minor(const float *tab, int ngc, int indminor, float frac, int g) {
  const int m0 = clampi(indminor - 1, 0, 17);
  return interpf(ld(tab + m0 * ngc + g), ld(tab + (m0 + 1) * ngc + g), frac);
}

__device__ __forceinline__ float spec_minor(const float *tab, int nspec, int ngc, int jm, float fm, int indminor, float frac, int g) {
  const int m0 = clampi(indminor - 1, 0, 17);
  const int j0 = clampi(jm - 1, 0, nspec - 2);
  const float a = interpf(ld(tab + (j0 * 19 + m0) * ngc + g), ld(tab + ((j0 + 1) * 19 + m0) * ngc + g), fm);
  const float b = interpf(ld(tab + (j0 * 19 + m0 + 1) * ngc + g), ld(tab + ((j0 + 1) * 19 + m0 + 1) * ngc + g), fm);
  return interpf(a, b, frac);
}

__device__ __forceinline__ float self_tau(const LwBand &B, int ngc, const Layer &L, int g) {
  const int i0 = clampi(L.indself - 1, 0, 8);
  return L.selffac * interpf(ld(B.selfref + i0 * ngc + g), ld(B.selfref + (i0 + 1) * ngc + g), L.selffrac);
}

__device__ __forceinline__ float for_tau(const LwBand &B, int ngc, const Layer &L, int g) {
  const int i0 = clampi(L.indfor - 1, 0, 2);
  return L.forfac * interpf(ld(B.forref + i0 * ngc + g), ld(B.forref + (i0 + 1) * ngc + g), L.forfrac);
}

__device__ __forceinline__ float frac_interp(const float *tab, int ncols, int jpl, float fpl, int g) {
  const int j0 = clampi(jpl - 1, 0, ncols - 2);
  return interpf(ld(tab + g * ncols + j0), ld(tab + g * ncols + j0 + 1), fpl);
}

__device__ __forceinline__ float chi(const Tables &T, int gas, int lev) { return ld(T.chi_mls + gas * 59 + lev); }

// ---------------------------------------------------------------------------
// Gas optics of band B at one layer: taug and Planck fractions for its g-points
// (taugb1..taugb16, lw:1597-4684).
// ---------------------------------------------------------------------------
template <int B>
__device__ __forceinline__ void taumol(const Tables &T, const Layer &L, float *taug, float *fracs) {
  constexpr int ngc = kNgc[B];
  const LwBand &K = T.lw[B];
  const int jp = L.jp, jt = L.jt, jt1 = L.jt1;
  const bool trop = L.trop;
  if constexpr (B == 0 || B == 1 || B == 9 || B == 10 || B == 13) {
    // single-species bands 1, 2, 10, 11, 14
    const int i0 = trop ? ind5((jp - 1) * 5 + (jt - 1), K.ka_rows) : ind5((jp - 13) * 5 + (jt - 1), K.kb_rows);
    const int i1 = trop ? ind5(jp * 5 + (jt1 - 1), K.ka_rows) : ind5((jp - 12) * 5 + (jt1 - 1), K.kb_rows);
    const float *tab = trop ? K.ka : K.kb;
    float corr = 1.0f, scalen2 = 0.0f, scaleo2 = 0.0f;
    if constexpr (B == 0) {
      corr = trop ? (L.pavel < 250.0f ? 1.0f - ((0.15f * (250.0f - L.pavel)) / 154.4f) : 1.0f)
                  : 1.0f - 0.15f * (L.pavel / 95.6f);
      scalen2 = L.colbrd * L.scaleminorn2;
    }
    if constexpr (B == 1) corr = 1.0f - ((0.05f * (L.pavel - 100.0f)) / 900.0f);
    if constexpr (B == 10) scaleo2 = L.colo2 * L.scaleminor;
#pragma unroll
    for (int g = 0; g < ngc; ++g) {
      const float major = major4(tab, ngc, i0, i1, g, L);
      float tau;
      if constexpr (B == 13) {
        tau = trop ? (L.colco2 * major + self_tau(K, ngc, L, g)) + for_tau(K, ngc, L, g) : L.colco2 * major;
      } else {
        if (trop) {
          tau = (L.colh2o * major + self_tau(K, ngc, L, g)) + for_tau(K, ngc, L, g);
        } else {
          tau = L.colh2o * major + for_tau(K, ngc, L, g);
        }
        if constexpr (B == 0) {
          const float taun2 = scalen2 * lin_minor(trop ? K.ka_mn2 : K.kb_mn2, ngc, L.indminor, L.minorfrac, g);
          tau = corr * (tau + taun2);
        }
        if constexpr (B == 1) {
          if (trop) tau = corr * tau;
        }
        if constexpr (B == 10) tau = tau + scaleo2 * lin_minor(trop ? K.ka_mo2 : K.kb_mo2, ngc, L.indminor, L.minorfrac, g);
      }
      taug[g] = tau;
      fracs[g] = ld((trop ? K.fracrefa : K.fracrefb) + g);
    }
  } else if constexpr (B == 2 || B == 3 || B == 4) {
    // bands 3, 4, 5: binary species in both regions
    float adjcoln2o = L.coln2o;
    if constexpr (B == 2) {
      const float chi_n2o = L.coln2o / L.coldry;
      const float chi_ref = chi(T, 3, clampi(jp, 0, 58));
      const float ratn2o = (1.0e20f * chi_n2o) / chi_ref;
      if (ratn2o > 1.5f) {
        const float adjfac = 0.5f + powf(ratn2o - 0.5f, 0.65f);
        adjcoln2o = ((adjfac * chi_ref) * L.coldry) * 1.0e-20f;
      }
    }
    if (trop) {
      float rpa, rma = 0.0f;
      if constexpr (B == 2) { rpa = chi(T, 0, 8) / chi(T, 1, 8); rma = chi(T, 0, 2) / chi(T, 1, 2); }
      if constexpr (B == 3) { rpa = chi(T, 0, 10) / chi(T, 1, 10); }
      if constexpr (B == 4) { rpa = chi(T, 0, 4) / chi(T, 1, 4); rma = chi(T, 0, 6) / chi(T, 1, 6); }
      const Spec s0 = specint(L.colh2o, L.rat_h2oco2, L.colco2, 8.0f);
      const Spec s1 = specint(L.colh2o, L.rat_h2oco2_1, L.colco2, 8.0f);
      const Spec sm = specint(L.colh2o, rma, L.colco2, 8.0f);
      const Spec sp = specint(L.colh2o, rpa, L.colco2, 8.0f);
      const int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
      const int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
      const Edge e0 = edge_factors(s0.sp, s0.fs, L.fac00, L.fac10);
      const Edge e1 = edge_factors(s1.sp, s1.fs, L.fac01, L.fac11);
#pragma unroll
      for (int g = 0; g < ngc; ++g) {
        const float tm0 = s0.sc * edge_major(K.ka, K.ka_rows, ngc, b0, e0, g);
        const float tm1 = s1.sc * edge_major(K.ka, K.ka_rows, ngc, b1, e1, g);
        float tau = ((tm0 + tm1) + self_tau(K, ngc, L, g)) + for_tau(K, ngc, L, g);
        if constexpr (B == 2) tau = tau + adjcoln2o * spec_minor(K.ka_mn2o, 9, ngc, sm.js, sm.fs, L.indminor, L.minorfrac, g);
        if constexpr (B == 4) {
          tau = tau + spec_minor(K.ka_mo3, 9, ngc, sm.js, sm.fs, L.indminor, L.minorfrac, g) * L.colo3;
          tau = tau + L.wx0 * ld(K.ccl4 + g);
        }
        taug[g] = tau;
        fracs[g] = frac_interp(K.fracrefa, 9, sp.js, sp.fs, g);
      }
    } else {
      float prim, r0, r1, rpb, rmb = 0.0f;
      if constexpr (B == 2) {
        prim = L.colh2o; r0 = L.rat_h2oco2; r1 = L.rat_h2oco2_1;
        rpb = chi(T, 0, 12) / chi(T, 1, 12); rmb = chi(T, 0, 12) / chi(T, 1, 12);
      } else {
        prim = L.colo3; r0 = L.rat_o3co2; r1 = L.rat_o3co2_1;
        rpb = B == 3 ? chi(T, 2, 12) / chi(T, 1, 12) : chi(T, 2, 42) / chi(T, 1, 42);
      }
      const Spec s0 = specint(prim, r0, L.colco2, 4.0f);
      const Spec s1 = specint(prim, r1, L.colco2, 4.0f);
      const Spec sm = specint(prim, rmb, L.colco2, 4.0f);
      const Spec sp = specint(prim, rpb, L.colco2, 4.0f);
      const int i0 = (jp - 13) * 25 + (jt - 1) * 5 + (s0.js - 1);
      const int i1 = (jp - 12) * 25 + (jt1 - 1) * 5 + (s1.js - 1);
      constexpr float kCorr4[14] = {1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 0.92f, 0.88f, 1.07f, 1.1f, 0.99f, 0.88f, 0.943f};
#pragma unroll
      for (int g = 0; g < ngc; ++g) {
        const float m0 = s0.sc * strat_binary(K.kb, K.kb_rows, ngc, i0, g, s0.fs, L.fac00, L.fac10);
        const float m1 = s1.sc * strat_binary(K.kb, K.kb_rows, ngc, i1, g, s1.fs, L.fac01, L.fac11);
        float tau;
        if constexpr (B == 2) tau = ((m0 + m1) + for_tau(K, ngc, L, g)) + adjcoln2o * spec_minor(K.kb_mn2o, 5, ngc, sm.js, sm.fs, L.indminor, L.minorfrac, g);
        if constexpr (B == 3) tau = (m0 + m1) * kCorr4[g];
        if constexpr (B == 4) tau = (m0 + m1) + L.wx0 * ld(K.ccl4 + g);
        taug[g] = tau;
        fracs[g] = frac_interp(K.fracrefb, 5, sp.js, sp.fs, g);
      }
      (void)sm;
    }
  } else if constexpr (B == 5) {
    const float chi_co2 = L.colco2 / L.coldry;
    const float chi_ref = chi(T, 1, clampi(jp, 0, 58));
    const float ratco2 = 1.0e20f * chi_co2 / chi_ref;
    float adjcolco2 = L.colco2;
    if (ratco2 > 3.0f) {
      const float adjfac = 2.0f + powf(fmaxf(ratco2 - 2.0f, 0.0f), 0.77f);
      adjcolco2 = adjfac * chi_ref * L.coldry * 1.0e-20f;
    }
    const int i0 = ind5((jp - 1) * 5 + (jt - 1), K.ka_rows), i1 = ind5(jp * 5 + (jt1 - 1), K.ka_rows);
#pragma unroll
    for (int g = 0; g < ngc; ++g) {
      const float cfc11 = L.wx1 * ld(K.cfc11adj + g);
      const float cfc12 = L.wx2 * ld(K.cfc12 + g);
      float tau;
      if (trop) {
        const float major = major4(K.ka, ngc, i0, i1, g, L);
        const float absco2 = lin_minor(K.ka_mco2, ngc, L.indminor, L.minorfrac, g);
        tau = ((((L.colh2o * major + self_tau(K, ngc, L, g)) + for_tau(K, ngc, L, g)) + adjcolco2 * absco2) + cfc11) + cfc12;
      } else {
        tau = cfc11 + cfc12;
      }
      taug[g] = tau;
      fracs[g] = ld(K.fracrefa + g);
    }
  } else if constexpr (B == 6) {
    constexpr float kCorr7[12] = {1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 0.92f, 0.88f, 1.07f, 1.1f, 0.99f, 0.855f, 1.0f};
    const float chi_co2 = L.colco2 / L.coldry;
    const float chi_ref = chi(T, 1, clampi(jp, 0, 58));
    const float ratco2 = (1.0e20f * chi_co2) / chi_ref;
    if (trop) {
      const float rpa = chi(T, 0, 2) / chi(T, 2, 2);
      const Spec s0 = specint(L.colh2o, L.rat_h2oo3, L.colo3, 8.0f);
      const Spec s1 = specint(L.colh2o, L.rat_h2oo3_1, L.colo3, 8.0f);
      const Spec sm = specint(L.colh2o, rpa, L.colo3, 8.0f);
      const Spec sp = sm;
      float adjcolco2 = L.colco2;
      if (ratco2 > 3.0f) {
        const float adjfac = 3.0f + powf(ratco2 - 3.0f, 0.79f);
        adjcolco2 = ((adjfac * chi_ref) * L.coldry) * 1.0e-20f;
      }
      const int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
      const int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
      const Edge e0 = edge_factors(s0.sp, s0.fs, L.fac00, L.fac10);
      const Edge e1 = edge_factors(s1.sp, s1.fs, L.fac01, L.fac11);
#pragma unroll
      for (int g = 0; g < ngc; ++g) {
        const float tm0 = s0.sc * edge_major(K.ka, K.ka_rows, ngc, b0, e0, g);
        const float tm1 = s1.sc * edge_major(K.ka, K.ka_rows, ngc, b1, e1, g);
        const float absco2 = spec_minor(K.ka_mco2, 9, ngc, sm.js, sm.fs, L.indminor, L.minorfrac, g);
        taug[g] = (((tm0 + tm1) + self_tau(K, ngc, L, g)) + for_tau(K, ngc, L, g)) + adjcolco2 * absco2;
        fracs[g] = frac_interp(K.fracrefa, 9, sp.js, sp.fs, g);
      }
    } else {
      float adjcolco2 = L.colco2;
      if (ratco2 > 3.0f) {
        const float adjfac = 2.0f + powf(ratco2 - 2.0f, 0.79f);
        adjcolco2 = ((adjfac * chi_ref) * L.coldry) * 1.0e-20f;
      }
      const int i0 = ind5((jp - 13) * 5 + (jt - 1), K.kb_rows), i1 = ind5((jp - 12) * 5 + (jt1 - 1), K.kb_rows);
#pragma unroll
      for (int g = 0; g < ngc; ++g) {
        const float major = major4(K.kb, ngc, i0, i1, g, L);
        const float absco2 = lin_minor(K.kb_mco2, ngc, L.indminor, L.minorfrac, g);
        taug[g] = (L.colo3 * major + adjcolco2 * absco2) * kCorr7[g];
        fracs[g] = ld(K.fracrefb + g);
      }
    }
  } else if constexpr (B == 7) {
    const float chi_co2 = L.colco2 / L.coldry;
    const float chi_ref = chi(T, 1, clampi(jp, 0, 58));
    const float ratco2 = (1.0e20f * chi_co2) / chi_ref;
    float adjcolco2 = L.colco2;
    if (ratco2 > 3.0f) {
      const float adjfac = 2.0f + powf(fmaxf(ratco2 - 2.0f, 0.0f), 0.65f);
      adjcolco2 = ((adjfac * chi_ref) * L.coldry) * 1.0e-20f;
    }
#pragma unroll
    for (int g = 0; g < ngc; ++g) {
      const float cfc12 = L.wx2 * ld(K.cfc12 + g);
      const float cfc22 = L.wx3 * ld(K.cfc22adj + g);
      float tau;
      if (trop) {
        const int i0 = ind5((jp - 1) * 5 + (jt - 1), K.ka_rows), i1 = ind5(jp * 5 + (jt1 - 1), K.ka_rows);
        const float major = major4(K.ka, ngc, i0, i1, g, L);
        tau = L.colh2o * major + self_tau(K, ngc, L, g);
        tau = tau + for_tau(K, ngc, L, g);
        tau = tau + adjcolco2 * lin_minor(K.ka_mco2, ngc, L.indminor, L.minorfrac, g);
        tau = tau + L.colo3 * lin_minor(K.ka_mo3, ngc, L.indminor, L.minorfrac, g);
        tau = tau + L.coln2o * lin_minor(K.ka_mn2o, ngc, L.indminor, L.minorfrac, g);
        tau = (tau + cfc12) + cfc22;
        fracs[g] = ld(K.fracrefa + g);
      } else {
        const int i0 = ind5((jp - 13) * 5 + (jt - 1), K.kb_rows), i1 = ind5((jp - 12) * 5 + (jt1 - 1), K.kb_rows);
        const float major = major4(K.kb, ngc, i0, i1, g, L);
        tau = L.colo3 * major + adjcolco2 * lin_minor(K.kb_mco2, ngc, L.indminor, L.minorfrac, g);
        tau = tau + L.coln2o * lin_minor(K.kb_mn2o, ngc, L.indminor, L.minorfrac, g);
        tau = (tau + cfc12) + cfc22;
        fracs[g] = ld(K.fracrefb + g);
      }
      taug[g] = tau;
    }
  } else if constexpr (B == 8) {
    const float chi_n2o = L.coln2o / L.coldry;
    const float chi_ref = chi(T, 3, clampi(jp, 0, 58));
    const float ratn2o = (1.0e20f * chi_n2o) / chi_ref;
    float adjcoln2o = L.coln2o;
    if (ratn2o > 1.5f) {
      const float adjfac = 0.5f + powf(ratn2o - 0.5f, 0.65f);
      adjcoln2o = ((adjfac * chi_ref) * L.coldry) * 1.0e-20f;
    }
    if (trop) {
      const float rpa = chi(T, 0, 8) / chi(T, 5, 8), rma = chi(T, 0, 2) / chi(T, 5, 2);
      const Spec s0 = specint(L.colh2o, L.rat_h2och4, L.colch4, 8.0f);
      const Spec s1 = specint(L.colh2o, L.rat_h2och4_1, L.colch4, 8.0f);
      const Spec sm = specint(L.colh2o, rma, L.colch4, 8.0f);
      const Spec sp = specint(L.colh2o, rpa, L.colch4, 8.0f);
      const int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
      const int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
      const Edge e0 = edge_factors(s0.sp, s0.fs, L.fac00, L.fac10);
      const Edge e1 = edge_factors(s1.sp, s1.fs, L.fac01, L.fac11);
#pragma unroll
      for (int g = 0; g < ngc; ++g) {
        const float tm0 = s0.sc * edge_major(K.ka, K.ka_rows, ngc, b0, e0, g);
        const float tm1 = s1.sc * edge_major(K.ka, K.ka_rows, ngc, b1, e1, g);
        const float absn2o = spec_minor(K.ka_mn2o, 9, ngc, sm.js, sm.fs, L.indminor, L.minorfrac, g);
        taug[g] = (((tm0 + tm1) + self_tau(K, ngc, L, g)) + for_tau(K, ngc, L, g)) + adjcoln2o * absn2o;
        fracs[g] = frac_interp(K.fracrefa, 9, sp.js, sp.fs, g);
      }
    } else {
      const int i0 = ind5((jp - 13) * 5 + (jt - 1), K.kb_rows), i1 = ind5((jp - 12) * 5 + (jt1 - 1), K.kb_rows);
#pragma unroll
      for (int g = 0; g < ngc; ++g) {
        const float major = major4(K.kb, ngc, i0, i1, g, L);
        taug[g] = L.colch4 * major + adjcoln2o * lin_minor(K.kb_mn2o, ngc, L.indminor, L.minorfrac, g);
        fracs[g] = ld(K.fracrefb + g);
      }
    }
  } else if constexpr (B == 11 || B == 14 || B == 15) {
    // bands 12, 15, 16: binary species in the troposphere only
    if (trop) {
      float prim, r0, r1, sec, rpa, rma = 0.0f;
      if constexpr (B == 11) {
        prim = L.colh2o; r0 = L.rat_h2oco2; r1 = L.rat_h2oco2_1; sec = L.colco2;
        rpa = chi(T, 0, 9) / chi(T, 1, 9);
      }
      if constexpr (B == 14) {
        prim = L.coln2o; r0 = L.rat_n2oco2; r1 = L.rat_n2oco2_1; sec = L.colco2;
        rpa = chi(T, 3, 0) / chi(T, 1, 0); rma = rpa;
      }
      if constexpr (B == 15) {
        prim = L.colh2o; r0 = L.rat_h2och4; r1 = L.rat_h2och4_1; sec = L.colch4;
        rpa = chi(T, 0, 5) / chi(T, 5, 5);
      }
      const Spec s0 = specint(prim, r0, sec, 8.0f);
      const Spec s1 = specint(prim, r1, sec, 8.0f);
      const Spec sm = specint(prim, rma, sec, 8.0f);
      const Spec sp = specint(prim, rpa, sec, 8.0f);
      const int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
      const int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
      const Edge e0 = edge_factors(s0.sp, s0.fs, L.fac00, L.fac10);
      const Edge e1 = edge_factors(s1.sp, s1.fs, L.fac01, L.fac11);
      const float scalen2 = L.colbrd * L.scaleminor;
#pragma unroll
      for (int g = 0; g < ngc; ++g) {
        const float tm0 = s0.sc * edge_major(K.ka, K.ka_rows, ngc, b0, e0, g);
        const float tm1 = s1.sc * edge_major(K.ka, K.ka_rows, ngc, b1, e1, g);
        float tau = ((tm0 + tm1) + self_tau(K, ngc, L, g)) + for_tau(K, ngc, L, g);
        if constexpr (B == 14) tau = tau + scalen2 * spec_minor(K.ka_mn2, 9, ngc, sm.js, sm.fs, L.indminor, L.minorfrac, g);
        taug[g] = tau;
        fracs[g] = frac_interp(K.fracrefa, 9, sp.js, sp.fs, g);
      }
      (void)sm;
      (void)scalen2;
    } else {
#pragma unroll
      for (int g = 0; g < ngc; ++g) {
        if constexpr (B == 15) {
          // nspb(16) = 0: both base rows collapse to 0 (lw:4660-4663)
          taug[g] = L.colch4 * major4(K.kb, ngc, 0, 0, g, L);
          fracs[g] = ld(K.fracrefb + g);
        } else {
          taug[g] = 0.0f;
          fracs[g] = 0.0f;
        }
      }
    }
  } else if constexpr (B == 12) {
    if (trop) {
      const float rpa = chi(T, 0, 4) / chi(T, 3, 4), rma = chi(T, 0, 0) / chi(T, 3, 0), rma3 = chi(T, 0, 2) / chi(T, 3, 2);
      const Spec s0 = specint(L.colh2o, L.rat_h2on2o, L.coln2o, 8.0f);
      const Spec s1 = specint(L.colh2o, L.rat_h2on2o_1, L.coln2o, 8.0f);
      const Spec sm = specint(L.colh2o, rma, L.coln2o, 8.0f);
      const float chi_co2 = L.colco2 / L.coldry;
      const float co2ref = 3.55e-4f;
      const float ratco2 = (1.0e20f * chi_co2) / co2ref;
      float adjcolco2 = L.colco2;
      if (ratco2 > 3.0f) {
        const float adjfac = 2.0f + powf(ratco2 - 2.0f, 0.68f);
        adjcolco2 = ((adjfac * co2ref) * L.coldry) * 1.0e-20f;
      }
      const Spec sc = specint(L.colh2o, rma3, L.coln2o, 8.0f);
      const Spec sp = specint(L.colh2o, rpa, L.coln2o, 8.0f);
      const int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
      const int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
      const Edge e0 = edge_factors(s0.sp, s0.fs, L.fac00, L.fac10);
      const Edge e1 = edge_factors(s1.sp, s1.fs, L.fac01, L.fac11);
#pragma unroll
      for (int g = 0; g < ngc; ++g) {
        const float tm0 = s0.sc * edge_major(K.ka, K.ka_rows, ngc, b0, e0, g);
        const float tm1 = s1.sc * edge_major(K.ka, K.ka_rows, ngc, b1, e1, g);
        const float absco2 = spec_minor(K.ka_mco2, 9, ngc, sm.js, sm.fs, L.indminor, L.minorfrac, g);
        const float absco = spec_minor(K.ka_mco, 9, ngc, sc.js, sc.fs, L.indminor, L.minorfrac, g);
        const float tau = (((tm0 + tm1) + self_tau(K, ngc, L, g)) + for_tau(K, ngc, L, g)) + adjcolco2 * absco2;
        taug[g] = tau + L.colco * absco;
        fracs[g] = frac_interp(K.fracrefa, 9, sp.js, sp.fs, g);
      }
    } else {
#pragma unroll
      for (int g = 0; g < ngc; ++g) {
        taug[g] = L.colo3 * lin_minor(K.kb_mo3, ngc, L.indminor, L.minorfrac, g);
        fracs[g] = ld(K.fracrefb + g);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Cloud optical depth of band B for a cloudy g-point of a layer
// (cldprmc, lw:5725-5830; ice options >= 3, liquid option 1)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float cloud_tau(const Tables &T, const Layer &L, int band, int iceflag, bool &active) {
  const float ciwp = L.ciwp, clwp = L.clwp, cswp = L.cswp;
  const float cwp = (ciwp + clwp) + cswp;
  active = cwp >= 1.0e-20f;
  const float factor = (L.rei - 2.0f) / 3.0f;
  int index = static_cast<int>(factor);
  if (index == 46) index = 45;
  const float fint = factor - static_cast<float>(index);
  float abscoice = interpf(ld(T.absice3 + jrow(index - 1, 46) * 16 + band), ld(T.absice3 + jrow(index, 46) * 16 + band), fint);
  float abscosno = 0.0f;
  if ((ciwp + cswp) == 0.0f) abscoice = 0.0f;
  if (iceflag == 5 && cswp > 0.0f) {
    const float fs = (L.res - 2.0f) / 3.0f;
    int is = static_cast<int>(fs);
    if (is == 46) is = 45;
    const float fints = fs - static_cast<float>(is);
    abscosno = interpf(ld(T.absice3 + jrow(is - 1, 46) * 16 + band), ld(T.absice3 + jrow(is, 46) * 16 + band), fints);
  }
  int il = static_cast<int>(L.rel - 1.5f);
  if (il == 0) il = 1;
  if (il == 58) il = 57;
  const float fl = (L.rel - 1.5f) - static_cast<float>(il);
  const float abscoliq = clwp == 0.0f ? 0.0f
      : interpf(ld(T.absliq1 + jrow(il - 1, 58) * 16 + band), ld(T.absliq1 + jrow(il, 58) * 16 + band), fl);
  return (ciwp * abscoice + clwp * abscoliq) + cswp * abscosno;
}

__device__ __forceinline__ int pade_index(const Tables &T, float od) {
  const float tblind = od / (T.lw_bpade + od);
  const float pos = static_cast<float>(T.lw_ntbl) * tblind + 0.5f;
  return clampi(static_cast<int>(pos), 0, T.lw_ntbl);
}

// Layer transfer terms of one g-point (_rtrnmc_clear_terms/_rtrnmc_cloudy_terms,
// lw:5157-5262).
struct Terms {
  float a, gassrc, atot, bbdtot, bbdgas, bbugas, bbutot;
};

__device__ __forceinline__ Terms layer_terms(const Tables &T, bool cloudy_layer, float odepth, float odcld,
                                             float plfrac, float blay, float dplankdn, float dplankup) {
  const float rec_6 = 0.166667f;
  Terms t;
  t.atot = 0.0f;
  t.bbutot = 0.0f;
  t.bbdtot = 0.0f;
  t.gassrc = 0.0f;
  if (cloudy_layer) {
    const float odtot = odepth + odcld;
    if (odtot < 0.06f) {
      const float odepth_rec = rec_6 * odepth, odtot_rec = rec_6 * odtot;
      t.a = odepth - 0.5f * odepth * odepth;
      t.gassrc = plfrac * (blay + dplankdn * odepth_rec) * t.a;
      t.atot = odtot - 0.5f * odtot * odtot;
      t.bbdtot = plfrac * (blay + dplankdn * odtot_rec);
      t.bbdgas = plfrac * (blay + dplankdn * odepth_rec);
      t.bbugas = plfrac * (blay + dplankup * odepth_rec);
      t.bbutot = plfrac * (blay + dplankup * odtot_rec);
    } else if (odepth <= 0.06f) {
      const float odepth_rec = rec_6 * odepth;
      t.a = odepth - 0.5f * odepth * odepth;
      t.gassrc = plfrac * (blay + dplankdn * odepth_rec) * t.a;
      const int it = pade_index(T, odtot);
      const float tfactot = ld(T.lw_pade_tfn + it);
      t.atot = 1.0f - ld(T.lw_pade_exp + it);
      t.bbdtot = plfrac * (blay + tfactot * dplankdn);
      t.bbdgas = plfrac * (blay + dplankdn * odepth_rec);
      t.bbugas = plfrac * (blay + dplankup * odepth_rec);
      t.bbutot = plfrac * (blay + tfactot * dplankup);
    } else {
      const int ig = pade_index(T, odepth);
      const float odtbl = ld(T.lw_pade_tau + ig);
      t.a = 1.0f - ld(T.lw_pade_exp + ig);
      const float tfacgas = ld(T.lw_pade_tfn + ig);
      t.gassrc = t.a * plfrac * (blay + tfacgas * dplankdn);
      const float odtot3 = odtbl + odcld;
      const int it = pade_index(T, odtot3);
      const float tfactot = ld(T.lw_pade_tfn + it);
      t.atot = 1.0f - ld(T.lw_pade_exp + it);
      t.bbdtot = plfrac * (blay + tfactot * dplankdn);
      t.bbdgas = plfrac * (blay + tfacgas * dplankdn);
      t.bbugas = plfrac * (blay + tfacgas * dplankup);
      t.bbutot = plfrac * (blay + tfactot * dplankup);
    }
  } else {
    if (odepth <= 0.06f) {
      const float odepth_rec = rec_6 * odepth;
      t.a = odepth - (0.5f * odepth) * odepth;
      t.bbdgas = plfrac * (blay + dplankdn * odepth_rec);
      t.bbugas = plfrac * (blay + dplankup * odepth_rec);
    } else {
      const int it = pade_index(T, odepth);
      t.a = 1.0f - ld(T.lw_pade_exp + it);
      const float tausfac = ld(T.lw_pade_tfn + it);
      t.bbdgas = plfrac * (blay + tausfac * dplankdn);
      t.bbugas = plfrac * (blay + tausfac * dplankup);
    }
  }
  return t;
}

__device__ __forceinline__ float planck(const Tables &T, int ind, float frac, int band) {
  return interpf(ld(T.totplnk + (ind - 1) * 16 + band), ld(T.totplnk + ind * 16 + band), frac);
}

// One band of one layer in a sweep.  kDown: downward sweep (radiances radA =
// radld, radB = radclrd); otherwise upward (radA = radlu, radB = radclru).
// Returns the band's g-ordered radiance sums of the new level.
template <int B, bool kDown>
__device__ __forceinline__ void band_sums(const Tables &T, const Layer &L, const uint32_t *mask, bool cloudy_layer,
                                          int iceflag, float secdiff, float *radA, float *radB, bool sep_clear,
                                          float &bandsum, float &bandsumc) {
  constexpr int ngc = kNgc[B];
  constexpr int gofs = kGofs[B];
  float taug[ngc], fracs[ngc];
  taumol<B>(T, L, taug, fracs);
  const float blay = planck(T, L.indlay, L.tlayfrac, B);
  const float dplankup = planck(T, L.indlev1, L.tlev1frac, B) - blay;
  const float dplankdn = planck(T, L.indlev0, L.tlev0frac, B) - blay;
  float tauc = 0.0f, abscld = 0.0f;
  bool active = false;
  if (cloudy_layer) {
    tauc = cloud_tau(T, L, B, iceflag, active);
  }
  bandsum = 0.0f;
  bandsumc = 0.0f;
#pragma unroll
  for (int g = 0; g < ngc; ++g) {
    const int G = gofs + g;
    const bool cld = (mask[G >> 5] >> (G & 31)) & 1u;
    float odepth = secdiff * taug[g];
    if (odepth < 0.0f) odepth = 0.0f;
    float odcld = 0.0f, efcl = 0.0f;
    if (cld) {
      const float t = active ? tauc : 0.0f;
      const float odcld_raw = secdiff * t;
      abscld = 1.0f - glibc_expf(T, -odcld_raw);
      odcld = odcld_raw;
      efcl = abscld * 1.0f;
    }
    const Terms tm = layer_terms(T, cloudy_layer, odepth, odcld, fracs[g], blay, dplankdn, dplankup);
    const float cf = cld ? 1.0f : 0.0f;
    float r = radA[G], rc = radB[G];
    if constexpr (kDown) {
      float rn;
      if (cloudy_layer) {
        rn = r - r * (tm.a + efcl * (1.0f - tm.a)) + tm.gassrc + cf * (tm.bbdtot * tm.atot - tm.gassrc);
      } else {
        rn = r + (tm.bbdgas - r) * tm.a;
      }
      const float rcn = sep_clear ? rc + (tm.bbdgas - rc) * tm.a : rn;
      radA[G] = rn;
      radB[G] = rcn;
      bandsum = bandsum + rn;
      bandsumc = bandsumc + rcn;
    } else {
      float rn;
      if (cloudy_layer) {
        const float gas = tm.bbugas * tm.a;
        rn = r - r * (tm.a + efcl * (1.0f - tm.a)) + gas + cf * (tm.bbutot * tm.atot - gas);
      } else {
        rn = r + (tm.bbugas - r) * tm.a;
      }
      const float rcn = sep_clear ? rc + (tm.bbugas - rc) * tm.a : rn;
      radA[G] = rn;
      radB[G] = rcn;
      bandsum = bandsum + rn;
      bandsumc = bandsumc + rcn;
    }
  }
}

template <int B, bool kDown>
__device__ __forceinline__ void band_step(const Tables &T, const Layer &L, const uint32_t *mask, bool cloudy_layer,
                                          int iceflag, float secdiff, float *radA, float *radB, bool sep_clear,
                                          float &total, float &totalc) {
  float bandsum, bandsumc;
  band_sums<B, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff, radA, radB, sep_clear, bandsum, bandsumc);
  total = total + (bandsum * 0.5f) * kDelwave[B];
  totalc = totalc + (bandsumc * 0.5f) * kDelwave[B];
}

template <bool kDown>
__device__ __forceinline__ void all_bands(const Tables &T, const Layer &L, const uint32_t *mask, bool cloudy_layer,
                                          int iceflag, const float *secdiff, float *radA, float *radB, bool sep,
                                          float &total, float &totalc) {
  band_step<0, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[0], radA, radB, sep, total, totalc);
  band_step<1, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[1], radA, radB, sep, total, totalc);
  band_step<2, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[2], radA, radB, sep, total, totalc);
  band_step<3, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[3], radA, radB, sep, total, totalc);
  band_step<4, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[4], radA, radB, sep, total, totalc);
  band_step<5, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[5], radA, radB, sep, total, totalc);
  band_step<6, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[6], radA, radB, sep, total, totalc);
  band_step<7, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[7], radA, radB, sep, total, totalc);
  band_step<8, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[8], radA, radB, sep, total, totalc);
  band_step<9, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[9], radA, radB, sep, total, totalc);
  band_step<10, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[10], radA, radB, sep, total, totalc);
  band_step<11, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[11], radA, radB, sep, total, totalc);
  band_step<12, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[12], radA, radB, sep, total, totalc);
  band_step<13, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[13], radA, radB, sep, total, totalc);
  band_step<14, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[14], radA, radB, sep, total, totalc);
  band_step<15, kDown>(T, L, mask, cloudy_layer, iceflag, secdiff[15], radA, radB, sep, total, totalc);
}

// Surface: rad0 = fracs(layer 0) * plankbnd, reflected downward radiance
// (lw:5648-5655); returns the level-0 upward flux sums.
template <int B>
__device__ __forceinline__ void surface_sums(const Tables &T, const Layer &L0, float plankbnd, float reflect,
                                             float *radA, float *radB, float &bandsum, float &bandsumc) {
  constexpr int ngc = kNgc[B];
  constexpr int gofs = kGofs[B];
  float taug[ngc], fracs[ngc];
  taumol<B>(T, L0, taug, fracs);
  bandsum = 0.0f;
  bandsumc = 0.0f;
#pragma unroll
  for (int g = 0; g < ngc; ++g) {
    const int G = gofs + g;
    const float rad0 = fracs[g] * plankbnd;
    const float lu = rad0 + reflect * radA[G];
    const float lc = rad0 + reflect * radB[G];
    radA[G] = lu;
    radB[G] = lc;
    bandsum = bandsum + lu;
    bandsumc = bandsumc + lc;
  }
}

template <int B>
__device__ __forceinline__ void surface_band(const Tables &T, const Layer &L0, float plankbnd, float reflect,
                                             float *radA, float *radB, float &total, float &totalc) {
  float bandsum, bandsumc;
  surface_sums<B>(T, L0, plankbnd, reflect, radA, radB, bandsum, bandsumc);
  total = total + (bandsum * 0.5f) * kDelwave[B];
  totalc = totalc + (bandsumc * 0.5f) * kDelwave[B];
}

// Column prologue of both schedules: buffer layers, laytrop, pwvcm, the band
// diffusivities (lw:5520-5539) and whether any layer is cloudy.
// Column set-up shared by both prologues: buffer layers, laytrop and pwvcm.
// Fields of the column context taken from the call and the 2-D inputs.
__device__ __forceinline__ void column_head(const LwArgs &a, int col, Col &C) {
  C.i = col / a.ny;
  C.j = col - C.i * a.ny;
  C.nk = a.nk;
  C.ny = a.ny;
  C.nlay = a.nlay;
  C.nbuf = a.nlay - a.nk;
  C.co2 = a.co2; C.n2o = a.n2o; C.ch4 = a.ch4; C.cfc11 = a.cfc11; C.cfc12 = a.cfc12;
  C.inflg = a.inflg; C.iceflg = a.iceflg;
  C.has_reqc = a.has_reqc; C.has_reqi = a.has_reqi; C.has_reqs = a.has_reqs; C.icloud = a.icloud;
  C.tsfc = ld(a.in.tsk + col);
  C.semiss = ld(a.in.emiss + col);
}

constexpr float kAmd = 28.9660f, kAmw = 18.0160f, kAvogad = 6.02214199e23f, kGrav = 9.8066f;

// Layer l's share of the column integrals: whether it is below the
// tropopause test pressure, its dry-air column and its water column
// (lw:1037-1064, 1263-1264).
__device__ __forceinline__ void column_layer(const Tables &T, const LwArgs &a, const Col &C, int l, bool &trop,
                                             float &coldry, float &wk0) {
  const float pavel = play_at(a, C, l);
  trop = glibc_logf(T, pavel) > 4.56f;
  const float h2o = h2o_at(a, C, l);
  const float amm = (1.0f - h2o) * kAmd + h2o * kAmw;
  const float pm = ((plev_at(a, C, l) - plev_at(a, C, l + 1)) * 1.0e3f) * kAvogad;
  float md = 1.0e2f * kGrav;
  md = md * amm;
  md = md * (1.0f + h2o);
  coldry = pm / md;
  wk0 = h2o * coldry;
}

__device__ __forceinline__ float column_pwvcm(const LwArgs &a, const Col &C, float amttl, float wvttl) {
  const float wvsh = (kAmw * wvttl) / (kAmd * amttl);
  return (wvsh * (1.0e3f * plev_at(a, C, 0))) / (1.0e2f * kGrav);
}

__device__ __forceinline__ void column_core(const Tables &T, const LwArgs &a, int col, Col &C) {
  column_head(a, col, C);
  column_setup(T, a, C);
  const int nlay = C.nlay;
  // column integrals: laytrop and pwvcm, summed in layer order
  int laytrop = 0;
  float amttl = 0.0f, wvttl = 0.0f;
  for (int l = 0; l < nlay; ++l) {
    bool trop;
    float coldry, wk0;
    column_layer(T, a, C, l, trop, coldry, wk0);
    laytrop += trop;
    amttl = (amttl + coldry) + wk0;
    wvttl = wvttl + wk0;
  }
  C.laytrop = laytrop;
  C.pwvcm = column_pwvcm(a, C, amttl, wvttl);
}

// Band diffusivities from the column water (lw:5520-5539).
__device__ __forceinline__ void column_secdiff(const Tables &T, const Col &C, float *secdiff) {
#pragma unroll
  for (int b = 0; b < kLwBands; ++b) {
    const bool variable = !(b == 0 || b == 3 || b >= 9);
    if (variable) {
      const float e = glibc_expf(T, kA2[b] * C.pwvcm);
      const float v = kA0[b] + kA1[b] * e;
      secdiff[b] = v < 1.50f ? 1.50f : (v > 1.80f ? 1.80f : v);
    } else {
      secdiff[b] = 1.66f;
    }
  }
}

__device__ __forceinline__ void column_prologue(const Tables &T, const LwArgs &a, int col, Col &C, float *secdiff,
                                                bool &has_cloud) {
  column_core(T, a, col, C);
  const int nlay = C.nlay;
  column_secdiff(T, C, secdiff);

  // cloudy layers and whether any layer is cloudy (lw:5566-5567, 5656)
  has_cloud = false;
  for (int l = 0; l < nlay; ++l) {
    uint32_t any = 0;
#pragma unroll
    for (int w = 0; w < kLwMaskWords; ++w) any |= a.mask[(static_cast<size_t>(l) * kLwMaskWords + w) * a.ncol + col];
    has_cloud |= any != 0u;
  }
}

__global__ void __launch_bounds__(128) lw_kernel(Tables T, LwArgs a) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= a.ncol) return;
  Col C;
  float secdiff[kLwBands];
  bool has_cloud;
  column_prologue(T, a, col, C, secdiff, has_cloud);
  const int nlay = C.nlay;

  float radA[kLwGpts], radB[kLwGpts];
  float dfl[kMaxLay + 1], dflc[kMaxLay + 1];
#pragma unroll 4
  for (int g = 0; g < kLwGpts; ++g) { radA[g] = 0.0f; radB[g] = 0.0f; }
  const float pi = 3.1415926535897932384626433832795f;
  const float fluxfac = pi * 2.0e4f;
  const float heatfac = (9.8066f * 8.6400e4f) / (1004.5f * 1.0e2f);
  dfl[nlay] = 0.0f * fluxfac;
  dflc[nlay] = 0.0f * fluxfac;

  // downward sweep, top to bottom
  bool iclddn = false;
  for (int l = nlay - 1; l >= 0; --l) {
    uint32_t mask[kLwMaskWords];
    uint32_t any = 0;
#pragma unroll
    for (int w = 0; w < kLwMaskWords; ++w) {
      mask[w] = a.mask[(static_cast<size_t>(l) * kLwMaskWords + w) * a.ncol + col];
      any |= mask[w];
    }
    const bool cloudy = any != 0u;
    iclddn = iclddn || cloudy;
    const Layer L = make_layer(T, a, C, l);
    float total = 0.0f, totalc = 0.0f;
    all_bands<true>(T, L, mask, cloudy, C.iceflg, secdiff, radA, radB, iclddn, total, totalc);
    dfl[l] = total * fluxfac;
    dflc[l] = totalc * fluxfac;
  }
  // surface emission and reflection
  float ufl_prev, uflc_prev;
  {
    const Layer L0 = make_layer(T, a, C, 0);
    const float bt = C.tsfc - 159.0f;
    const int indbound = clampi(static_cast<int>(bt), 1, 180);
    const float tbndfrac = bt - static_cast<float>(indbound);
    const float reflect = 1.0f - C.semiss;
    float total = 0.0f, totalc = 0.0f;
#define SURF(B) surface_band<B>(T, L0, C.semiss * planck(T, indbound, tbndfrac, B), reflect, radA, radB, total, totalc)
    SURF(0); SURF(1); SURF(2); SURF(3); SURF(4); SURF(5); SURF(6); SURF(7);
    SURF(8); SURF(9); SURF(10); SURF(11); SURF(12); SURF(13); SURF(14); SURF(15);
#undef SURF
    ufl_prev = total * fluxfac;
    uflc_prev = totalc * fluxfac;
  }
  const float upb = ufl_prev, upbc = uflc_prev;
  // upward sweep, bottom to top, with the heating rate of each layer
  const size_t rbase = static_cast<size_t>(C.i) * C.nk * C.ny + C.j;
  for (int l = 0; l < nlay; ++l) {
    uint32_t mask[kLwMaskWords];
    uint32_t any = 0;
#pragma unroll
    for (int w = 0; w < kLwMaskWords; ++w) {
      mask[w] = a.mask[(static_cast<size_t>(l) * kLwMaskWords + w) * a.ncol + col];
      any |= mask[w];
    }
    const bool cloudy = any != 0u;
    const Layer L = make_layer(T, a, C, l);
    float total = 0.0f, totalc = 0.0f;
    all_bands<false>(T, L, mask, cloudy, C.iceflg, secdiff, radA, radB, has_cloud, total, totalc);
    const float ufl = total * fluxfac, uflc = totalc * fluxfac;
    if (l < C.nk) {
      const float fnet0 = ufl_prev - dfl[l], fnet1 = ufl - dfl[l + 1];
      const float fnetc0 = uflc_prev - dflc[l], fnetc1 = uflc - dflc[l + 1];
      const float dp = L.plev0 - L.plev1;
      float htr = heatfac * (fnet0 - fnet1) / dp;
      float htrc = heatfac * (fnetc0 - fnetc1) / dp;
      if (l >= a.fp64_from) {
        htr = heating64(heatfac, ufl_prev, dfl[l], ufl, dfl[l + 1], L.plev0, L.plev1);
        htrc = heating64(heatfac, uflc_prev, dflc[l], uflc, dflc[l + 1], L.plev0, L.plev1);
      }
      const float pi3d = ld(a.in.pi3d + rbase + static_cast<size_t>(l) * C.ny);
      a.rthraten[rbase + static_cast<size_t>(l) * C.ny] = (htr / 86400.0f) / pi3d;
      a.rthratenc[rbase + static_cast<size_t>(l) * C.ny] = (htrc / 86400.0f) / pi3d;
    }
    ufl_prev = ufl;
    uflc_prev = uflc;
  }
  // 2-D outputs (lw:7059-7077)
  a.upt[col] = ufl_prev;
  a.uptc[col] = uflc_prev;
  a.dnt[col] = dfl[nlay];
  a.dntc[col] = dflc[nlay];
  a.upb[col] = upb;
  a.upbc[col] = upbc;
  a.dnb[col] = dfl[0];
  a.dnbc[col] = dflc[0];
  a.glw[col] = dfl[0];
  a.olr[col] = ufl_prev;
  a.lwcf[col] = uflc_prev - ufl_prev;
#pragma unroll
  for (int q = 0; q < 4; ++q) a.zero2[q][col] = 0.0f;
}

// ---------------------------------------------------------------------------
// Sweep schedule, every domain size.  Columns are processed in chunks; per
// chunk:
//   lw_colprep_kernel  warp = column: buffer layers, column integrals (laytrop,
//                      pwvcm, summed in layer order), band diffusivities, and
//                      whether any layer is cloudy;
//   lw_layer_kernel    thread = (layer, column): the layer set-up (make_layer)
//                      once; the inputs of the gas optics go to a
//                      structure-of-arrays record, each band's Planck terms and
//                      cloud optical depth and the layer's cloud flag to the
//                      layer record;
//   lw_gas_kernel      thread = (layer, column), grid.y = band: the band's gas
//                      optical depths and Planck fractions (taumol) into the
//                      layer record, so every warp runs one band's code;
//   lw_sweep_kernel    block = kLwSweepCols columns x 140 g-points, thread =
//                      one g-point: the downward and upward radiance sweeps of
//                      rtrnmc (lw:5476-5722) from the layer records; each
//                      level's radiances go to shared memory, where they are
//                      summed in g-point order per band and the band terms in
//                      band order (lw:170-199); then fluxes, heating rates and
//                      the 2-D outputs.
// Operation for operation these are the reference's statements in its order,
// the same as the fused lw_kernel's, so the results are bit-identical.
// ---------------------------------------------------------------------------

// Layer record (kLwRec floats): taug of each band's g-points from a 16-byte
// boundary (kLwPadOfs), the Planck fractions likewise from kLwRecFracs, per
// band (blay, dplankup, dplankdn, cloud optical depth) from kLwRecBand, and
// the layer's cloud flag at kLwRecFlags.
constexpr int kLwPadOfs[kLwBands] = {0, 12, 24, 40, 56, 72, 80, 92, 100, 112, 120, 128, 136, 140, 144, 148};
constexpr int kLwPadG = 152;
constexpr int kLwRecFracs = kLwPadG, kLwRecBand = 2 * kLwPadG, kLwRecFlags = kLwRecBand + 4 * kLwBands;
constexpr int kLwRec = kLwRecFlags + 4;
static_assert(kLwRec % 4 == 0, "layer records are float4 aligned");
__constant__ int kLwPadOfsDev[kLwBands] = {0, 12, 24, 40, 56, 72, 80, 92, 100, 112, 120, 128, 136, 140, 144, 148};
__constant__ int kNgcDev[kLwBands] = {10, 12, 16, 14, 16, 8, 12, 8, 12, 6, 8, 8, 4, 2, 2, 2};
__constant__ int kGofsDev[kLwBands] = {0, 10, 22, 38, 52, 68, 76, 88, 96, 108, 114, 122, 130, 134, 136, 138};

// The Layer fields taumol reads, stored field by field ([field][layer][column]).
#define RRTMG_LW_GAS_FLOATS(X)                                                                                   \
  X(pavel) X(coldry) X(wx0) X(wx1) X(wx2) X(wx3) X(colh2o) X(colco2) X(colo3) X(coln2o) X(colco) X(colch4)      \
  X(colo2) X(colbrd) X(fac00) X(fac01) X(fac10) X(fac11) X(rat_h2oco2) X(rat_h2oco2_1) X(rat_h2oo3)             \
  X(rat_h2oo3_1) X(rat_h2on2o) X(rat_h2on2o_1) X(rat_h2och4) X(rat_h2och4_1) X(rat_n2oco2) X(rat_n2oco2_1)      \
  X(rat_o3co2) X(rat_o3co2_1) X(selffac) X(selffrac) X(forfac) X(forfrac) X(minorfrac) X(scaleminor)            \
  X(scaleminorn2)
#define RRTMG_LW_GAS_INTS(X) X(jp) X(jt) X(jt1) X(indself) X(indfor) X(indminor) X(trop)
#define RRTMG_LW_COUNT(name) +1
constexpr int kLwGasFields = 0 RRTMG_LW_GAS_FLOATS(RRTMG_LW_COUNT) RRTMG_LW_GAS_INTS(RRTMG_LW_COUNT);
#undef RRTMG_LW_COUNT

// Per-column record, computed once per column.
struct ColRec {
  Col C;
  float secdiff[kLwBands];
  int has_cloud;
};
constexpr size_t kColRecFloats = (sizeof(ColRec) + 15) / 16 * 4;

// scratch of one chunk: column records, then the gas fields, then the layer records
__device__ __forceinline__ const ColRec *col_records(const LwArgs &a) {
  return reinterpret_cast<const ColRec *>(a.scratch);
}
__device__ __forceinline__ float *gas_fields(const LwArgs &a) {
  return a.scratch + kColRecFloats * static_cast<size_t>(a.chunk_capacity);
}
__device__ __forceinline__ float *layer_records(const LwArgs &a) {
  return gas_fields(a) + static_cast<size_t>(kLwGasFields) * a.nlay * a.chunk_capacity;
}

__device__ __forceinline__ bool load_mask(const LwArgs &a, int l, int col, uint32_t *mask) {
  uint32_t any = 0;
#pragma unroll
  for (int w = 0; w < kLwMaskWords; ++w) {
    mask[w] = a.mask[(static_cast<size_t>(l) * kLwMaskWords + w) * a.ncol + col];
    any |= mask[w];
  }
  return any != 0u;
}

// A warp per column: the lanes take the buffer levels of the column set-up
// and the layers of the column integrals, whose sums are then taken in layer
// order from shared memory (the operations and order of column_prologue).
__global__ void __launch_bounds__(128) lw_colprep_kernel(Tables T, LwArgs a) {
  __shared__ float s_cd[4][kMaxLay], s_wk[4][kMaxLay];
  __shared__ float s_tlev[4][kMaxBuf + 1], s_o3[4][kMaxBuf];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lc = blockIdx.x * 4 + w;
  if (lc >= a.chunk_count || dead_column(a.live, a.chunk_first + lc)) return;  // whole warps
  const int col = a.chunk_first + lc;
  ColRec r;
  Col &C = r.C;
  column_head(a, col, C);
  column_setup<true>(T, a, C, lane, s_tlev[w], s_o3[w]);
  const int nlay = C.nlay;
  int trop_count = 0;
  bool cloud = false;
  for (int l = lane; l < nlay; l += 32) {
    bool trop;
    column_layer(T, a, C, l, trop, s_cd[w][l], s_wk[w][l]);
    trop_count += trop;
    uint32_t mask[kLwMaskWords];
    cloud = load_mask(a, l, col, mask) || cloud;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) trop_count += __shfl_xor_sync(0xffffffffu, trop_count, o);
  const bool has_cloud = __any_sync(0xffffffffu, cloud);
  __syncwarp();
  float amttl = 0.0f, wvttl = 0.0f;
  for (int l = 0; l < nlay; ++l) {
    amttl = (amttl + s_cd[w][l]) + s_wk[w][l];
    wvttl = wvttl + s_wk[w][l];
  }
  C.laytrop = trop_count;
  C.pwvcm = column_pwvcm(a, C, amttl, wvttl);
  column_secdiff(T, C, r.secdiff);
  r.has_cloud = has_cloud ? 1 : 0;
  if (lane == 0) reinterpret_cast<ColRec *>(a.scratch)[lc] = r;
}

// thread = (layer, chunk column), columns fastest
// Resident blocks per SM the register allocation must allow (measured at
// 425 x 425 x 50: without them the layer and gas kernels take 242 and 254
// registers, two blocks per SM, and the LW optics take 42 ms instead of 27;
// the sweep at 56 registers instead of 67 takes 27.7 ms instead of 32.9).
constexpr int kLwLayerMinBlocks = 6;
constexpr int kLwGasMinBlocks = 8;
constexpr int kLwSweepMinBlocks = 4;
__global__ void __launch_bounds__(128, kLwLayerMinBlocks) lw_layer_kernel(Tables T, LwArgs a) {
  const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int l = static_cast<int>(idx / a.chunk_count);
  const int lc = static_cast<int>(idx - static_cast<long long>(l) * a.chunk_count);
  if (l >= a.nlay) return;
  const int col = a.chunk_first + lc;
  if (dead_column(a.live, col)) return;
  const Col &C = col_records(a)[lc].C;
  const Layer L = make_layer(T, a, C, l);
  float *gas = gas_fields(a) + static_cast<size_t>(l) * a.chunk_capacity + lc;
  const size_t fstride = static_cast<size_t>(a.nlay) * a.chunk_capacity;
  int f = 0;
#define RRTMG_LW_PUT(name) gas[static_cast<size_t>(f++) * fstride] = L.name;
#define RRTMG_LW_PUTI(name) gas[static_cast<size_t>(f++) * fstride] = __int_as_float(L.name);
  RRTMG_LW_GAS_FLOATS(RRTMG_LW_PUT)
  RRTMG_LW_GAS_INTS(RRTMG_LW_PUTI)
#undef RRTMG_LW_PUT
#undef RRTMG_LW_PUTI
  uint32_t mask[kLwMaskWords];
  const bool cloudy = load_mask(a, l, col, mask);
  float4 *rec = reinterpret_cast<float4 *>(layer_records(a) + (static_cast<size_t>(lc) * a.nlay + l) * kLwRec);
  const int iceflag = C.iceflg;
#pragma unroll 1
  for (int b = 0; b < kLwBands; ++b) {
    const float blay = planck(T, L.indlay, L.tlayfrac, b);
    const float dplankup = planck(T, L.indlev1, L.tlev1frac, b) - blay;
    const float dplankdn = planck(T, L.indlev0, L.tlev0frac, b) - blay;
    float teff = 0.0f;
    if (cloudy) {
      bool active = false;
      const float tauc = cloud_tau(T, L, b, iceflag, active);
      teff = active ? tauc : 0.0f;
    }
    rec[kLwRecBand / 4 + b] = make_float4(blay, dplankup, dplankdn, teff);
  }
  rec[kLwRecFlags / 4] = make_float4(cloudy ? 1.0f : 0.0f, 0.0f, 0.0f, 0.0f);
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

template <int B>
__device__ __forceinline__ void gas_band(const Tables &T, const Layer &L, float4 *rec) {
  constexpr int ngc = kNgc[B], pofs = kLwPadOfs[B];
  float taug[ngc], fracs[ngc];
  taumol<B>(T, L, taug, fracs);
  store_padded<ngc>(rec + pofs / 4, taug);
  store_padded<ngc>(rec + (kLwRecFracs + pofs) / 4, fracs);
}

// Blocks of (layer, chunk column) pairs taken kLwGasGroup at a time, each
// group through all 16 bands before the next: the group's gas fields (44
// words per pair, 11.5 MB) stay in L2 across its bands, and each band's code
// runs on a full wave of blocks.
constexpr int kLwGasGroup = 512;

// thread = (layer, chunk column) of block `blk`; band from the block order above
__global__ void __launch_bounds__(128, kLwGasMinBlocks) lw_gas_kernel(Tables T, LwArgs a, int nblk) {
  const int group = blockIdx.x / (kLwGasGroup * kLwBands);
  const int g0 = group * kLwGasGroup;
  const int gsize = nblk - g0 < kLwGasGroup ? nblk - g0 : kLwGasGroup;
  const int within = blockIdx.x - group * kLwGasGroup * kLwBands;
  const int band = within / gsize;
  const int blk = g0 + (within - band * gsize);
  const long long idx = static_cast<long long>(blk) * blockDim.x + threadIdx.x;
  const int l = static_cast<int>(idx / a.chunk_count);
  const int lc = static_cast<int>(idx - static_cast<long long>(l) * a.chunk_count);
  if (l >= a.nlay || dead_column(a.live, a.chunk_first + lc)) return;
  const float *gas = gas_fields(a) + static_cast<size_t>(l) * a.chunk_capacity + lc;
  const size_t fstride = static_cast<size_t>(a.nlay) * a.chunk_capacity;
  Layer L{};
  int f = 0;
#define RRTMG_LW_GET(name) L.name = gas[static_cast<size_t>(f++) * fstride];
#define RRTMG_LW_GETI(name) L.name = __float_as_int(gas[static_cast<size_t>(f++) * fstride]);
  RRTMG_LW_GAS_FLOATS(RRTMG_LW_GET)
  RRTMG_LW_GAS_INTS(RRTMG_LW_GETI)
#undef RRTMG_LW_GET
#undef RRTMG_LW_GETI
  float4 *rec = reinterpret_cast<float4 *>(layer_records(a) + (static_cast<size_t>(lc) * a.nlay + l) * kLwRec);
  switch (band) {
    case 0: gas_band<0>(T, L, rec); break;
    case 1: gas_band<1>(T, L, rec); break;
    case 2: gas_band<2>(T, L, rec); break;
    case 3: gas_band<3>(T, L, rec); break;
    case 4: gas_band<4>(T, L, rec); break;
    case 5: gas_band<5>(T, L, rec); break;
    case 6: gas_band<6>(T, L, rec); break;
    case 7: gas_band<7>(T, L, rec); break;
    case 8: gas_band<8>(T, L, rec); break;
    case 9: gas_band<9>(T, L, rec); break;
    case 10: gas_band<10>(T, L, rec); break;
    case 11: gas_band<11>(T, L, rec); break;
    case 12: gas_band<12>(T, L, rec); break;
    case 13: gas_band<13>(T, L, rec); break;
    case 14: gas_band<14>(T, L, rec); break;
    default: gas_band<15>(T, L, rec); break;
  }
}

// One g-point of band_sums: the new radiances (rA, rB) after one layer, from
// the g-point's gas optical depth tg and Planck fraction fr, its band's
// (blay, dplankup, dplankdn, cloud optical depth) bq, its McICA bit cld and
// the layer's cloud flag.
template <bool kDown>
__device__ __forceinline__ void lw_step(const Tables &T, float tg, float fr, float4 bq, bool cld, bool cloudy_layer,
                                        float secdiff, float &rA, float &rB, bool sep_clear) {
  float odepth = secdiff * tg;
  if (odepth < 0.0f) odepth = 0.0f;
  float odcld = 0.0f, efcl = 0.0f;
  if (cld) {
    const float odcld_raw = secdiff * bq.w;
    const float abscld = 1.0f - glibc_expf(T, -odcld_raw);
    odcld = odcld_raw;
    efcl = abscld * 1.0f;
  }
  const Terms tm = layer_terms(T, cloudy_layer, odepth, odcld, fr, bq.x, bq.z, bq.y);
  const float cf = cld ? 1.0f : 0.0f;
  const float r = rA, rc = rB;
  float rn;
  if constexpr (kDown) {
    if (cloudy_layer) {
      rn = r - r * (tm.a + efcl * (1.0f - tm.a)) + tm.gassrc + cf * (tm.bbdtot * tm.atot - tm.gassrc);
    } else {
      rn = r + (tm.bbdgas - r) * tm.a;
    }
    rB = sep_clear ? rc + (tm.bbdgas - rc) * tm.a : rn;
  } else {
    if (cloudy_layer) {
      const float gas = tm.bbugas * tm.a;
      rn = r - r * (tm.a + efcl * (1.0f - tm.a)) + gas + cf * (tm.bbutot * tm.atot - gas);
    } else {
      rn = r + (tm.bbugas - r) * tm.a;
    }
    rB = sep_clear ? rc + (tm.bbugas - rc) * tm.a : rn;
  }
  rA = rn;
}

constexpr int kLwSweepCols = 2;                            // columns per block
constexpr int kLwSweepThreads = 288;                       // 2 x 140 g-points in 9 warps; 8 padding threads
constexpr int kLwRing = 8;                                 // levels of radiances per ordered-sum round
static_assert(kLwSweepThreads >= kLwSweepCols * kLwGpts && kLwSweepThreads % 32 == 0, "sweep block shape");

struct LwSweepShared {
  float ring[kLwRing][kLwSweepCols][2][kLwGpts];      // total, clear radiance of each g-point
  float bands[kLwRing][kLwSweepCols][2][kLwBands];    // each band's radiance sum
  float flux[kLwSweepCols][4][kMaxLay + 1];           // up total, up clear, down total, down clear per level
};

// Sums the ring's levels in two rounds of independent chains: (column,
// total/clear, level, band) adds the band's radiances in g-point order, then
// (column, total/clear, level) adds the band terms (bandsum * 0.5) * delwave in
// band order (band_step, lw:170-199) and multiplies by fluxfac.  The
// operations and their order are those of one sequential sum per level.
__device__ __forceinline__ void lw_flush(LwSweepShared &S, int count, int type0, int level0, int dir) {
  __syncthreads();
  const float pi = 3.1415926535897932384626433832795f;
  const float fluxfac = pi * 2.0e4f;
  const int band_chains = kLwSweepCols * 2 * count * kLwBands;
  for (int ch = threadIdx.x; ch < band_chains; ch += kLwSweepThreads) {
    const int b = ch % kLwBands;
    const int rest = ch / kLwBands;
    const int j = rest % count;
    const int cq = rest / count;  // column * 2 + total/clear
    const float *v = S.ring[j][cq >> 1][cq & 1] + kGofsDev[b];
    const int ngc = kNgcDev[b];
    float bandsum = 0.0f;
    for (int g = 0; g < ngc; ++g) bandsum = bandsum + v[g];
    S.bands[j][cq >> 1][cq & 1][b] = bandsum;
  }
  __syncthreads();
  const int chains = kLwSweepCols * 2 * count;
  for (int ch = threadIdx.x; ch < chains; ch += kLwSweepThreads) {
    const int j = ch % count;
    const int cq = ch / count;
    const float *bs = S.bands[j][cq >> 1][cq & 1];
    float total = 0.0f;
#pragma unroll
    for (int b = 0; b < kLwBands; ++b) total = total + (bs[b] * 0.5f) * kDelwave[b];
    S.flux[cq >> 1][type0 + (cq & 1)][level0 + dir * j] = total * fluxfac;
  }
  __syncthreads();
}

// Block = kLwSweepCols consecutive columns of the chunk.  A column past the
// chunk or the live count repeats the block's first column so that every
// thread takes the same barriers; its results are not written.
__global__ void __launch_bounds__(kLwSweepThreads, kLwSweepMinBlocks) lw_sweep_kernel(Tables T, LwArgs a) {
  __shared__ __align__(16) LwSweepShared S;
  const int lc0 = blockIdx.x * kLwSweepCols;
  if (lc0 >= a.chunk_count || dead_column(a.live, a.chunk_first + lc0)) return;  // whole block
  const int tid = threadIdx.x;
  const bool writer = tid < kLwSweepCols * kLwGpts;
  const int cslot = writer ? tid / kLwGpts : kLwSweepCols - 1;
  const int G = writer ? tid - cslot * kLwGpts : kLwGpts - 1;
  const int lc_own = lc0 + cslot;
  const bool live = lc_own < a.chunk_count && !dead_column(a.live, a.chunk_first + lc_own);
  const int lc = live ? lc_own : lc0;
  const int col = a.chunk_first + lc;
  int band = kLwBands - 1;
  while (G < kGofsDev[band]) --band;
  const int P = kLwPadOfsDev[band] + (G - kGofsDev[band]);
  const ColRec &R = col_records(a)[lc];
  const float sd = R.secdiff[band];
  const bool has_cloud = R.has_cloud != 0;
  const int nlay = a.nlay, nk = a.nk;
  const float *recs = layer_records(a) + static_cast<size_t>(lc) * nlay * kLwRec;
  const uint32_t *mword = a.mask + col + static_cast<size_t>(G >> 5) * a.ncol;
  const size_t mstride = static_cast<size_t>(kLwMaskWords) * a.ncol;
  const uint32_t bit = 1u << (G & 31);
  const float pi = 3.1415926535897932384626433832795f;
  const float fluxfac = pi * 2.0e4f;
  if (tid < kLwSweepCols * 2) S.flux[tid >> 1][2 + (tid & 1)][nlay] = 0.0f * fluxfac;  // no downward flux at the top

  // downward sweep, top to bottom: layer l gives level l; next layer loaded ahead
  float rA = 0.0f, rB = 0.0f;
  bool iclddn = false;
  int filled = 0, level0 = nlay - 1;
  const float *q = recs + static_cast<size_t>(nlay - 1) * kLwRec;
  float nx_tg = q[P], nx_fr = q[kLwRecFracs + P];
  float4 nx_bq = *reinterpret_cast<const float4 *>(q + kLwRecBand + 4 * band);
  float nx_flag = q[kLwRecFlags];
  uint32_t nx_word = mword[static_cast<size_t>(nlay - 1) * mstride];
  for (int l = nlay - 1; l >= 0; --l) {
    const float tg = nx_tg, fr = nx_fr, flag = nx_flag;
    const float4 bq = nx_bq;
    const uint32_t word = nx_word;
    if (l > 0) {
      q = recs + static_cast<size_t>(l - 1) * kLwRec;
      nx_tg = q[P];
      nx_fr = q[kLwRecFracs + P];
      nx_bq = *reinterpret_cast<const float4 *>(q + kLwRecBand + 4 * band);
      nx_flag = q[kLwRecFlags];
      nx_word = mword[static_cast<size_t>(l - 1) * mstride];
    }
    const bool cloudy = flag != 0.0f;
    iclddn = iclddn || cloudy;
    lw_step<true>(T, tg, fr, bq, (word & bit) != 0u, cloudy, sd, rA, rB, iclddn);
    if (writer) {
      S.ring[filled][cslot][0][G] = rA;
      S.ring[filled][cslot][1][G] = rB;
    }
    if (++filled == kLwRing || l == 0) {
      lw_flush(S, filled, 2, level0, -1);
      level0 -= filled;
      filled = 0;
    }
  }
  // surface emission and reflection: level 0 upward (surface_sums, lw:5648-5655)
  {
    const float bt = R.C.tsfc - 159.0f;
    const int indbound = clampi(static_cast<int>(bt), 1, 180);
    const float tbndfrac = bt - static_cast<float>(indbound);
    const float reflect = 1.0f - R.C.semiss;
    const float plankbnd = R.C.semiss * planck(T, indbound, tbndfrac, band);
    const float rad0 = recs[kLwRecFracs + P] * plankbnd;
    rA = rad0 + reflect * rA;
    rB = rad0 + reflect * rB;
    if (writer) {
      S.ring[0][cslot][0][G] = rA;
      S.ring[0][cslot][1][G] = rB;
    }
    filled = 1;
    level0 = 0;
  }
  // upward sweep, bottom to top: layer l gives level l + 1
  q = recs;
  nx_tg = q[P];
  nx_fr = q[kLwRecFracs + P];
  nx_bq = *reinterpret_cast<const float4 *>(q + kLwRecBand + 4 * band);
  nx_flag = q[kLwRecFlags];
  nx_word = mword[0];
  for (int l = 0; l < nlay; ++l) {
    const float tg = nx_tg, fr = nx_fr, flag = nx_flag;
    const float4 bq = nx_bq;
    const uint32_t word = nx_word;
    if (l + 1 < nlay) {
      q = recs + static_cast<size_t>(l + 1) * kLwRec;
      nx_tg = q[P];
      nx_fr = q[kLwRecFracs + P];
      nx_bq = *reinterpret_cast<const float4 *>(q + kLwRecBand + 4 * band);
      nx_flag = q[kLwRecFlags];
      nx_word = mword[static_cast<size_t>(l + 1) * mstride];
    }
    lw_step<false>(T, tg, fr, bq, (word & bit) != 0u, flag != 0.0f, sd, rA, rB, has_cloud);
    if (writer) {
      S.ring[filled][cslot][0][G] = rA;
      S.ring[filled][cslot][1][G] = rB;
    }
    if (++filled == kLwRing || l == nlay - 1) {
      lw_flush(S, filled, 0, level0, 1);
      level0 += filled;
      filled = 0;
    }
  }

  // heating rates and theta tendencies (lw:5706-5712, 7040-7057) and the 2-D
  // outputs (lw:7059-7077) of the block's live columns
  const float heatfac = (9.8066f * 8.6400e4f) / (1004.5f * 1.0e2f);
  for (int qq = tid; qq < kLwSweepCols * nk; qq += kLwSweepThreads) {
    const int cs = qq / nk, l = qq - cs * nk;
    const int lcq = lc0 + cs;
    if (lcq >= a.chunk_count || dead_column(a.live, a.chunk_first + lcq)) continue;
    const int cq = a.chunk_first + lcq;
    const int i = cq / a.ny, j = cq - i * a.ny;
    const float(*fx)[kMaxLay + 1] = S.flux[cs];
    const float fnet0 = fx[0][l] - fx[2][l], fnet1 = fx[0][l + 1] - fx[2][l + 1];
    const float fnetc0 = fx[1][l] - fx[3][l], fnetc1 = fx[1][l + 1] - fx[3][l + 1];
    const size_t rbase = static_cast<size_t>(i) * nk * a.ny + j;
    const size_t wbase = static_cast<size_t>(i) * (nk + 1) * a.ny + j;
    const float plev0 = pa_to_hpa(ld(a.in.p8w + wbase + static_cast<size_t>(l) * a.ny));
    const float plev1 = pa_to_hpa(ld(a.in.p8w + wbase + static_cast<size_t>(l + 1) * a.ny));
    const float dp = plev0 - plev1;
    float htr = heatfac * (fnet0 - fnet1) / dp;
    float htrc = heatfac * (fnetc0 - fnetc1) / dp;
    if (l >= a.fp64_from) {
      htr = heating64(heatfac, fx[0][l], fx[2][l], fx[0][l + 1], fx[2][l + 1], plev0, plev1);
      htrc = heating64(heatfac, fx[1][l], fx[3][l], fx[1][l + 1], fx[3][l + 1], plev0, plev1);
    }
    const float pi3d = ld(a.in.pi3d + rbase + static_cast<size_t>(l) * a.ny);
    a.rthraten[rbase + static_cast<size_t>(l) * a.ny] = (htr / 86400.0f) / pi3d;
    a.rthratenc[rbase + static_cast<size_t>(l) * a.ny] = (htrc / 86400.0f) / pi3d;
  }
  if (G == 0 && writer && live) {
    const float(*fx)[kMaxLay + 1] = S.flux[cslot];
    const float uflt = fx[0][nlay], ufltc = fx[1][nlay];
    const float dflt = 0.0f * fluxfac;
    a.upt[col] = uflt;
    a.uptc[col] = ufltc;
    a.dnt[col] = dflt;
    a.dntc[col] = dflt;
    a.upb[col] = fx[0][0];
    a.upbc[col] = fx[1][0];
    a.dnb[col] = fx[2][0];
    a.dnbc[col] = fx[3][0];
    a.glw[col] = fx[2][0];
    a.olr[col] = uflt;
    a.lwcf[col] = ufltc - uflt;
#pragma unroll
    for (int z = 0; z < 4; ++z) a.zero2[z][col] = 0.0f;
  }
}

}  // namespace

cudaError_t launch_lw(const Tables &T, const LwArgs &a, cudaStream_t stream) {
  const int threads = 128;
  const int blocks = (a.ncol + threads - 1) / threads;
  lw_kernel<<<blocks, threads, 0, stream>>>(T, a);
  return cudaGetLastError();
}

size_t lw_scratch_floats(int nlay, int chunk) {
  return (kColRecFloats + (static_cast<size_t>(kLwGasFields) + kLwRec) * nlay) * static_cast<size_t>(chunk);
}

cudaError_t launch_lw_chunk_optics(const Tables &T, const LwArgs &a, cudaStream_t stream) {
  const int threads = 128;
  lw_colprep_kernel<<<(a.chunk_count + 3) / 4, threads, 0, stream>>>(T, a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long long layers = static_cast<long long>(a.chunk_count) * a.nlay;
  const unsigned blocks = static_cast<unsigned>((layers + threads - 1) / threads);
  lw_layer_kernel<<<blocks, threads, 0, stream>>>(T, a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  lw_gas_kernel<<<blocks * kLwBands, threads, 0, stream>>>(T, a, static_cast<int>(blocks));
  return cudaGetLastError();
}

cudaError_t launch_lw_chunk_sweep(const Tables &T, const LwArgs &a, cudaStream_t stream) {
  lw_sweep_kernel<<<(a.chunk_count + kLwSweepCols - 1) / kLwSweepCols, kLwSweepThreads, 0, stream>>>(T, a);
  return cudaGetLastError();
}

}  // namespace rrtmg

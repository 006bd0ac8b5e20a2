/*
 * Oracle: RRTMG longwave restatement (test infrastructure only).
 * Reference file: src/wrf_jax/physics/module_ra_rrtmg_lw.py ("lw:").
 * Every statement below cites the reference lines it restates.
 */
#include "oracle_internal.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ONEMINUS (1.0f - 1.0e-6f)

static const int LW_NGC[LW_NBND] = {10, 12, 16, 14, 16, 8, 12, 8, 12, 6, 8, 8, 4, 2, 2, 2};
/* lwdatinit delwave (common:736-738) */
static const float LW_DELWAVE[LW_NBND] = {340.0f, 150.0f, 130.0f, 70.0f, 120.0f, 160.0f, 100.0f, 100.0f,
                                          210.0f, 90.0f, 320.0f, 280.0f, 170.0f, 130.0f, 220.0f, 650.0f};
/* rtrnmc diffusivity fit (lw:5520-5531) */
static const float LW_A0[LW_NBND] = {1.66f, 1.55f, 1.58f, 1.66f, 1.54f, 1.454f, 1.89f, 1.33f,
                                     1.668f, 1.66f, 1.66f, 1.66f, 1.66f, 1.66f, 1.66f, 1.66f};
static const float LW_A1[LW_NBND] = {0.0f, 0.25f, 0.22f, 0.0f, 0.13f, 0.446f, -0.10f, 0.40f,
                                     -0.006f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
static const float LW_A2[LW_NBND] = {0.0f, -12.0f, -11.7f, 0.0f, -0.72f, -0.243f, 0.19f, -0.062f,
                                     0.414f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};

int ora_lw_cache_init(const ora_tables *t, ora_lw_cache *c)
{
    char name[64];
    int gofs = 0;
    for (int b = 0; b < LW_NBND; ++b) {
        ora_lw_band *B = &c->band[b];
        B->ngc = LW_NGC[b];
        B->gofs = gofs;
        gofs += B->ngc;
#define GET(field) (snprintf(name, sizeof name, "lw%d." #field, b + 1), (const float *)ora_table(t, name, NULL))
        int n;
        snprintf(name, sizeof name, "lw%d.ka", b + 1);
        B->ka = (const float *)ora_table(t, name, &n);
        B->ka_rows = n / B->ngc;
        snprintf(name, sizeof name, "lw%d.kb", b + 1);
        B->kb = (const float *)ora_table(t, name, &n);
        B->kb_rows = B->kb ? n / B->ngc : 0;
        B->fracrefa = GET(fracrefa);
        B->fracrefb = GET(fracrefb);
        B->selfref = GET(selfref);
        B->forref = GET(forref);
        B->ka_mn2 = GET(ka_mn2);
        B->kb_mn2 = GET(kb_mn2);
        B->ka_mn2o = GET(ka_mn2o);
        B->kb_mn2o = GET(kb_mn2o);
        B->ka_mo3 = GET(ka_mo3);
        B->kb_mo3 = GET(kb_mo3);
        B->ka_mco2 = GET(ka_mco2);
        B->kb_mco2 = GET(kb_mco2);
        B->ka_mco = GET(ka_mco);
        B->ka_mo2 = GET(ka_mo2);
        B->kb_mo2 = GET(kb_mo2);
        B->ccl4 = GET(ccl4);
        B->cfc11adj = GET(cfc11adj);
        B->cfc12 = GET(cfc12);
        B->cfc22adj = GET(cfc22adj);
#undef GET
        if (!B->ka || !B->fracrefa || !B->selfref || !B->forref) return -1;
    }
    c->preflog = (const float *)ora_table(t, "lw.preflog", NULL);
    c->tref = (const float *)ora_table(t, "lw.tref", NULL);
    c->chi_mls = (const float *)ora_table(t, "lw.chi_mls", NULL);
    c->totplnk = (const float *)ora_table(t, "lw.totplnk", NULL);
    c->totplk16 = (const float *)ora_table(t, "lw.totplk16", NULL);
    c->absice0 = (const float *)ora_table(t, "lw.absice0", NULL);
    c->absice1 = (const float *)ora_table(t, "lw.absice1", NULL);
    c->absice2 = (const float *)ora_table(t, "lw.absice2", NULL);
    c->absice3 = (const float *)ora_table(t, "lw.absice3", NULL);
    c->absliq1 = (const float *)ora_table(t, "lw.absliq1", NULL);
    const float *absliq0 = (const float *)ora_table(t, "lw.absliq0", NULL);
    c->absliq0 = absliq0 ? absliq0[0] : 0.0f;
    int n;
    c->pade_tau = (const float *)ora_table(t, "lw.pade_tau_tbl", &n);
    c->ntbl = n - 1;
    c->pade_exp = (const float *)ora_table(t, "lw.pade_exp_tbl", NULL);
    c->pade_tfn = (const float *)ora_table(t, "lw.pade_tfn_tbl", NULL);
    const float *bp = (const float *)ora_table(t, "lw.pade_bpade", NULL);
    if (!c->preflog || !c->tref || !c->chi_mls || !c->totplnk || !c->absice3 || !c->absliq1 ||
        !c->pade_tau || !c->pade_exp || !c->pade_tfn || !bp)
        return -1;
    c->bpade = bp[0];
    return 0;
}

int ora_lw_nlayers(double p_top, int nk)
{
    /* rrtmg_lw_nlayers (common:1243-1247), kme = nk + 1, deltap = 4 */
    double layers_above = p_top * 0.01 / 4.0;
    return (nk + 1) + (int)(layers_above + 0.5) - 1;
}

/* ------------------------------------------------------------------------ */
/* per-column state                                                          */
/* ------------------------------------------------------------------------ */
typedef struct {
    int nlay, laytrop;
    int fp64_from;   /* first layer whose heating is formed in binary64 (FP64 mode) */
    float play[MAX_LAY], plev[MAX_LAY + 1], tlay[MAX_LAY], tlev[MAX_LAY + 1];
    float h2o[MAX_LAY], o3[MAX_LAY], co2[MAX_LAY], ch4[MAX_LAY], n2o[MAX_LAY], o2[MAX_LAY];
    float cfc11[MAX_LAY], cfc12[MAX_LAY], cfc22[MAX_LAY], ccl4[MAX_LAY];
    float tsfc, semiss;
    /* inatm */
    float coldry[MAX_LAY], wkl[7][MAX_LAY], wbrodl[MAX_LAY], wx[4][MAX_LAY], pwvcm;
    /* setcoef */
    int jp[MAX_LAY], jt[MAX_LAY], jt1[MAX_LAY], indself[MAX_LAY], indfor[MAX_LAY], indminor[MAX_LAY];
    float planklay[MAX_LAY][LW_NBND], planklev[MAX_LAY + 1][LW_NBND], plankbnd[LW_NBND];
    float colh2o[MAX_LAY], colco2[MAX_LAY], colo3[MAX_LAY], coln2o[MAX_LAY], colco[MAX_LAY];
    float colch4[MAX_LAY], colo2[MAX_LAY], colbrd[MAX_LAY];
    float fac00[MAX_LAY], fac01[MAX_LAY], fac10[MAX_LAY], fac11[MAX_LAY];
    float rat_h2oco2[MAX_LAY], rat_h2oco2_1[MAX_LAY], rat_h2oo3[MAX_LAY], rat_h2oo3_1[MAX_LAY];
    float rat_h2on2o[MAX_LAY], rat_h2on2o_1[MAX_LAY], rat_h2och4[MAX_LAY], rat_h2och4_1[MAX_LAY];
    float rat_n2oco2[MAX_LAY], rat_n2oco2_1[MAX_LAY], rat_o3co2[MAX_LAY], rat_o3co2_1[MAX_LAY];
    float selffac[MAX_LAY], selffrac[MAX_LAY], forfac[MAX_LAY], forfrac[MAX_LAY];
    float minorfrac[MAX_LAY], scaleminor[MAX_LAY], scaleminorn2[MAX_LAY];
    /* optical properties, (lay, g) and (g, lay) */
    float taug[MAX_LAY][LW_NGPT], fracs[MAX_LAY][LW_NGPT];
    unsigned char cldf[LW_NGPT][MAX_LAY];
    float ciwp[LW_NGPT][MAX_LAY], clwp[LW_NGPT][MAX_LAY], cswp[LW_NGPT][MAX_LAY];
    float taucmc[LW_NGPT][MAX_LAY];
    ora_cloud cloud;
    ora_binary32 cdf_work[LW_NGPT * MAX_LAY];
    /* radiative transfer */
    float urad[MAX_LAY + 1][LW_NGPT], drad[MAX_LAY + 1][LW_NGPT];
    float clrurad[MAX_LAY + 1][LW_NGPT], clrdrad[MAX_LAY + 1][LW_NGPT];
    float totuflux[MAX_LAY + 1], totdflux[MAX_LAY + 1], totuclfl[MAX_LAY + 1], totdclfl[MAX_LAY + 1];
    float htr[MAX_LAY], htrc[MAX_LAY];
} lw_col;

/* ------------------------------------------------------------------------ */
/* atmosphere preparation (lw:6789-6917, 6633-6786)                          */
/* ------------------------------------------------------------------------ */
static void lw_prepare(const ora_cache *C, const ora_in *in, int col, lw_col *S)
{
    const int nk = in->nk;
    const int nlay = ora_lw_nlayers(in->p_top, nk);
    S->nlay = nlay;
    S->fp64_from = in->fp64_steps ? (nk > 5 ? nk - 5 : 0) : MAX_LAY + 1;
    const float *p3d = in->p3d + (size_t)col * nk;
    const float *t3d = in->t3d + (size_t)col * nk;
    const float *p8w = in->p8w + (size_t)col * (nk + 1);
    const float *t8w = in->t8w + (size_t)col * (nk + 1);
    const float *qv = in->qv + (size_t)col * nk;
    const float *o3 = in->o3 + (size_t)col * nk;

    /* plev / play (lw:6690-6698) */
    for (int k = 0; k <= nk; ++k) S->plev[k] = ora_pa_to_hpa(p8w[k]);
    for (int lev = nk; lev < nlay; ++lev) S->plev[lev + 1] = S->plev[lev] - 4.0f;
    S->plev[nlay] = 0.0f;
    for (int k = 0; k < nk; ++k) S->play[k] = ora_pa_to_hpa(p3d[k]);
    for (int lay = nk; lay < nlay; ++lay) S->play[lay] = 0.5f * (S->plev[lay] + S->plev[lay + 1]);

    /* buffer-layer interface temperatures (lw:6633-6650) */
    float varint[MAX_LAY + 1] = {0};
    for (int lev = 0; lev <= nlay; ++lev) {
        float p = S->plev[lev];
        int count = 0;
        for (int i = 0; i < C->nprof; ++i) count += (C->pprof[i] >= p);
        int idx = clampi(count - 1, 0, C->nprof - 1);
        int idx1 = idx + 1 < C->nprof - 1 ? idx + 1 : C->nprof - 1;
        float p0 = C->pprof[idx], p1 = C->pprof[idx1], t0 = C->tprof[idx], t1 = C->tprof[idx1];
        float w = (idx == C->nprof - 1) ? 0.0f : (p - p0) / (p1 - p0);
        varint[lev] = w * (t1 - t0) + t0;
    }
    for (int k = 0; k <= nk; ++k) S->tlev[k] = t8w[k];
    float offset = S->tlev[nk - 1] - varint[nk - 1];
    for (int lev = nk; lev <= nlay; ++lev) S->tlev[lev] = varint[lev] + offset;
    for (int k = 0; k < nk; ++k) S->tlay[k] = t3d[k];
    for (int lev = nk; lev <= nlay; ++lev) S->tlay[lev - 1] = 0.5f * (S->tlev[lev] + S->tlev[lev - 1]);

    /* gases (lw:6868-6899, 6750-6764) */
    for (int l = 0; l < nlay; ++l) {
        int k = l < nk ? l : nk - 1;
        float q = fmaxf(qv[k], 1.0e-12f);
        S->h2o[l] = q * 1.607793f;
        S->co2[l] = in->co2;
        S->n2o[l] = in->n2o;
        S->ch4[l] = in->ch4;
        S->cfc11[l] = in->cfc11;
        S->cfc12[l] = in->cfc12;
        S->cfc22[l] = 0.169e-9f;
        S->ccl4[l] = 0.093e-9f;
        S->o2[l] = 0.209488f;
    }
    /* ozone above the model top (lw:6766-6786) */
    float o3mmr[MAX_LAY];
    ora_o3data(C, S->plev, nlay, o3mmr);
    const float amdo = 0.603461f;
    for (int k = 0; k < nk; ++k) S->o3[k] = o3[k];
    for (int l = nk; l < nlay; ++l) {
        float top = o3[nk - 1] - o3mmr[nk - 1] * amdo;
        top = top + o3mmr[l] * amdo;
        if (top <= 0.0f) top = o3mmr[l] * amdo;
        S->o3[l] = top;
    }
    S->tsfc = in->tsk[col];
    S->semiss = in->emiss[col];
}

/* inatm (lw:953-1135) */
static void lw_inatm(lw_col *S)
{
    const int n = S->nlay;
    const float amd = 28.9660f, amw = 18.0160f, avogad = 6.02214199e23f, grav = 9.8066f;
    float amttl = 0.0f, wvttl = 0.0f;
    for (int l = 0; l < n; ++l) {
        float h2o = S->h2o[l];
        float amm = (1.0f - h2o) * amd + h2o * amw;
        float pm = ((S->plev[l] - S->plev[l + 1]) * 1.0e3f) * avogad;
        float md = 1.0e2f * grav;
        md = md * amm;
        md = md * (1.0f + h2o);
        float coldry = pm / md;
        S->coldry[l] = coldry;
        float vmr[7] = {h2o, S->co2[l], S->o3[l], S->n2o[l], 0.0f, S->ch4[l], S->o2[l]};
        float summol = 0.0f;
        for (int m = 1; m < 7; ++m) summol = summol + vmr[m];
        S->wbrodl[l] = coldry * (1.0f - summol);
        for (int m = 0; m < 7; ++m) S->wkl[m][l] = vmr[m] * coldry;
        float cross[4] = {S->ccl4[l], S->cfc11[l], S->cfc12[l], S->cfc22[l]};
        for (int m = 0; m < 4; ++m) S->wx[m][l] = (cross[m] * coldry) * 1.0e-20f;
    }
    for (int l = 0; l < n; ++l) {
        amttl = (amttl + S->coldry[l]) + S->wkl[0][l];
        wvttl = wvttl + S->wkl[0][l];
    }
    float wvsh = (amw * wvttl) / (amd * amttl);
    S->pwvcm = (wvsh * (1.0e3f * S->plev[0])) / (1.0e2f * grav);
}

/* setcoef (lw:1175-1441) */
static void lw_setcoef(const ora_lw_cache *L, lw_col *S)
{
    const int n = S->nlay;
    const float *totplnk = L->totplnk;       /* (181, 16) */
    const float *chi = L->chi_mls;           /* (7, 59) */
#define CHI(g, j) chi[(g) * 59 + (j)]
    /* Planck functions */
    float bt = S->tsfc - 159.0f;
    int indbound = clampi((int)bt, 1, 180);
    float tbndfrac = bt - (float)indbound;
    float t0 = S->tlev[0] - 159.0f;
    int indlev0 = clampi((int)t0, 1, 180);
    float t0frac = t0 - (float)indlev0;
    for (int b = 0; b < LW_NBND; ++b) {
        float lo = totplnk[(indbound - 1) * 16 + b], hi = totplnk[indbound * 16 + b];
        S->plankbnd[b] = S->semiss * interpf(lo, hi, tbndfrac);
        lo = totplnk[(indlev0 - 1) * 16 + b];
        hi = totplnk[indlev0 * 16 + b];
        S->planklev[0][b] = interpf(lo, hi, t0frac);
    }
    for (int l = 0; l < n; ++l) {
        float tl = S->tlay[l] - 159.0f;
        int indlay = clampi((int)tl, 1, 180);
        float tlayfrac = tl - (float)indlay;
        float tv = S->tlev[l + 1] - 159.0f;
        int indlev = clampi((int)tv, 1, 180);
        float tlevfrac = tv - (float)indlev;
        for (int b = 0; b < LW_NBND; ++b) {
            S->planklay[l][b] = interpf(totplnk[(indlay - 1) * 16 + b], totplnk[indlay * 16 + b], tlayfrac);
            S->planklev[l + 1][b] = interpf(totplnk[(indlev - 1) * 16 + b], totplnk[indlev * 16 + b], tlevfrac);
        }
    }

    const float stpfac = 296.0f / 1013.0f;
    int laytrop = 0;
    for (int l = 0; l < n; ++l) {
        float pavel = S->play[l], tavel = S->tlay[l], coldry = S->coldry[l];
        float plog = logf(pavel);
        int jp = clampi((int)(36.0f - 5.0f * (plog + 0.04f)), 1, 58);
        float fp = 5.0f * (L->preflog[jp - 1] - plog);
        float tf = (tavel - L->tref[jp - 1]) / 15.0f;
        int jt = clampi((int)(3.0f + tf), 1, 4);
        float ft = tf - (float)(jt - 3);
        float tf1 = (tavel - L->tref[jp]) / 15.0f;
        int jt1 = clampi((int)(3.0f + tf1), 1, 4);
        float ft1 = tf1 - (float)(jt1 - 3);
        float water = S->wkl[0][l] / coldry;
        float scalefac = (pavel * stpfac) / tavel;
        int trop = plog > 4.56f;
        laytrop += trop;
        float forfac_base = scalefac / (1.0f + water);
        float ftf = (332.0f - tavel) / 36.0f;
        int indfor_t = clampi((int)ftf, 1, 2);
        float forfrac_t = ftf - (float)indfor_t;
        float fsf = (tavel - 188.0f) / 36.0f;
        S->indfor[l] = trop ? indfor_t : 3;
        S->forfrac[l] = trop ? forfrac_t : fsf - 1.0f;
        float fself = (tavel - 188.0f) / 7.2f;
        int indself_t = clampi((int)fself - 7, 1, 9);
        float selffrac_t = fself - (float)(indself_t + 7);
        S->indself[l] = trop ? indself_t : 0;
        S->selffrac[l] = trop ? selffrac_t : 0.0f;
        S->scaleminor[l] = pavel / tavel;
        S->scaleminorn2[l] = S->scaleminor[l] * (S->wbrodl[l] / (coldry + S->wkl[0][l]));
        float fminor = (tavel - 180.8f) / 7.2f;
        S->indminor[l] = clampi((int)fminor, 1, 18);
        S->minorfrac[l] = fminor - (float)S->indminor[l];
        const float tiny = 1.0e-20f;
        float fallback = 1.0e-32f * coldry;
        S->colh2o[l] = tiny * S->wkl[0][l];
        S->colco2[l] = tiny * S->wkl[1][l];
        S->colo3[l] = tiny * S->wkl[2][l];
        S->coln2o[l] = tiny * S->wkl[3][l];
        S->colco[l] = tiny * S->wkl[4][l];
        S->colch4[l] = tiny * S->wkl[5][l];
        S->colo2[l] = tiny * S->wkl[6][l];
        if (S->colco2[l] == 0.0f) S->colco2[l] = fallback;
        if (S->colo3[l] == 0.0f) S->colo3[l] = fallback;
        if (S->coln2o[l] == 0.0f) S->coln2o[l] = fallback;
        if (S->colco[l] == 0.0f) S->colco[l] = fallback;
        if (S->colch4[l] == 0.0f) S->colch4[l] = fallback;
        S->colbrd[l] = tiny * S->wbrodl[l];
        int j0 = jp - 1, j1 = jp;
        S->rat_h2oco2[l] = CHI(0, j0) / CHI(1, j0);
        S->rat_h2oco2_1[l] = CHI(0, j1) / CHI(1, j1);
        S->rat_h2oo3[l] = trop ? CHI(0, j0) / CHI(2, j0) : 0.0f;
        S->rat_h2oo3_1[l] = trop ? CHI(0, j1) / CHI(2, j1) : 0.0f;
        S->rat_h2on2o[l] = trop ? CHI(0, j0) / CHI(3, j0) : 0.0f;
        S->rat_h2on2o_1[l] = trop ? CHI(0, j1) / CHI(3, j1) : 0.0f;
        S->rat_h2och4[l] = trop ? CHI(0, j0) / CHI(5, j0) : 0.0f;
        S->rat_h2och4_1[l] = trop ? CHI(0, j1) / CHI(5, j1) : 0.0f;
        S->rat_n2oco2[l] = trop ? CHI(3, j0) / CHI(1, j0) : 0.0f;
        S->rat_n2oco2_1[l] = trop ? CHI(3, j1) / CHI(1, j1) : 0.0f;
        S->rat_o3co2[l] = trop ? 0.0f : CHI(2, j0) / CHI(1, j0);
        S->rat_o3co2_1[l] = trop ? 0.0f : CHI(2, j1) / CHI(1, j1);
        float compfp = 1.0f - fp;
        S->fac10[l] = compfp * ft;
        S->fac00[l] = compfp * (1.0f - ft);
        S->fac11[l] = fp * ft1;
        S->fac01[l] = fp * (1.0f - ft1);
        S->selffac[l] = S->colh2o[l] * (water * forfac_base);
        S->forfac[l] = S->colh2o[l] * forfac_base;
        S->jp[l] = jp;
        S->jt[l] = jt;
        S->jt1[l] = jt1;
    }
    S->laytrop = laytrop;
#undef CHI
}

/* ------------------------------------------------------------------------ */
/* taumol helpers (lw:108-168, 1444-1594)                                    */
/* ------------------------------------------------------------------------ */
typedef struct { float sc, sp, fs; int js; } spec_t;

static inline spec_t specint(float primary, float ratio, float secondary, float scale)
{
    spec_t s;
    s.sc = primary + ratio * secondary;
    float q = primary / s.sc;
    s.sp = q > ONEMINUS ? ONEMINUS : q;
    float sm = scale * s.sp;
    s.js = 1 + (int)sm;
    s.fs = sm - floorf(sm);
    return s;
}

typedef struct { float f000, f100, f200, f010, f110, f210; int low, high; } edge_t;

static inline edge_t edge_factors(float specparm, float fs, float fa, float fb)
{
    edge_t e;
    e.low = specparm < 0.125f;
    e.high = specparm > 0.875f;
    if (e.low) {
        float p = fs - 1.0f;
        float p2 = p * p, p4 = p2 * p2;
        float fk0 = p4, fk1 = (1.0f - p) - 2.0f * p4, fk2 = p + p4;
        e.f000 = fk0 * fa; e.f100 = fk1 * fa; e.f200 = fk2 * fa;
        e.f010 = fk0 * fb; e.f110 = fk1 * fb; e.f210 = fk2 * fb;
    } else if (e.high) {
        float p = 0.0f - fs;
        float p2 = p * p, p4 = p2 * p2;
        float fk0 = p4, fk1 = (1.0f - p) - 2.0f * p4, fk2 = p + p4;
        e.f000 = fk0 * fa; e.f100 = fk1 * fa; e.f200 = fk2 * fa;
        e.f010 = fk0 * fb; e.f110 = fk1 * fb; e.f210 = fk2 * fb;
    } else {
        e.f000 = (1.0f - fs) * fa; e.f100 = fs * fa; e.f200 = 0.0f;
        e.f010 = (1.0f - fs) * fb; e.f110 = fs * fb; e.f210 = 0.0f;
    }
    return e;
}

#define SAFE(tab, rows, ngc, r, g) (tab)[clampi((r), 0, (rows) - 1) * (ngc) + (g)]

static inline float edge_major(const float *tab, int rows, int ngc, int base, edge_t e, int g)
{
    float s;
    if (e.low) {
        s = e.f000 * SAFE(tab, rows, ngc, base, g);
        s = s + e.f100 * SAFE(tab, rows, ngc, base + 1, g);
        s = s + e.f200 * SAFE(tab, rows, ngc, base + 2, g);
        s = s + e.f010 * SAFE(tab, rows, ngc, base + 9, g);
        s = s + e.f110 * SAFE(tab, rows, ngc, base + 10, g);
        s = s + e.f210 * SAFE(tab, rows, ngc, base + 11, g);
    } else if (e.high) {
        s = e.f200 * SAFE(tab, rows, ngc, base - 1, g);
        s = s + e.f100 * SAFE(tab, rows, ngc, base, g);
        s = s + e.f000 * SAFE(tab, rows, ngc, base + 1, g);
        s = s + e.f210 * SAFE(tab, rows, ngc, base + 8, g);
        s = s + e.f110 * SAFE(tab, rows, ngc, base + 9, g);
        s = s + e.f010 * SAFE(tab, rows, ngc, base + 10, g);
    } else {
        s = e.f000 * SAFE(tab, rows, ngc, base, g);
        s = s + e.f100 * SAFE(tab, rows, ngc, base + 1, g);
        s = s + e.f010 * SAFE(tab, rows, ngc, base + 9, g);
        s = s + e.f110 * SAFE(tab, rows, ngc, base + 10, g);
    }
    return s;
}

/* 4-point major interpolation in a 5x table: rows ind0, ind0+1, ind1, ind1+1 */
static inline float major4(const float *tab, int ngc, int ind0, int ind1, int g,
                           float f00, float f10, float f01, float f11)
{
    float s = f00 * tab[ind0 * ngc + g];
    s = s + f10 * tab[(ind0 + 1) * ngc + g];
    s = s + f01 * tab[ind1 * ngc + g];
    s = s + f11 * tab[(ind1 + 1) * ngc + g];
    return s;
}

/* stratospheric binary-species interpolation (rows i, i+1, i+5, i+6) */
static inline float strat_binary(const float *tab, int rows, int ngc, int ind, int g, float fs, float fa, float fb)
{
    float comp = 1.0f - fs;
    float s000 = comp * fa, s100 = fs * fa, s010 = comp * fb, s110 = fs * fb;
    float s = s000 * SAFE(tab, rows, ngc, ind, g);
    s = s + s100 * SAFE(tab, rows, ngc, ind + 1, g);
    s = s + s010 * SAFE(tab, rows, ngc, ind + 5, g);
    s = s + s110 * SAFE(tab, rows, ngc, ind + 6, g);
    return s;
}

static inline int ind5(int v, int rows) { return clampi(v, 0, rows - 2); }

static inline float lin_minor(const float *tab, int rows, int ngc, int indminor, float frac, int g)
{
    int m0 = clampi(indminor - 1, 0, rows - 2);
    return interpf(tab[m0 * ngc + g], tab[(m0 + 1) * ngc + g], frac);
}

/* minor gas with a species dimension: tab (nspec, 19, ngc) */
static inline float spec_minor(const float *tab, int nspec, int ngc, int jm, float fm, int indminor, float frac, int g)
{
    int m0 = clampi(indminor - 1, 0, 19 - 2);
    int j0 = clampi(jm - 1, 0, nspec - 2);
    float a = interpf(tab[(j0 * 19 + m0) * ngc + g], tab[((j0 + 1) * 19 + m0) * ngc + g], fm);
    float b = interpf(tab[(j0 * 19 + m0 + 1) * ngc + g], tab[((j0 + 1) * 19 + m0 + 1) * ngc + g], fm);
    return interpf(a, b, frac);
}

static inline float self_tau(const ora_lw_band *B, const lw_col *S, int l, int g)
{
    int i0 = clampi(S->indself[l] - 1, 0, 10 - 2);
    return S->selffac[l] * interpf(B->selfref[i0 * B->ngc + g], B->selfref[(i0 + 1) * B->ngc + g], S->selffrac[l]);
}

static inline float for_tau(const ora_lw_band *B, const lw_col *S, int l, int g)
{
    int i0 = clampi(S->indfor[l] - 1, 0, 4 - 2);
    return S->forfac[l] * interpf(B->forref[i0 * B->ngc + g], B->forref[(i0 + 1) * B->ngc + g], S->forfrac[l]);
}

/* fracs interpolated in a (ngc, ncol) Planck-fraction table */
static inline float frac_interp(const float *tab, int ncols, int jpl, float fpl, int g)
{
    int j0 = clampi(jpl - 1, 0, ncols - 2);
    return interpf(tab[g * ncols + j0], tab[g * ncols + j0 + 1], fpl);
}

/* Test knob (ora_set_libm_perturbation): move the two results the reference
 * takes from XLA's binary32 libm rather than glibc -- the minor-gas scaling
 * power (lw:134-144) and the cloud absorptance exponential (lw:5564) -- by a
 * given number of ulps, to bound what a last-place libm difference does to
 * the outputs.  Zero (the default) leaves glibc's results untouched. */
static int g_pow_ulps = 0, g_exp_ulps = 0;

void ora_set_libm_perturbation(int exp_ulps, int pow_ulps)
{
    g_exp_ulps = exp_ulps;
    g_pow_ulps = pow_ulps;
}

static inline float nudge_ulps(float v, int ulps)
{
    for (; ulps > 0; --ulps) v = nextafterf(v, INFINITY);
    for (; ulps < 0; ++ulps) v = nextafterf(v, -INFINITY);
    return v;
}

static inline float active_pow(float base, float exponent)
{
    float r = powf(base, exponent);
    return g_pow_ulps && exponent != 0.0f && base != 1.0f ? nudge_ulps(r, g_pow_ulps) : r;
}

/* exp of a cloud optical depth; exp(0) = 1 is exact in every libm */
static inline float cloud_expf(float x)
{
    float r = expf(x);
    return g_exp_ulps && x != 0.0f ? nudge_ulps(r, g_exp_ulps) : r;
}

/* ------------------------------------------------------------------------ */
/* taumol per band (lw:1597-4684)                                            */
/* ------------------------------------------------------------------------ */
static void lw_taumol(const ora_lw_cache *L, lw_col *S)
{
    const int n = S->nlay;
    const float *chi = L->chi_mls;
#define CHI(g, j) chi[(g) * 59 + (j)]
    for (int l = 0; l < n; ++l) {
        const int trop = l < S->laytrop;
        const int jp = S->jp[l], jt = S->jt[l], jt1 = S->jt1[l];
        const float f00 = S->fac00[l], f01 = S->fac01[l], f10 = S->fac10[l], f11 = S->fac11[l];
        const float colh2o = S->colh2o[l], colco2 = S->colco2[l], colo3 = S->colo3[l];
        const float coln2o = S->coln2o[l], colch4 = S->colch4[l], colco = S->colco[l];
        const float coldry = S->coldry[l], pavel = S->play[l], mfrac = S->minorfrac[l];
        const int indm = S->indminor[l];

        /* ---- band 1 (lw:1597-1784) ---- */
        {
            const ora_lw_band *B = &L->band[0];
            const int ngc = B->ngc;
            for (int g = 0; g < ngc; ++g) {
                float taun2, major, corr, tau;
                float scalen2 = S->colbrd[l] * S->scaleminorn2[l];
                if (trop) {
                    int i0 = ind5((jp - 1) * 5 + (jt - 1), B->ka_rows), i1 = ind5(jp * 5 + (jt1 - 1), B->ka_rows);
                    major = major4(B->ka, ngc, i0, i1, g, f00, f10, f01, f11);
                    taun2 = scalen2 * lin_minor(B->ka_mn2, 19, ngc, indm, mfrac, g);
                    corr = pavel < 250.0f ? 1.0f - ((0.15f * (250.0f - pavel)) / 154.4f) : 1.0f;
                    tau = corr * (((colh2o * major + self_tau(B, S, l, g)) + for_tau(B, S, l, g)) + taun2);
                    S->fracs[l][B->gofs + g] = B->fracrefa[g];
                } else {
                    int i0 = ind5((jp - 13) * 5 + (jt - 1), B->kb_rows), i1 = ind5((jp - 12) * 5 + (jt1 - 1), B->kb_rows);
                    major = major4(B->kb, ngc, i0, i1, g, f00, f10, f01, f11);
                    taun2 = scalen2 * lin_minor(B->kb_mn2, 19, ngc, indm, mfrac, g);
                    corr = 1.0f - 0.15f * (pavel / 95.6f);
                    tau = corr * ((colh2o * major + for_tau(B, S, l, g)) + taun2);
                    S->fracs[l][B->gofs + g] = B->fracrefb[g];
                }
                S->taug[l][B->gofs + g] = tau;
            }
        }
        /* ---- band 2 (lw:1787-1924) ---- */
        {
            const ora_lw_band *B = &L->band[1];
            const int ngc = B->ngc;
            for (int g = 0; g < ngc; ++g) {
                float tau;
                if (trop) {
                    int i0 = ind5((jp - 1) * 5 + (jt - 1), B->ka_rows), i1 = ind5(jp * 5 + (jt1 - 1), B->ka_rows);
                    float major = major4(B->ka, ngc, i0, i1, g, f00, f10, f01, f11);
                    float corr = 1.0f - ((0.05f * (pavel - 100.0f)) / 900.0f);
                    tau = corr * ((colh2o * major + self_tau(B, S, l, g)) + for_tau(B, S, l, g));
                    S->fracs[l][B->gofs + g] = B->fracrefa[g];
                } else {
                    int i0 = ind5((jp - 13) * 5 + (jt - 1), B->kb_rows), i1 = ind5((jp - 12) * 5 + (jt1 - 1), B->kb_rows);
                    float major = major4(B->kb, ngc, i0, i1, g, f00, f10, f01, f11);
                    tau = colh2o * major + for_tau(B, S, l, g);
                    S->fracs[l][B->gofs + g] = B->fracrefb[g];
                }
                S->taug[l][B->gofs + g] = tau;
            }
        }
        /* ---- band 3 (lw:1927-2235) ---- */
        {
            const ora_lw_band *B = &L->band[2];
            const int ngc = B->ngc;
            float chi_n2o = coln2o / coldry;
            float chi_ref = CHI(3, clampi(jp, 0, 58));
            float ratn2o = (1.0e20f * chi_n2o) / chi_ref;
            float adjcoln2o = coln2o;
            if (ratn2o > 1.5f) {
                float adjfac = 0.5f + active_pow(ratn2o - 0.5f, 0.65f);
                adjcoln2o = ((adjfac * chi_ref) * coldry) * 1.0e-20f;
            }
            if (trop) {
                float rpa = CHI(0, 8) / CHI(1, 8), rma = CHI(0, 2) / CHI(1, 2);
                spec_t s0 = specint(colh2o, S->rat_h2oco2[l], colco2, 8.0f);
                spec_t s1 = specint(colh2o, S->rat_h2oco2_1[l], colco2, 8.0f);
                spec_t sm = specint(colh2o, rma, colco2, 8.0f);
                spec_t sp = specint(colh2o, rpa, colco2, 8.0f);
                int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
                int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
                edge_t e0 = edge_factors(s0.sp, s0.fs, f00, f10), e1 = edge_factors(s1.sp, s1.fs, f01, f11);
                for (int g = 0; g < ngc; ++g) {
                    float tm0 = s0.sc * edge_major(B->ka, B->ka_rows, ngc, b0, e0, g);
                    float tm1 = s1.sc * edge_major(B->ka, B->ka_rows, ngc, b1, e1, g);
                    float absn2o = spec_minor(B->ka_mn2o, 9, ngc, sm.js, sm.fs, indm, mfrac, g);
                    float tau = (((tm0 + tm1) + self_tau(B, S, l, g)) + for_tau(B, S, l, g)) + adjcoln2o * absn2o;
                    S->taug[l][B->gofs + g] = tau;
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefa, 9, sp.js, sp.fs, g);
                }
            } else {
                float rpb = CHI(0, 12) / CHI(1, 12), rmb = CHI(0, 12) / CHI(1, 12);
                spec_t s0 = specint(colh2o, S->rat_h2oco2[l], colco2, 4.0f);
                spec_t s1 = specint(colh2o, S->rat_h2oco2_1[l], colco2, 4.0f);
                spec_t sm = specint(colh2o, rmb, colco2, 4.0f);
                spec_t sp = specint(colh2o, rpb, colco2, 4.0f);
                int i0 = (jp - 13) * 25 + (jt - 1) * 5 + (s0.js - 1);
                int i1 = (jp - 12) * 25 + (jt1 - 1) * 5 + (s1.js - 1);
                for (int g = 0; g < ngc; ++g) {
                    float m0 = s0.sc * strat_binary(B->kb, B->kb_rows, ngc, i0, g, s0.fs, f00, f10);
                    float m1 = s1.sc * strat_binary(B->kb, B->kb_rows, ngc, i1, g, s1.fs, f01, f11);
                    float absn2o = spec_minor(B->kb_mn2o, 5, ngc, sm.js, sm.fs, indm, mfrac, g);
                    float tau = ((m0 + m1) + for_tau(B, S, l, g)) + adjcoln2o * absn2o;
                    S->taug[l][B->gofs + g] = tau;
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefb, 5, sp.js, sp.fs, g);
                }
            }
        }
        /* ---- band 4 (lw:2238-2457) ---- */
        {
            const ora_lw_band *B = &L->band[3];
            const int ngc = B->ngc;
            static const float corr4[14] = {1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 0.92f, 0.88f, 1.07f, 1.1f, 0.99f, 0.88f, 0.943f};
            if (trop) {
                float rpa = CHI(0, 10) / CHI(1, 10);
                spec_t s0 = specint(colh2o, S->rat_h2oco2[l], colco2, 8.0f);
                spec_t s1 = specint(colh2o, S->rat_h2oco2_1[l], colco2, 8.0f);
                spec_t sp = specint(colh2o, rpa, colco2, 8.0f);
                int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
                int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
                edge_t e0 = edge_factors(s0.sp, s0.fs, f00, f10), e1 = edge_factors(s1.sp, s1.fs, f01, f11);
                for (int g = 0; g < ngc; ++g) {
                    float tm0 = s0.sc * edge_major(B->ka, B->ka_rows, ngc, b0, e0, g);
                    float tm1 = s1.sc * edge_major(B->ka, B->ka_rows, ngc, b1, e1, g);
                    S->taug[l][B->gofs + g] = ((tm0 + tm1) + self_tau(B, S, l, g)) + for_tau(B, S, l, g);
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefa, 9, sp.js, sp.fs, g);
                }
            } else {
                float rpb = CHI(2, 12) / CHI(1, 12);
                spec_t s0 = specint(colo3, S->rat_o3co2[l], colco2, 4.0f);
                spec_t s1 = specint(colo3, S->rat_o3co2_1[l], colco2, 4.0f);
                spec_t sp = specint(colo3, rpb, colco2, 4.0f);
                int i0 = (jp - 13) * 25 + (jt - 1) * 5 + (s0.js - 1);
                int i1 = (jp - 12) * 25 + (jt1 - 1) * 5 + (s1.js - 1);
                for (int g = 0; g < ngc; ++g) {
                    float m0 = s0.sc * strat_binary(B->kb, B->kb_rows, ngc, i0, g, s0.fs, f00, f10);
                    float m1 = s1.sc * strat_binary(B->kb, B->kb_rows, ngc, i1, g, s1.fs, f01, f11);
                    S->taug[l][B->gofs + g] = (m0 + m1) * corr4[g];
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefb, 5, sp.js, sp.fs, g);
                }
            }
        }
        /* ---- band 5 (lw:2460-2719) ---- */
        {
            const ora_lw_band *B = &L->band[4];
            const int ngc = B->ngc;
            const float wx_ccl4 = S->wx[0][l];
            if (trop) {
                float rpa = CHI(0, 4) / CHI(1, 4), rma = CHI(0, 6) / CHI(1, 6);
                spec_t s0 = specint(colh2o, S->rat_h2oco2[l], colco2, 8.0f);
                spec_t s1 = specint(colh2o, S->rat_h2oco2_1[l], colco2, 8.0f);
                spec_t sm = specint(colh2o, rma, colco2, 8.0f);
                spec_t sp = specint(colh2o, rpa, colco2, 8.0f);
                int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
                int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
                edge_t e0 = edge_factors(s0.sp, s0.fs, f00, f10), e1 = edge_factors(s1.sp, s1.fs, f01, f11);
                for (int g = 0; g < ngc; ++g) {
                    float tm0 = s0.sc * edge_major(B->ka, B->ka_rows, ngc, b0, e0, g);
                    float tm1 = s1.sc * edge_major(B->ka, B->ka_rows, ngc, b1, e1, g);
                    float abso3 = spec_minor(B->ka_mo3, 9, ngc, sm.js, sm.fs, indm, mfrac, g);
                    float tau = ((((tm0 + tm1) + self_tau(B, S, l, g)) + for_tau(B, S, l, g)) + abso3 * colo3) + wx_ccl4 * B->ccl4[g];
                    S->taug[l][B->gofs + g] = tau;
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefa, 9, sp.js, sp.fs, g);
                }
            } else {
                float rpb = CHI(2, 42) / CHI(1, 42);
                spec_t s0 = specint(colo3, S->rat_o3co2[l], colco2, 4.0f);
                spec_t s1 = specint(colo3, S->rat_o3co2_1[l], colco2, 4.0f);
                spec_t sp = specint(colo3, rpb, colco2, 4.0f);
                int i0 = (jp - 13) * 25 + (jt - 1) * 5 + (s0.js - 1);
                int i1 = (jp - 12) * 25 + (jt1 - 1) * 5 + (s1.js - 1);
                for (int g = 0; g < ngc; ++g) {
                    float m0 = s0.sc * strat_binary(B->kb, B->kb_rows, ngc, i0, g, s0.fs, f00, f10);
                    float m1 = s1.sc * strat_binary(B->kb, B->kb_rows, ngc, i1, g, s1.fs, f01, f11);
                    S->taug[l][B->gofs + g] = (m0 + m1) + wx_ccl4 * B->ccl4[g];
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefb, 5, sp.js, sp.fs, g);
                }
            }
        }
        /* ---- band 6 (lw:2722-2863) ---- */
        {
            const ora_lw_band *B = &L->band[5];
            const int ngc = B->ngc;
            float chi_co2 = colco2 / coldry;
            float chi_ref = CHI(1, clampi(jp, 0, 58));
            float ratco2 = 1.0e20f * chi_co2 / chi_ref;
            float adjcolco2 = colco2;
            if (ratco2 > 3.0f) {
                float adjfac = 2.0f + active_pow(fmaxf(ratco2 - 2.0f, 0.0f), 0.77f);
                adjcolco2 = adjfac * chi_ref * coldry * 1.0e-20f;
            }
            for (int g = 0; g < ngc; ++g) {
                float cfc11 = S->wx[1][l] * B->cfc11adj[g];
                float cfc12 = S->wx[2][l] * B->cfc12[g];
                float tau;
                if (trop) {
                    int i0 = ind5((jp - 1) * 5 + (jt - 1), B->ka_rows), i1 = ind5(jp * 5 + (jt1 - 1), B->ka_rows);
                    float major = major4(B->ka, ngc, i0, i1, g, f00, f10, f01, f11);
                    float absco2 = lin_minor(B->ka_mco2, 19, ngc, indm, mfrac, g);
                    tau = ((((colh2o * major + self_tau(B, S, l, g)) + for_tau(B, S, l, g)) + adjcolco2 * absco2) + cfc11) + cfc12;
                } else {
                    tau = cfc11 + cfc12;
                }
                S->taug[l][B->gofs + g] = tau;
                S->fracs[l][B->gofs + g] = B->fracrefa[g];
            }
        }
        /* ---- band 7 (lw:2866-3113) ---- */
        {
            const ora_lw_band *B = &L->band[6];
            const int ngc = B->ngc;
            static const float corr7[12] = {1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 0.92f, 0.88f, 1.07f, 1.1f, 0.99f, 0.855f, 1.0f};
            float chi_co2 = colco2 / coldry;
            float chi_ref = CHI(1, clampi(jp, 0, 58));
            float ratco2 = (1.0e20f * chi_co2) / chi_ref;
            if (trop) {
                float rpa = CHI(0, 2) / CHI(2, 2), rma = CHI(0, 2) / CHI(2, 2);
                spec_t s0 = specint(colh2o, S->rat_h2oo3[l], colo3, 8.0f);
                spec_t s1 = specint(colh2o, S->rat_h2oo3_1[l], colo3, 8.0f);
                spec_t sm = specint(colh2o, rma, colo3, 8.0f);
                spec_t sp = specint(colh2o, rpa, colo3, 8.0f);
                float adjcolco2 = colco2;
                if (ratco2 > 3.0f) {
                    float adjfac = 3.0f + active_pow(ratco2 - 3.0f, 0.79f);
                    adjcolco2 = ((adjfac * chi_ref) * coldry) * 1.0e-20f;
                }
                int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
                int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
                edge_t e0 = edge_factors(s0.sp, s0.fs, f00, f10), e1 = edge_factors(s1.sp, s1.fs, f01, f11);
                for (int g = 0; g < ngc; ++g) {
                    float tm0 = s0.sc * edge_major(B->ka, B->ka_rows, ngc, b0, e0, g);
                    float tm1 = s1.sc * edge_major(B->ka, B->ka_rows, ngc, b1, e1, g);
                    float absco2 = spec_minor(B->ka_mco2, 9, ngc, sm.js, sm.fs, indm, mfrac, g);
                    S->taug[l][B->gofs + g] = (((tm0 + tm1) + self_tau(B, S, l, g)) + for_tau(B, S, l, g)) + adjcolco2 * absco2;
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefa, 9, sp.js, sp.fs, g);
                }
            } else {
                float adjcolco2 = colco2;
                if (ratco2 > 3.0f) {
                    float adjfac = 2.0f + active_pow(ratco2 - 2.0f, 0.79f);
                    adjcolco2 = ((adjfac * chi_ref) * coldry) * 1.0e-20f;
                }
                int i0 = ind5((jp - 13) * 5 + (jt - 1), B->kb_rows), i1 = ind5((jp - 12) * 5 + (jt1 - 1), B->kb_rows);
                for (int g = 0; g < ngc; ++g) {
                    float major = major4(B->kb, ngc, i0, i1, g, f00, f10, f01, f11);
                    float absco2 = lin_minor(B->kb_mco2, 19, ngc, indm, mfrac, g);
                    S->taug[l][B->gofs + g] = (colo3 * major + adjcolco2 * absco2) * corr7[g];
                    S->fracs[l][B->gofs + g] = B->fracrefb[g];
                }
            }
        }
        /* ---- band 8 (lw:3116-3353) ---- */
        {
            const ora_lw_band *B = &L->band[7];
            const int ngc = B->ngc;
            float chi_co2 = colco2 / coldry;
            float chi_ref = CHI(1, clampi(jp, 0, 58));
            float ratco2 = (1.0e20f * chi_co2) / chi_ref;
            float adjcolco2 = colco2;
            if (ratco2 > 3.0f) {
                float adjfac = 2.0f + active_pow(fmaxf(ratco2 - 2.0f, 0.0f), 0.65f);
                adjcolco2 = ((adjfac * chi_ref) * coldry) * 1.0e-20f;
            }
            for (int g = 0; g < ngc; ++g) {
                float cfc12 = S->wx[2][l] * B->cfc12[g];
                float cfc22 = S->wx[3][l] * B->cfc22adj[g];
                float tau;
                if (trop) {
                    int i0 = ind5((jp - 1) * 5 + (jt - 1), B->ka_rows), i1 = ind5(jp * 5 + (jt1 - 1), B->ka_rows);
                    float major = major4(B->ka, ngc, i0, i1, g, f00, f10, f01, f11);
                    float absco2 = lin_minor(B->ka_mco2, 19, ngc, indm, mfrac, g);
                    float abso3 = lin_minor(B->ka_mo3, 19, ngc, indm, mfrac, g);
                    float absn2o = lin_minor(B->ka_mn2o, 19, ngc, indm, mfrac, g);
                    tau = colh2o * major + self_tau(B, S, l, g);
                    tau = tau + for_tau(B, S, l, g);
                    tau = tau + adjcolco2 * absco2;
                    tau = tau + colo3 * abso3;
                    tau = tau + coln2o * absn2o;
                    tau = (tau + cfc12) + cfc22;
                    S->fracs[l][B->gofs + g] = B->fracrefa[g];
                } else {
                    int i0 = ind5((jp - 13) * 5 + (jt - 1), B->kb_rows), i1 = ind5((jp - 12) * 5 + (jt1 - 1), B->kb_rows);
                    float major = major4(B->kb, ngc, i0, i1, g, f00, f10, f01, f11);
                    float absco2 = lin_minor(B->kb_mco2, 19, ngc, indm, mfrac, g);
                    float absn2o = lin_minor(B->kb_mn2o, 19, ngc, indm, mfrac, g);
                    tau = colo3 * major + adjcolco2 * absco2;
                    tau = tau + coln2o * absn2o;
                    tau = (tau + cfc12) + cfc22;
                    S->fracs[l][B->gofs + g] = B->fracrefb[g];
                }
                S->taug[l][B->gofs + g] = tau;
            }
        }
        /* ---- band 9 (lw:3356-3580) ---- */
        {
            const ora_lw_band *B = &L->band[8];
            const int ngc = B->ngc;
            float chi_n2o = coln2o / coldry;
            float chi_ref = CHI(3, clampi(jp, 0, 58));
            float ratn2o = (1.0e20f * chi_n2o) / chi_ref;
            float adjcoln2o = coln2o;
            if (ratn2o > 1.5f) {
                float adjfac = 0.5f + active_pow(ratn2o - 0.5f, 0.65f);
                adjcoln2o = ((adjfac * chi_ref) * coldry) * 1.0e-20f;
            }
            if (trop) {
                float rpa = CHI(0, 8) / CHI(5, 8), rma = CHI(0, 2) / CHI(5, 2);
                spec_t s0 = specint(colh2o, S->rat_h2och4[l], colch4, 8.0f);
                spec_t s1 = specint(colh2o, S->rat_h2och4_1[l], colch4, 8.0f);
                spec_t sm = specint(colh2o, rma, colch4, 8.0f);
                spec_t sp = specint(colh2o, rpa, colch4, 8.0f);
                int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
                int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
                edge_t e0 = edge_factors(s0.sp, s0.fs, f00, f10), e1 = edge_factors(s1.sp, s1.fs, f01, f11);
                for (int g = 0; g < ngc; ++g) {
                    float tm0 = s0.sc * edge_major(B->ka, B->ka_rows, ngc, b0, e0, g);
                    float tm1 = s1.sc * edge_major(B->ka, B->ka_rows, ngc, b1, e1, g);
                    float absn2o = spec_minor(B->ka_mn2o, 9, ngc, sm.js, sm.fs, indm, mfrac, g);
                    S->taug[l][B->gofs + g] = (((tm0 + tm1) + self_tau(B, S, l, g)) + for_tau(B, S, l, g)) + adjcoln2o * absn2o;
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefa, 9, sp.js, sp.fs, g);
                }
            } else {
                int i0 = ind5((jp - 13) * 5 + (jt - 1), B->kb_rows), i1 = ind5((jp - 12) * 5 + (jt1 - 1), B->kb_rows);
                for (int g = 0; g < ngc; ++g) {
                    float major = major4(B->kb, ngc, i0, i1, g, f00, f10, f01, f11);
                    float absn2o = lin_minor(B->kb_mn2o, 19, ngc, indm, mfrac, g);
                    S->taug[l][B->gofs + g] = colch4 * major + adjcoln2o * absn2o;
                    S->fracs[l][B->gofs + g] = B->fracrefb[g];
                }
            }
        }
        /* ---- band 10 (lw:3583-3701) ---- */
        {
            const ora_lw_band *B = &L->band[9];
            const int ngc = B->ngc;
            for (int g = 0; g < ngc; ++g) {
                float tau;
                if (trop) {
                    int i0 = ind5((jp - 1) * 5 + (jt - 1), B->ka_rows), i1 = ind5(jp * 5 + (jt1 - 1), B->ka_rows);
                    float major = major4(B->ka, ngc, i0, i1, g, f00, f10, f01, f11);
                    tau = (colh2o * major + self_tau(B, S, l, g)) + for_tau(B, S, l, g);
                    S->fracs[l][B->gofs + g] = B->fracrefa[g];
                } else {
                    int i0 = ind5((jp - 13) * 5 + (jt - 1), B->kb_rows), i1 = ind5((jp - 12) * 5 + (jt1 - 1), B->kb_rows);
                    float major = major4(B->kb, ngc, i0, i1, g, f00, f10, f01, f11);
                    tau = colh2o * major + for_tau(B, S, l, g);
                    S->fracs[l][B->gofs + g] = B->fracrefb[g];
                }
                S->taug[l][B->gofs + g] = tau;
            }
        }
        /* ---- band 11 (lw:3704-3859) ---- */
        {
            const ora_lw_band *B = &L->band[10];
            const int ngc = B->ngc;
            float scaleo2 = S->colo2[l] * S->scaleminor[l];
            for (int g = 0; g < ngc; ++g) {
                float tau;
                if (trop) {
                    int i0 = ind5((jp - 1) * 5 + (jt - 1), B->ka_rows), i1 = ind5(jp * 5 + (jt1 - 1), B->ka_rows);
                    float major = major4(B->ka, ngc, i0, i1, g, f00, f10, f01, f11);
                    float tauo2 = scaleo2 * lin_minor(B->ka_mo2, 19, ngc, indm, mfrac, g);
                    tau = ((colh2o * major + self_tau(B, S, l, g)) + for_tau(B, S, l, g)) + tauo2;
                    S->fracs[l][B->gofs + g] = B->fracrefa[g];
                } else {
                    int i0 = ind5((jp - 13) * 5 + (jt - 1), B->kb_rows), i1 = ind5((jp - 12) * 5 + (jt1 - 1), B->kb_rows);
                    float major = major4(B->kb, ngc, i0, i1, g, f00, f10, f01, f11);
                    float tauo2 = scaleo2 * lin_minor(B->kb_mo2, 19, ngc, indm, mfrac, g);
                    tau = (colh2o * major + for_tau(B, S, l, g)) + tauo2;
                    S->fracs[l][B->gofs + g] = B->fracrefb[g];
                }
                S->taug[l][B->gofs + g] = tau;
            }
        }
        /* ---- band 12 (lw:3862-3993) ---- */
        {
            const ora_lw_band *B = &L->band[11];
            const int ngc = B->ngc;
            if (trop) {
                float rpa = CHI(0, 9) / CHI(1, 9);
                spec_t s0 = specint(colh2o, S->rat_h2oco2[l], colco2, 8.0f);
                spec_t s1 = specint(colh2o, S->rat_h2oco2_1[l], colco2, 8.0f);
                spec_t sp = specint(colh2o, rpa, colco2, 8.0f);
                int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
                int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
                edge_t e0 = edge_factors(s0.sp, s0.fs, f00, f10), e1 = edge_factors(s1.sp, s1.fs, f01, f11);
                for (int g = 0; g < ngc; ++g) {
                    float tm0 = s0.sc * edge_major(B->ka, B->ka_rows, ngc, b0, e0, g);
                    float tm1 = s1.sc * edge_major(B->ka, B->ka_rows, ngc, b1, e1, g);
                    S->taug[l][B->gofs + g] = ((tm0 + tm1) + self_tau(B, S, l, g)) + for_tau(B, S, l, g);
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefa, 9, sp.js, sp.fs, g);
                }
            } else {
                for (int g = 0; g < ngc; ++g) {
                    S->taug[l][B->gofs + g] = 0.0f;
                    S->fracs[l][B->gofs + g] = 0.0f;
                }
            }
        }
        /* ---- band 13 (lw:3996-4235) ---- */
        {
            const ora_lw_band *B = &L->band[12];
            const int ngc = B->ngc;
            if (trop) {
                float rpa = CHI(0, 4) / CHI(3, 4), rma = CHI(0, 0) / CHI(3, 0), rma3 = CHI(0, 2) / CHI(3, 2);
                spec_t s0 = specint(colh2o, S->rat_h2on2o[l], coln2o, 8.0f);
                spec_t s1 = specint(colh2o, S->rat_h2on2o_1[l], coln2o, 8.0f);
                spec_t sm = specint(colh2o, rma, coln2o, 8.0f);
                float chi_co2 = colco2 / coldry;
                const float co2ref = 3.55e-4f;
                float ratco2 = (1.0e20f * chi_co2) / co2ref;
                float adjcolco2 = colco2;
                if (ratco2 > 3.0f) {
                    float adjfac = 2.0f + active_pow(ratco2 - 2.0f, 0.68f);
                    adjcolco2 = ((adjfac * co2ref) * coldry) * 1.0e-20f;
                }
                spec_t sc = specint(colh2o, rma3, coln2o, 8.0f);
                spec_t sp = specint(colh2o, rpa, coln2o, 8.0f);
                int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
                int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
                edge_t e0 = edge_factors(s0.sp, s0.fs, f00, f10), e1 = edge_factors(s1.sp, s1.fs, f01, f11);
                for (int g = 0; g < ngc; ++g) {
                    float tm0 = s0.sc * edge_major(B->ka, B->ka_rows, ngc, b0, e0, g);
                    float tm1 = s1.sc * edge_major(B->ka, B->ka_rows, ngc, b1, e1, g);
                    float absco2 = spec_minor(B->ka_mco2, 9, ngc, sm.js, sm.fs, indm, mfrac, g);
                    float absco = spec_minor(B->ka_mco, 9, ngc, sc.js, sc.fs, indm, mfrac, g);
                    float tau = (((tm0 + tm1) + self_tau(B, S, l, g)) + for_tau(B, S, l, g)) + adjcolco2 * absco2;
                    S->taug[l][B->gofs + g] = tau + colco * absco;
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefa, 9, sp.js, sp.fs, g);
                }
            } else {
                for (int g = 0; g < ngc; ++g) {
                    float abso3 = lin_minor(B->kb_mo3, 19, ngc, indm, mfrac, g);
                    S->taug[l][B->gofs + g] = colo3 * abso3;
                    S->fracs[l][B->gofs + g] = B->fracrefb[g];
                }
            }
        }
        /* ---- band 14 (lw:4238-4353) ---- */
        {
            const ora_lw_band *B = &L->band[13];
            const int ngc = B->ngc;
            for (int g = 0; g < ngc; ++g) {
                if (trop) {
                    int i0 = ind5((jp - 1) * 5 + (jt - 1), B->ka_rows), i1 = ind5(jp * 5 + (jt1 - 1), B->ka_rows);
                    float major = major4(B->ka, ngc, i0, i1, g, f00, f10, f01, f11);
                    S->taug[l][B->gofs + g] = (colco2 * major + self_tau(B, S, l, g)) + for_tau(B, S, l, g);
                    S->fracs[l][B->gofs + g] = B->fracrefa[g];
                } else {
                    int i0 = ind5((jp - 13) * 5 + (jt - 1), B->kb_rows), i1 = ind5((jp - 12) * 5 + (jt1 - 1), B->kb_rows);
                    float major = major4(B->kb, ngc, i0, i1, g, f00, f10, f01, f11);
                    S->taug[l][B->gofs + g] = colco2 * major;
                    S->fracs[l][B->gofs + g] = B->fracrefb[g];
                }
            }
        }
        /* ---- band 15 (lw:4356-4526) ---- */
        {
            const ora_lw_band *B = &L->band[14];
            const int ngc = B->ngc;
            if (trop) {
                float rpa = CHI(3, 0) / CHI(1, 0), rma = CHI(3, 0) / CHI(1, 0);
                spec_t s0 = specint(coln2o, S->rat_n2oco2[l], colco2, 8.0f);
                spec_t s1 = specint(coln2o, S->rat_n2oco2_1[l], colco2, 8.0f);
                spec_t sm = specint(coln2o, rma, colco2, 8.0f);
                spec_t sp = specint(coln2o, rpa, colco2, 8.0f);
                int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
                int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
                edge_t e0 = edge_factors(s0.sp, s0.fs, f00, f10), e1 = edge_factors(s1.sp, s1.fs, f01, f11);
                float scalen2 = S->colbrd[l] * S->scaleminor[l];
                for (int g = 0; g < ngc; ++g) {
                    float tm0 = s0.sc * edge_major(B->ka, B->ka_rows, ngc, b0, e0, g);
                    float tm1 = s1.sc * edge_major(B->ka, B->ka_rows, ngc, b1, e1, g);
                    float taun2 = scalen2 * spec_minor(B->ka_mn2, 9, ngc, sm.js, sm.fs, indm, mfrac, g);
                    S->taug[l][B->gofs + g] = (((tm0 + tm1) + self_tau(B, S, l, g)) + for_tau(B, S, l, g)) + taun2;
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefa, 9, sp.js, sp.fs, g);
                }
            } else {
                for (int g = 0; g < ngc; ++g) {
                    S->taug[l][B->gofs + g] = 0.0f;
                    S->fracs[l][B->gofs + g] = 0.0f;
                }
            }
        }
        /* ---- band 16 (lw:4529-4682) ---- */
        {
            const ora_lw_band *B = &L->band[15];
            const int ngc = B->ngc;
            if (trop) {
                float rpa = CHI(0, 5) / CHI(5, 5);
                spec_t s0 = specint(colh2o, S->rat_h2och4[l], colch4, 8.0f);
                spec_t s1 = specint(colh2o, S->rat_h2och4_1[l], colch4, 8.0f);
                spec_t sp = specint(colh2o, rpa, colch4, 8.0f);
                int b0 = (jp - 1) * 45 + (jt - 1) * 9 + (s0.js - 1);
                int b1 = jp * 45 + (jt1 - 1) * 9 + (s1.js - 1);
                edge_t e0 = edge_factors(s0.sp, s0.fs, f00, f10), e1 = edge_factors(s1.sp, s1.fs, f01, f11);
                for (int g = 0; g < ngc; ++g) {
                    float tm0 = s0.sc * edge_major(B->ka, B->ka_rows, ngc, b0, e0, g);
                    float tm1 = s1.sc * edge_major(B->ka, B->ka_rows, ngc, b1, e1, g);
                    S->taug[l][B->gofs + g] = ((tm0 + tm1) + self_tau(B, S, l, g)) + for_tau(B, S, l, g);
                    S->fracs[l][B->gofs + g] = frac_interp(B->fracrefa, 9, sp.js, sp.fs, g);
                }
            } else {
                /* nspb(16) = 0: both base rows collapse to 0 (lw:4660-4663) */
                for (int g = 0; g < ngc; ++g) {
                    float major = major4(B->kb, ngc, 0, 0, g, f00, f10, f01, f11);
                    S->taug[l][B->gofs + g] = colch4 * major;
                    S->fracs[l][B->gofs + g] = B->fracrefb[g];
                }
            }
        }
    }
#undef CHI
}

/* ------------------------------------------------------------------------ */
/* clouds: McICA (common:1156-1191) and cldprmc (lw:5725-5830)               */
/* ------------------------------------------------------------------------ */
static int lw_clouds(const ora_cache *C, const ora_in *in, int col, lw_col *S)
{
    const ora_lw_cache *L = &C->lw;
    const int nk = in->nk, nlay = S->nlay;
    float pdel[MAX_LAY];
    for (int k = 0; k < nk; ++k) pdel[k] = S->plev[k] - S->plev[k + 1];
    ora_cloud *cl = &S->cloud;
    ora_cloud_paths(C, in, col, S->tlay, pdel, cl);
    for (int l = nk; l < nlay; ++l) {
        cl->cldfrac[l] = 0.0f; cl->clwp[l] = 0.0f; cl->ciwp[l] = 0.0f; cl->cswp[l] = 0.0f;
        cl->rel[l] = 10.0f; cl->rei[l] = 10.0f; cl->res[l] = 10.0f;
    }
    unsigned char cloudy[LW_NGPT * MAX_LAY];
    ora_mcica_overlap2(S->play, cl->cldfrac, nlay, LW_NGPT, 150, cloudy, S->cdf_work);
    const int icld = in->cldovrlp;
    for (int g = 0; g < LW_NGPT; ++g)
        for (int l = 0; l < nlay; ++l) {
            int c = icld >= 1 ? cloudy[g * nlay + l] : 0;
            S->cldf[g][l] = (unsigned char)c;
            S->ciwp[g][l] = c ? cl->ciwp[l] : 0.0f;
            S->clwp[g][l] = c ? cl->clwp[l] : 0.0f;
            S->cswp[g][l] = c ? cl->cswp[l] : 0.0f;
        }
    const int inflag = icld >= 1 ? cl->inflg : 0;
    const int iceflag = icld >= 1 ? cl->iceflg : 0;
    const int liqflag = icld >= 1 ? cl->liqflg : 0;
    if (inflag == 0) {
        for (int g = 0; g < LW_NGPT; ++g)
            for (int l = 0; l < nlay; ++l) S->taucmc[g][l] = 0.0f;
        return 0;
    }
    if (iceflag < 3 || liqflag != 1) return -2;   /* only reachable flag combinations */
    for (int g = 0; g < LW_NGPT; ++g) {
        int band = 0;
        while (g >= L->band[band].gofs + L->band[band].ngc) ++band;
        for (int l = 0; l < nlay; ++l) {
            float cldf = (float)S->cldf[g][l];
            float ciwp = S->ciwp[g][l], clwp = S->clwp[g][l], cswp = S->cswp[g][l];
            float cwp = (ciwp + clwp) + cswp;
            const float tau_in = 0.0f;
            int active = (cldf >= 1.0e-20f) && ((cwp >= 1.0e-20f) || (tau_in >= 1.0e-20f));
            float radice = S->cloud.rei[l], radliq = S->cloud.rel[l], radsno = S->cloud.res[l];
            float factor = (radice - 2.0f) / 3.0f;
            int index = (int)factor;
            if (index == 46) index = 45;
            float fint = factor - (float)index;
            float abscoice = interpf(L->absice3[jrow(index - 1, 46) * 16 + band],
                                     L->absice3[jrow(index, 46) * 16 + band], fint);
            float abscosno = 0.0f;
            if ((ciwp + cswp) == 0.0f) { abscoice = 0.0f; abscosno = 0.0f; }
            if (iceflag == 5 && cswp > 0.0f) {
                float fs = (radsno - 2.0f) / 3.0f;
                int is = (int)fs;
                if (is == 46) is = 45;
                float fints = fs - (float)is;
                abscosno = interpf(L->absice3[jrow(is - 1, 46) * 16 + band], L->absice3[jrow(is, 46) * 16 + band], fints);
            }
            int il = (int)(radliq - 1.5f);
            if (il == 0) il = 1;
            if (il == 58) il = 57;
            float fl = (radliq - 1.5f) - (float)il;
            float abscoliq = clwp == 0.0f ? 0.0f
                : interpf(L->absliq1[jrow(il - 1, 58) * 16 + band], L->absliq1[jrow(il, 58) * 16 + band], fl);
            float tau = (ciwp * abscoice + clwp * abscoliq) + cswp * abscosno;
            S->taucmc[g][l] = active ? tau : tau_in;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* rtrnmc (lw:5140-5262, 5476-5722)                                          */
/* ------------------------------------------------------------------------ */
static inline int pade_index(const ora_lw_cache *L, float od)
{
    float tblind = od / (L->bpade + od);
    float pos = (float)L->ntbl * tblind + 0.5f;
    return clampi((int)pos, 0, L->ntbl);
}

static void lw_rtrnmc(const ora_lw_cache *L, lw_col *S)
{
    const int n = S->nlay;
    float secdiff[LW_NBND];
    for (int b = 0; b < LW_NBND; ++b) {
        int variable = !(b == 0 || b == 3 || b >= 9);
        if (variable) {
            float e = expf(LW_A2[b] * S->pwvcm);
            float v = LW_A0[b] + LW_A1[b] * e;
            secdiff[b] = v < 1.50f ? 1.50f : (v > 1.80f ? 1.80f : v);
        } else {
            secdiff[b] = 1.66f;
        }
    }
    int icldlyr[MAX_LAY];
    for (int l = 0; l < n; ++l) {
        int any = 0;
        for (int g = 0; g < LW_NGPT; ++g) any |= S->cldf[g][l];
        icldlyr[l] = any;
    }
    const float rec_6 = 0.166667f;
    for (int g = 0; g < LW_NGPT; ++g) {
        int band = 0;
        while (g >= L->band[band].gofs + L->band[band].ngc) ++band;
        const float sd = secdiff[band];
        float atr[MAX_LAY], bbug[MAX_LAY], bbut[MAX_LAY], atot_l[MAX_LAY], efcl[MAX_LAY];
        float radld = 0.0f, radclrd = 0.0f;
        int iclddn = 0;
        S->drad[n][g] = 0.0f;
        S->clrdrad[n][g] = 0.0f;
        for (int l = n - 1; l >= 0; --l) {
            float plfrac = S->fracs[l][g], blay = S->planklay[l][band];
            float dplankup = S->planklev[l + 1][band] - blay;
            float dplankdn = S->planklev[l][band] - blay;
            float odepth = sd * S->taug[l][g];
            if (odepth < 0.0f) odepth = 0.0f;
            int cldf = S->cldf[g][l];
            float odcld_raw = sd * S->taucmc[g][l];
            float abscld = 1.0f - cloud_expf(-odcld_raw);
            float odcld = cldf ? odcld_raw : 0.0f;
            float efclfrac = cldf ? abscld * (float)cldf : 0.0f;
            efcl[l] = efclfrac;
            int cloudy = icldlyr[l];
            if (cloudy) iclddn = 1;
            float a, bbugas, bbutot = 0.0f, atot = 0.0f, bbd_for_clear, radld_new;
            if (cloudy) {
                /* _rtrnmc_cloudy_terms (lw:5207-5262) */
                float odtot = odepth + odcld;
                float gassrc, bbdtot, bbdgas;
                if (odtot < 0.06f) {
                    float odepth_rec = rec_6 * odepth, odtot_rec = rec_6 * odtot;
                    a = odepth - 0.5f * odepth * odepth;
                    gassrc = plfrac * (blay + dplankdn * odepth_rec) * a;
                    atot = odtot - 0.5f * odtot * odtot;
                    bbdtot = plfrac * (blay + dplankdn * odtot_rec);
                    bbdgas = plfrac * (blay + dplankdn * odepth_rec);
                    bbugas = plfrac * (blay + dplankup * odepth_rec);
                    bbutot = plfrac * (blay + dplankup * odtot_rec);
                } else if (odepth <= 0.06f) {
                    float odepth_rec = rec_6 * odepth;
                    a = odepth - 0.5f * odepth * odepth;
                    gassrc = plfrac * (blay + dplankdn * odepth_rec) * a;
                    int it = pade_index(L, odtot);
                    float tfactot = L->pade_tfn[it];
                    atot = 1.0f - L->pade_exp[it];
                    bbdtot = plfrac * (blay + tfactot * dplankdn);
                    bbdgas = plfrac * (blay + dplankdn * odepth_rec);
                    bbugas = plfrac * (blay + dplankup * odepth_rec);
                    bbutot = plfrac * (blay + tfactot * dplankup);
                } else {
                    int ig = pade_index(L, odepth);
                    float odtbl = L->pade_tau[ig];
                    a = 1.0f - L->pade_exp[ig];
                    float tfacgas = L->pade_tfn[ig];
                    gassrc = a * plfrac * (blay + tfacgas * dplankdn);
                    float odtot3 = odtbl + odcld;
                    int it = pade_index(L, odtot3);
                    float tfactot = L->pade_tfn[it];
                    atot = 1.0f - L->pade_exp[it];
                    bbdtot = plfrac * (blay + tfactot * dplankdn);
                    bbdgas = plfrac * (blay + tfacgas * dplankdn);
                    bbugas = plfrac * (blay + tfacgas * dplankup);
                    bbutot = plfrac * (blay + tfactot * dplankup);
                }
                float cf = (float)cldf;
                radld_new = radld - radld * (a + efclfrac * (1.0f - a)) + gassrc + cf * (bbdtot * atot - gassrc);
                bbd_for_clear = bbdgas;
            } else {
                /* _rtrnmc_clear_terms (lw:5157-5204) */
                float bbd;
                if (odepth <= 0.06f) {
                    float odepth_rec = rec_6 * odepth;
                    a = odepth - (0.5f * odepth) * odepth;
                    bbd = plfrac * (blay + dplankdn * odepth_rec);
                    bbugas = plfrac * (blay + dplankup * odepth_rec);
                } else {
                    int it = pade_index(L, odepth);
                    a = 1.0f - L->pade_exp[it];
                    float tausfac = L->pade_tfn[it];
                    bbd = plfrac * (blay + tausfac * dplankdn);
                    bbugas = plfrac * (blay + tausfac * dplankup);
                }
                radld_new = radld + (bbd - radld) * a;
                bbd_for_clear = bbd;
            }
            float radclrd_new = iclddn ? radclrd + (bbd_for_clear - radclrd) * a : radld_new;
            radld = radld_new;
            radclrd = radclrd_new;
            S->drad[l][g] = radld;
            S->clrdrad[l][g] = radclrd;
            atr[l] = a;
            bbug[l] = bbugas;
            bbut[l] = bbutot;
            atot_l[l] = atot;
        }
        /* surface (lw:5648-5655) */
        float rad0 = S->fracs[0][g] * S->plankbnd[band];
        float reflect = 1.0f - S->semiss;
        float radlu = rad0 + reflect * radld;
        float radclru = rad0 + reflect * radclrd;
        S->urad[0][g] = radlu;
        S->clrurad[0][g] = radclru;
        for (int l = 0; l < n; ++l) {
            float a = atr[l];
            float radlu_new;
            if (icldlyr[l]) {
                float gas = bbug[l] * a;
                float cf = (float)S->cldf[g][l];
                radlu_new = radlu - radlu * (a + efcl[l] * (1.0f - a)) + gas + cf * (bbut[l] * atot_l[l] - gas);
            } else {
                radlu_new = radlu + (bbug[l] - radlu) * a;
            }
            float radclru_new = iclddn ? radclru + (bbug[l] - radclru) * a : radlu_new;
            radlu = radlu_new;
            radclru = radclru_new;
            S->urad[l + 1][g] = radlu;
            S->clrurad[l + 1][g] = radclru;
        }
    }
    /* g-point and band sums (lw:170-199), then fluxes and heating (lw:5702-5712) */
    const float pi = 3.1415926535897932384626433832795f;
    const float fluxfac = pi * 2.0e4f;
    const float heatfac = (9.8066f * 8.6400e4f) / (1004.5f * 1.0e2f);
    float (*rads[4])[LW_NGPT] = {S->urad, S->drad, S->clrurad, S->clrdrad};
    float *tots[4] = {S->totuflux, S->totdflux, S->totuclfl, S->totdclfl};
    for (int q = 0; q < 4; ++q) {
        for (int lev = 0; lev <= n; ++lev) {
            float total = 0.0f;
            for (int b = 0; b < LW_NBND; ++b) {
                float bandsum = 0.0f;
                for (int g = L->band[b].gofs; g < L->band[b].gofs + L->band[b].ngc; ++g)
                    bandsum = bandsum + rads[q][lev][g];
                float bflux = bandsum * 0.5f;
                total = total + bflux * LW_DELWAVE[b];
            }
            tots[q][lev] = total * fluxfac;
        }
    }
    for (int l = 0; l < n; ++l) {
        float fnet0 = S->totuflux[l] - S->totdflux[l], fnet1 = S->totuflux[l + 1] - S->totdflux[l + 1];
        float fnetc0 = S->totuclfl[l] - S->totdclfl[l], fnetc1 = S->totuclfl[l + 1] - S->totdclfl[l + 1];
        float dp = S->plev[l] - S->plev[l + 1];
        S->htr[l] = heatfac * (fnet0 - fnet1) / dp;
        S->htrc[l] = heatfac * (fnetc0 - fnetc1) / dp;
        if (l >= S->fp64_from) {
            /* FP64 mode: net fluxes, their difference and dF/dp in binary64 */
            S->htr[l] = ora_heating64(heatfac, S->totuflux[l], S->totdflux[l], S->totuflux[l + 1],
                                      S->totdflux[l + 1], S->plev[l], S->plev[l + 1]);
            S->htrc[l] = ora_heating64(heatfac, S->totuclfl[l], S->totdclfl[l], S->totuclfl[l + 1],
                                       S->totdclfl[l + 1], S->plev[l], S->plev[l + 1]);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* driver                                                                    */
/* ------------------------------------------------------------------------ */
typedef struct { const ora_cache *C; const ora_in *in; ora_out *out; int nlay; } lw_job;

static int lw_one_column(void *ctx, int col)
{
    lw_job *J = (lw_job *)ctx;
    const ora_cache *C = J->C;
    const ora_in *in = J->in;
    ora_out *out = J->out;
    const int nk = in->nk, nlay = J->nlay;
    lw_col *S = (lw_col *)malloc(sizeof(lw_col));
    if (!S) return 1;
    lw_prepare(C, in, col, S);
    lw_inatm(S);
    if (lw_clouds(C, in, col, S) != 0) { free(S); return 2; }
    lw_setcoef(&C->lw, S);
    lw_taumol(&C->lw, S);
    lw_rtrnmc(&C->lw, S);
    /* WRF outputs (lw:7035-7077) */
    const float *pi3d = in->pi3d + (size_t)col * nk;
    for (int k = 0; k < nk; ++k) {
        out->rthraten[(size_t)col * nk + k] = (S->htr[k] / 86400.0f) / pi3d[k];
        out->rthratenc[(size_t)col * nk + k] = (S->htrc[k] / 86400.0f) / pi3d[k];
    }
    out->up_top[col] = S->totuflux[nlay];
    out->upc_top[col] = S->totuclfl[nlay];
    out->dn_top[col] = S->totdflux[nlay];
    out->dnc_top[col] = S->totdclfl[nlay];
    out->up_sfc[col] = S->totuflux[0];
    out->upc_sfc[col] = S->totuclfl[0];
    out->dn_sfc[col] = S->totdflux[0];
    out->dnc_sfc[col] = S->totdclfl[0];
    if (out->taug)
        for (int l = 0; l < nlay; ++l)
            for (int g = 0; g < LW_NGPT; ++g) {
                out->taug[((size_t)col * nlay + l) * LW_NGPT + g] = S->taug[l][g];
                out->fracs_or_taur[((size_t)col * nlay + l) * LW_NGPT + g] = S->fracs[l][g];
            }
    if (out->cldfmc)
        for (int g = 0; g < LW_NGPT; ++g)
            for (int l = 0; l < nlay; ++l) {
                out->cldfmc[((size_t)col * LW_NGPT + g) * nlay + l] = (float)S->cldf[g][l];
                out->taucmc[((size_t)col * LW_NGPT + g) * nlay + l] = S->taucmc[g][l];
            }
    if (out->uflx)
        for (int lev = 0; lev <= nlay; ++lev) {
            out->uflx[(size_t)col * (nlay + 1) + lev] = S->totuflux[lev];
            out->dflx[(size_t)col * (nlay + 1) + lev] = S->totdflux[lev];
            out->uflxc[(size_t)col * (nlay + 1) + lev] = S->totuclfl[lev];
            out->dflxc[(size_t)col * (nlay + 1) + lev] = S->totdclfl[lev];
        }
    if (out->hr)
        for (int l = 0; l < nlay; ++l) {
            out->hr[(size_t)col * nlay + l] = S->htr[l];
            out->hrc[(size_t)col * nlay + l] = S->htrc[l];
        }
    free(S);
    return 0;
}

int ora_lw_columns(const ora_tables *t, const ora_in *in, ora_out *out, int nthreads)
{
    const int nlay = ora_lw_nlayers(in->p_top, in->nk);
    if (in->nk < 4 || nlay > MAX_LAY) return -1;
    lw_job J = {ora_cache_of(t), in, out, nlay};
    return ora_parallel_for(in->ncol, nthreads, lw_one_column, &J);
}

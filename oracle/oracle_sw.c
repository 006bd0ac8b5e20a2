/*
 * Oracle: RRTMG shortwave restatement (test infrastructure only).
 * Reference file: src/wrf_jax/physics/module_ra_rrtmg_sw.py ("sw:").
 * The reference's WRF adapter calls every kernel with rounding_token=None,
 * so each statement is one binary32 operation in the order written.
 */
#include "oracle_internal.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ONEMINUS (1.0f - 1.0e-6f)

static const int SW_NGC[SW_NBND] = {6, 12, 8, 8, 10, 10, 2, 10, 8, 6, 6, 8, 6, 12};

int ora_sw_cache_init(const ora_tables *t, ora_sw_cache *c)
{
    char name[64];
    int gofs = 0;
    for (int b = 0; b < SW_NBND; ++b) {
        ora_sw_band *B = &c->band[b];
        const int bn = b + 16;
        B->ngc = SW_NGC[b];
        B->gofs = gofs;
        gofs += B->ngc;
        int n;
#define GET(field) (snprintf(name, sizeof name, "sw%d." #field, bn), (const float *)ora_table(t, name, &n))
        B->ka = GET(ka);
        B->ka_rows = B->ka ? n / B->ngc : 0;
        B->kb = GET(kb);
        B->kb_rows = B->kb ? n / B->ngc : 0;
        B->selfref = GET(selfref);
        B->forref = GET(forref);
        B->forref_rows = B->forref ? n / B->ngc : 0;
        B->sfluxref = GET(sfluxref);
        B->sflux_cols = B->sfluxref ? n / B->ngc : 0;
        B->rayla = GET(rayla);
        B->raylb = GET(raylb);
        B->absch4 = GET(absch4);
        B->abso3a = GET(abso3a);
        B->abso3b = GET(abso3b);
        B->absh2o = GET(absh2o);
        B->absco2 = GET(absco2);
        const float *rayl = GET(rayl);
        if (rayl && n == 1) { B->rayl = rayl[0]; B->rayl_g = NULL; }
        else { B->rayl_g = rayl; B->rayl = 0.0f; }
        const float *v;
        v = GET(strrat);   B->strrat = v ? v[0] : 0.0f;
        v = GET(strrat1);  B->strrat1 = v ? v[0] : 0.0f;
        v = GET(givfac);   B->givfac = v ? v[0] : 0.0f;
        v = GET(scalekur); B->scalekur = v ? v[0] : 0.0f;
        const int32_t *lr = (const int32_t *)GET(layreffr);
        B->layreffr = lr ? lr[0] : 0;
#undef GET
        if (!B->sfluxref) return -1;
    }
#define T(field) (const float *)ora_table(t, "sw." #field, NULL)
    c->preflog = T(preflog);
    c->tref = T(tref);
    c->extliq1 = T(extliq1); c->ssaliq1 = T(ssaliq1); c->asyliq1 = T(asyliq1);
    c->extice2 = T(extice2); c->ssaice2 = T(ssaice2); c->asyice2 = T(asyice2);
    c->extice3 = T(extice3); c->ssaice3 = T(ssaice3); c->asyice3 = T(asyice3); c->fdlice3 = T(fdlice3);
    c->abari = T(abari); c->bbari = T(bbari); c->cbari = T(cbari);
    c->dbari = T(dbari); c->ebari = T(ebari); c->fbari = T(fbari);
#undef T
    int n;
    c->pade_exp = (const float *)ora_table(t, "sw.pade_exp_tbl", &n);
    c->ntbl = n - 1;
    const float *bp = (const float *)ora_table(t, "sw.pade_bpade", NULL);
    if (!c->preflog || !c->tref || !c->extliq1 || !c->extice3 || !c->pade_exp || !bp) return -1;
    c->bpade = bp[0];
    return 0;
}

/* ------------------------------------------------------------------------ */
typedef struct {
    int nlay, laytrop;
    int fp64_from;     /* first layer whose heating is formed in binary64 (FP64 mode) */
    int fp64_reftra;   /* FP64 mode: reftra in binary64 when zwo >= 0.999 */
    float play[MAX_LAY], plev[MAX_LAY + 1], tlay[MAX_LAY], tlev[MAX_LAY + 1];
    float h2o[MAX_LAY], o3[MAX_LAY];
    float coldry[MAX_LAY], wkl[7][MAX_LAY], pdp[MAX_LAY], adjflux;
    int jp[MAX_LAY], jt[MAX_LAY], jt1[MAX_LAY], indself[MAX_LAY], indfor[MAX_LAY];
    float colh2o[MAX_LAY], colco2[MAX_LAY], colo3[MAX_LAY], coln2o[MAX_LAY], colch4[MAX_LAY];
    float colo2[MAX_LAY], colmol[MAX_LAY];
    float fac00[MAX_LAY], fac01[MAX_LAY], fac10[MAX_LAY], fac11[MAX_LAY];
    float selffac[MAX_LAY], selffrac[MAX_LAY], forfac[MAX_LAY], forfrac[MAX_LAY];
    float taug[MAX_LAY][SW_NGPT], taur[MAX_LAY][SW_NGPT], sfluxzen[SW_NGPT];
    unsigned char cldf[SW_NGPT][MAX_LAY];
    float ciwp[SW_NGPT][MAX_LAY], clwp[SW_NGPT][MAX_LAY], cswp[SW_NGPT][MAX_LAY];
    float taucmc[SW_NGPT][MAX_LAY], ssacmc[SW_NGPT][MAX_LAY], asmcmc[SW_NGPT][MAX_LAY], taormc[SW_NGPT][MAX_LAY];
    ora_cloud cloud;
    ora_binary32 cdf_work[SW_NGPT * MAX_LAY];
    /* spectral flux sums, bottom-up levels */
    float bbfu[MAX_LAY + 1], bbfd[MAX_LAY + 1], bbcu[MAX_LAY + 1], bbcd[MAX_LAY + 1];
    float bbfddir[MAX_LAY + 1], bbcddir[MAX_LAY + 1];
    float swhr[MAX_LAY], swhrc[MAX_LAY];
} sw_col;

/* adapter (sw:2442-2580) */
static void sw_prepare(const ora_cache *C, const ora_in *in, int col, sw_col *S)
{
    const int nk = in->nk, nlay = nk + 1;
    S->nlay = nlay;
    S->fp64_from = in->fp64_steps ? (in->nk > 5 ? in->nk - 5 : 0) : MAX_LAY + 1;
    S->fp64_reftra = in->fp64_steps;
    const float *p3d = in->p3d + (size_t)col * nk;
    const float *t3d = in->t3d + (size_t)col * nk;
    const float *p8w = in->p8w + (size_t)col * (nk + 1);
    const float *t8w = in->t8w + (size_t)col * (nk + 1);
    const float *qv = in->qv + (size_t)col * nk;
    const float *o3 = in->o3 + (size_t)col * nk;
    for (int k = 0; k <= nk; ++k) S->plev[k] = ora_pa_to_hpa(p8w[k]);
    S->plev[nk + 1] = 1.0e-5f;
    for (int k = 0; k <= nk; ++k) S->tlev[k] = t8w[k];
    S->tlev[nk + 1] = t8w[nk];
    for (int k = 0; k < nk; ++k) S->play[k] = ora_pa_to_hpa(p3d[k]);
    S->play[nk] = 0.5f * S->plev[nk];
    for (int k = 0; k < nk; ++k) S->tlay[k] = t3d[k];
    S->tlay[nk] = t8w[nk];
    for (int l = 0; l < nlay; ++l) {
        int k = l < nk ? l : nk - 1;
        S->h2o[l] = fmaxf(qv[k], 1.0e-12f) * 1.607793f;
    }
    float o3mmr[MAX_LAY];
    ora_o3data(C, S->plev, nk + 1, o3mmr);
    const float amdo = 0.603461f;
    for (int k = 0; k < nk; ++k) S->o3[k] = o3[k];
    float top = (o3[nk - 1] - o3mmr[nk - 1] * amdo) + o3mmr[nk] * amdo;
    if (top <= 0.0f) top = o3mmr[nk] * amdo;
    S->o3[nk] = top;
}

/* inatm_sw (sw:1250-1406, 114-150) */
static void sw_inatm(const ora_in *in, sw_col *S)
{
    const int n = S->nlay;
    const float amd = 28.9660f, amw = 18.0160f, avogad = 6.02214199e23f, grav = 9.8066f;
    for (int l = 0; l < n; ++l) {
        float h2o = S->h2o[l];
        S->pdp[l] = S->plev[l] - S->plev[l + 1];
        float amm = (1.0f - h2o) * amd + h2o * amw;
        float num = (S->pdp[l] * 1.0e3f) * avogad;
        float den = ((1.0e2f * grav) * amm) * (1.0f + h2o);
        float coldry = num / den;
        S->coldry[l] = coldry;
        float vmr[7] = {h2o, in->co2, S->o3[l], in->n2o, 0.0f, in->ch4, 0.209488f};
        for (int m = 0; m < 7; ++m) S->wkl[m][l] = vmr[m] * coldry;
    }
    float solvar = in->solcon / 1.36822e3f;
    S->adjflux = 1.0f * solvar;
}

/* clouds: McICA (common:1194-1240) + cldprmc_sw (sw:1409-1626) */
static int sw_clouds(const ora_cache *C, const ora_in *in, int col, sw_col *S, int icld)
{
    const ora_sw_cache *W = &C->sw;
    const int nk = in->nk, n = S->nlay;
    float pdel[MAX_LAY];
    for (int k = 0; k < nk; ++k) pdel[k] = S->plev[k] - S->plev[k + 1];
    ora_cloud *cl = &S->cloud;
    ora_cloud_paths(C, in, col, S->tlay, pdel, cl);
    cl->cldfrac[nk] = 0.0f; cl->clwp[nk] = 0.0f; cl->ciwp[nk] = 0.0f; cl->cswp[nk] = 0.0f;
    cl->rel[nk] = 10.0f; cl->rei[nk] = 10.0f; cl->res[nk] = 10.0f;
    unsigned char cloudy[SW_NGPT * MAX_LAY];
    ora_mcica_overlap2(S->play, cl->cldfrac, n, SW_NGPT, 1, cloudy, S->cdf_work);
    const int iceflag = cl->iceflg;
    for (int g = 0; g < SW_NGPT; ++g)
        for (int l = 0; l < n; ++l) {
            int c = icld >= 1 ? cloudy[g * n + l] : 0;
            S->cldf[g][l] = (unsigned char)c;
            S->ciwp[g][l] = c ? cl->ciwp[l] : 0.0f;
            S->clwp[g][l] = c ? cl->clwp[l] : 0.0f;
            S->cswp[g][l] = (c && iceflag == 5) ? cl->cswp[l] : 0.0f;
        }
    if (icld == 0) {
        for (int g = 0; g < SW_NGPT; ++g)
            for (int l = 0; l < n; ++l) {
                S->taucmc[g][l] = 0.0f; S->taormc[g][l] = 0.0f;
                S->asmcmc[g][l] = 0.0f; S->ssacmc[g][l] = 1.0f;
            }
        return 0;
    }
    if (cl->inflg < 2 || cl->liqflg != 1 || iceflag < 3) return -2;
    const float cldmin = 1.0e-20f;
    for (int g = 0; g < SW_NGPT; ++g) {
        int band = 0;
        while (g >= W->band[band].gofs + W->band[band].ngc) ++band;
        for (int l = 0; l < n; ++l) {
            float cldf = (float)S->cldf[g][l];
            float ciwp = S->ciwp[g][l], clwp = S->clwp[g][l], cswp = S->cswp[g][l];
            const float tau_in = 0.0f, ssa_in = 1.0f, asm_in = 0.0f;
            float cwp = (ciwp + clwp) + cswp;
            int active = (cldf >= cldmin) && ((cwp >= cldmin) || (tau_in >= cldmin));
            if (!active) {
                S->taucmc[g][l] = tau_in; S->ssacmc[g][l] = ssa_in;
                S->asmcmc[g][l] = asm_in; S->taormc[g][l] = tau_in;
                continue;
            }
            float radice = cl->rei[l];
            float radliq = cl->rel[l];
            float radsno = iceflag == 5 ? cl->res[l] : 0.0f;
            /* ice, iceflag >= 3 (sw:1503-1512) */
            float factor = (radice - 2.0f) / 3.0f;
            int index = (int)factor;
            if (index == 46) index = 45;
            float fint = factor - (float)index;
            int r0 = jrow(index - 1, 46), r1 = jrow(index, 46);
            float extice = interpf(W->extice3[r0 * 14 + band], W->extice3[r1 * 14 + band], fint);
            float ssaice = interpf(W->ssaice3[r0 * 14 + band], W->ssaice3[r1 * 14 + band], fint);
            float gice = interpf(W->asyice3[r0 * 14 + band], W->asyice3[r1 * 14 + band], fint);
            float fdelta = interpf(W->fdlice3[r0 * 14 + band], W->fdlice3[r1 * 14 + band], fint);
            float fw = fdelta + 0.5f / ssaice;
            float forwice = fw > gice ? gice : fw;
            if ((ciwp + cswp) == 0.0f) { extice = 0.0f; ssaice = 0.0f; gice = 0.0f; forwice = 0.0f; }
            float extsno = 0.0f, ssasno = 0.0f, gsno = 0.0f, forwsno = 0.0f;
            if (iceflag == 5 && cswp > 0.0f) {
                float fs = (radsno - 2.0f) / 3.0f;
                int is = (int)fs;
                if (is == 46) is = 45;
                float fints = fs - (float)is;
                int s0 = jrow(is - 1, 46), s1 = jrow(is, 46);
                extsno = interpf(W->extice3[s0 * 14 + band], W->extice3[s1 * 14 + band], fints);
                ssasno = interpf(W->ssaice3[s0 * 14 + band], W->ssaice3[s1 * 14 + band], fints);
                gsno = interpf(W->asyice3[s0 * 14 + band], W->asyice3[s1 * 14 + band], fints);
                float fds = interpf(W->fdlice3[s0 * 14 + band], W->fdlice3[s1 * 14 + band], fints);
                float fw2 = fds + 0.5f / ssasno;
                forwsno = fw2 > gsno ? gsno : fw2;
            }
            /* liquid (sw:1544-1557) */
            float fl = radliq - 1.5f;
            int il = (int)fl;
            if (il == 0) il = 1;
            if (il == 58) il = 57;
            float fint_liq = (radliq - 1.5f) - (float)il;
            int q0 = jrow(il - 1, 58), q1 = jrow(il, 58);
            float extliq = interpf(W->extliq1[q0 * 14 + band], W->extliq1[q1 * 14 + band], fint_liq);
            float ssaliq = interpf(W->ssaliq1[q0 * 14 + band], W->ssaliq1[q1 * 14 + band], fint_liq);
            if (fint_liq < 0.0f && ssaliq > 1.0f) ssaliq = W->ssaliq1[q0 * 14 + band];
            float gliq = interpf(W->asyliq1[q0 * 14 + band], W->asyliq1[q1 * 14 + band], fint_liq);
            if (clwp == 0.0f) { extliq = 0.0f; ssaliq = 0.0f; gliq = 0.0f; }
            float forwliq = gliq * gliq;
            float tauliqorig = clwp * extliq;
            float tauiceorig = ciwp * extice;
            float ssaliq_d = ssaliq * (1.0f - forwliq) / (1.0f - forwliq * ssaliq);
            float tauliq = (1.0f - forwliq * ssaliq) * tauliqorig;
            float ssaice_d = ssaice * (1.0f - forwice) / (1.0f - forwice * ssaice);
            float tauice = (1.0f - forwice * ssaice) * tauiceorig;
            float scatliq = ssaliq_d * tauliq;
            float scatice = ssaice_d * tauice;
            float tau_new, taor_new, scatsno = 0.0f;
            if (iceflag == 5) {
                float tausnoorig = cswp * extsno;
                float ssasno_d = ssasno * (1.0f - forwsno) / (1.0f - forwsno * ssasno);
                float tausno = (1.0f - forwsno * ssasno) * tausnoorig;
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
            float ssa_new, asm_new;
            if (iceflag == 5) {
                float ssum = (scatliq + scatice) + scatsno;
                ssa_new = ssum / tau_new;
                float num = (scatliq * (gliq - forwliq) / (1.0f - forwliq) + scatice * (gice - forwice) / (1.0f - forwice))
                            + scatsno * (gsno - forwsno) / (1.0f - forwsno);
                asm_new = num / ssum;
            } else {
                float ssum = scatliq + scatice;
                ssa_new = ssum / tau_new;
                float num = scatliq * (gliq - forwliq) / (1.0f - forwliq) + scatice * (gice - forwice) / (1.0f - forwice);
                asm_new = num / ssum;
            }
            S->taucmc[g][l] = tau_new;
            S->ssacmc[g][l] = ssa_new;
            S->asmcmc[g][l] = asm_new;
            S->taormc[g][l] = taor_new;
        }
    }
    return 0;
}

/* setcoef_sw (sw:7101-7306) */
static void sw_setcoef(const ora_sw_cache *W, sw_col *S)
{
    const int n = S->nlay;
    const float stpfac = 296.0f / 1013.0f;
    int laytrop = 0;
    for (int l = 0; l < n; ++l) {
        float pavel = S->play[l], tavel = S->tlay[l], coldry = S->coldry[l];
        float plog = logf(pavel);
        int jp = clampi((int)(36.0f - 5.0f * (plog + 0.04f)), 1, 58);
        float fp = 5.0f * (W->preflog[jp - 1] - plog);
        float tf = (tavel - W->tref[jp - 1]) / 15.0f;
        int jt = clampi((int)(3.0f + tf), 1, 4);
        float ft = tf - (float)(jt - 3);
        float tf1 = (tavel - W->tref[jp]) / 15.0f;
        int jt1 = clampi((int)(3.0f + tf1), 1, 4);
        float ft1 = tf1 - (float)(jt1 - 3);
        float water = S->wkl[0][l] / coldry;
        float scalefac = (pavel * stpfac) / tavel;
        int trop = plog > 4.56f;
        laytrop += trop;
        float forfac = scalefac / (1.0f + water);
        float ftf = (332.0f - tavel) / 36.0f;
        int indfor_t = clampi((int)ftf, 1, 2);
        float forfrac_t = ftf - (float)indfor_t;
        float fsf = (tavel - 188.0f) / 36.0f;
        S->indfor[l] = trop ? indfor_t : 3;
        S->forfrac[l] = trop ? forfrac_t : fsf - 1.0f;
        float selffac_t = water * forfac;
        float fself = (tavel - 188.0f) / 7.2f;
        int indself_t = clampi((int)fself - 7, 1, 9);
        float selffrac_t = fself - (float)(indself_t + 7);
        S->indself[l] = trop ? indself_t : 0;
        S->selffac[l] = trop ? selffac_t : 0.0f;
        S->selffrac[l] = trop ? selffrac_t : 0.0f;
        S->forfac[l] = forfac;
        const float cs = 1.0e-20f;
        S->colh2o[l] = cs * S->wkl[0][l];
        S->colco2[l] = cs * S->wkl[1][l];
        S->colo3[l] = cs * S->wkl[2][l];
        S->coln2o[l] = cs * S->wkl[3][l];
        S->colch4[l] = cs * S->wkl[5][l];
        S->colo2[l] = cs * S->wkl[6][l];
        S->colmol[l] = cs * coldry + S->colh2o[l];
        float fallback = 1.0e-32f * coldry;
        if (S->colco2[l] == 0.0f) S->colco2[l] = fallback;
        if (S->coln2o[l] == 0.0f) S->coln2o[l] = fallback;
        if (S->colch4[l] == 0.0f) S->colch4[l] = fallback;
        if (S->colo2[l] == 0.0f) S->colo2[l] = fallback;
        float compfp = 1.0f - fp;
        S->fac10[l] = compfp * ft;
        S->fac00[l] = compfp * (1.0f - ft);
        S->fac11[l] = fp * ft1;
        S->fac01[l] = fp * (1.0f - ft1);
        S->jp[l] = jp;
        S->jt[l] = jt;
        S->jt1[l] = jt1;
    }
    S->laytrop = laytrop;
}

/* ------------------------------------------------------------------------ */
/* taumol16..29 (sw:4043-6675)                                               */
/* ------------------------------------------------------------------------ */
typedef struct {
    float sc, fs, f[8];
    int js0;
} sw_spec;

/* species weights for scale 8 (troposphere) or 4 (stratosphere) */
static inline sw_spec sw_species(float primary, float ratio_secondary, const sw_col *S, int l, float scale)
{
    sw_spec s;
    s.sc = primary + ratio_secondary;
    float q = primary / s.sc;
    float sp = q > ONEMINUS ? ONEMINUS : q;
    float sm = scale * sp;
    int js = 1 + (int)sm;
    s.fs = sm - floorf(sm);
    float comp = 1.0f - s.fs;
    s.js0 = clampi(js - 1, 0, scale > 4.0f ? 7 : 3);
    s.f[0] = comp * S->fac00[l];  /* fac000 */
    s.f[1] = s.fs * S->fac00[l];  /* fac100 */
    s.f[2] = comp * S->fac10[l];  /* fac010 */
    s.f[3] = s.fs * S->fac10[l];  /* fac110 */
    s.f[4] = comp * S->fac01[l];  /* fac001 */
    s.f[5] = s.fs * S->fac01[l];  /* fac101 */
    s.f[6] = comp * S->fac11[l];  /* fac011 */
    s.f[7] = s.fs * S->fac11[l];  /* fac111 */
    return s;
}

/* 8-point interpolation in a (ns, 5, np) table stored as rows (jp*5+jt)*ns+js */
static inline float k8(const float *tab, int ngc, int ns, int js0, int jt0, int jt10, int jp0, int jp1, const float *f, int g)
{
#define R(js, jt, jp) tab[(((jp) * 5 + (jt)) * ns + (js)) * ngc + g]
    float s = f[0] * R(js0, jt0, jp0);
    s = s + f[1] * R(js0 + 1, jt0, jp0);
    s = s + f[2] * R(js0, jt0 + 1, jp0);
    s = s + f[3] * R(js0 + 1, jt0 + 1, jp0);
    s = s + f[4] * R(js0, jt10, jp1);
    s = s + f[5] * R(js0 + 1, jt10, jp1);
    s = s + f[6] * R(js0, jt10 + 1, jp1);
    s = s + f[7] * R(js0 + 1, jt10 + 1, jp1);
#undef R
    return s;
}

/* 4-point interpolation in a (5, np) table stored as rows jp*5+jt */
static inline float k4(const float *tab, int ngc, int jt0, int jt10, int jp0, int jp1,
                       float f00, float f10, float f01, float f11, int g)
{
    float s = f00 * tab[(jp0 * 5 + jt0) * ngc + g];
    s = s + f10 * tab[(jp0 * 5 + jt0 + 1) * ngc + g];
    s = s + f01 * tab[(jp1 * 5 + jt10) * ngc + g];
    s = s + f11 * tab[(jp1 * 5 + jt10 + 1) * ngc + g];
    return s;
}

static inline float self_interp(const ora_sw_band *B, const sw_col *S, int l, int g)
{
    int i0 = clampi(S->indself[l] - 1, 0, 8);
    int i1 = i0 + 1;
    return B->selfref[i0 * B->ngc + g] + S->selffrac[l] * (B->selfref[i1 * B->ngc + g] - B->selfref[i0 * B->ngc + g]);
}

static inline float for_interp(const ora_sw_band *B, const sw_col *S, int l, int g, int cap)
{
    int i0 = clampi(S->indfor[l] - 1, 0, cap);
    int i1 = jrow(i0 + 1, B->forref_rows);
    return B->forref[i0 * B->ngc + g] + S->forfrac[l] * (B->forref[i1 * B->ngc + g] - B->forref[i0 * B->ngc + g]);
}

static inline float sflux_interp(const ora_sw_band *B, int js0, float fs, int g)
{
    const float *t = B->sfluxref;
    int c = B->sflux_cols;
    return t[g * c + js0] + fs * (t[g * c + js0 + 1] - t[g * c + js0]);
}

/* solar-source layer rules */
static int trop_crossing_layer(const sw_col *S, int layreffr)
{
    const int n = S->nlay, laytrop = S->laytrop;
    for (int l = 0; l < n; ++l) {
        int next = l + 1 < n ? S->jp[l + 1] : S->jp[l];
        if (l < laytrop && S->jp[l] < layreffr && next >= layreffr) return (l + 1 < laytrop - 1) ? l + 1 : laytrop - 1;
    }
    return laytrop - 1;
}

static int strat_crossing_layer(const sw_col *S, int layreffr)
{
    const int n = S->nlay;
    for (int l = 1; l < n; ++l)
        if (l >= S->laytrop && S->jp[l - 1] < layreffr && S->jp[l] >= layreffr) return l;
    return n - 1;
}

static void sw_taumol(const ora_sw_cache *W, sw_col *S)
{
    const int n = S->nlay, laytrop = S->laytrop;
    sw_spec trop_spec[MAX_LAY], strat_spec[MAX_LAY];
    for (int b = 0; b < SW_NBND; ++b) {
        const ora_sw_band *B = &W->band[b];
        const int ngc = B->ngc, go = B->gofs;
        const int bn = b + 16;
        for (int l = 0; l < n; ++l) {
            const int trop = l < laytrop;
            const int jp = S->jp[l];
            const int jt0 = clampi(S->jt[l] - 1, 0, 3), jt10 = clampi(S->jt1[l] - 1, 0, 3);
            const int jp0 = clampi(jp - 1, 0, 11), jp1 = jp0 + 1;
            const int kjp0 = clampi(jp - 13, 0, 45), kjp1 = clampi(jp - 12, 0, 46);
            const float f00 = S->fac00[l], f10 = S->fac10[l], f01 = S->fac01[l], f11 = S->fac11[l];
            const float colh2o = S->colh2o[l], colmol = S->colmol[l];
            sw_spec sp8, sp4;
            int has_spec = 1;
            switch (bn) {
            case 16: sp8 = sw_species(colh2o, B->strrat1 * S->colch4[l], S, l, 8.0f); break;
            case 17: case 19: case 21:
                sp8 = sw_species(colh2o, B->strrat * S->colco2[l], S, l, 8.0f); break;
            case 18: sp8 = sw_species(colh2o, B->strrat * S->colch4[l], S, l, 8.0f); break;
            case 22: sp8 = sw_species(colh2o, (1.6f * B->strrat) * S->colo2[l], S, l, 8.0f); break;
            case 24: sp8 = sw_species(colh2o, B->strrat * S->colo2[l], S, l, 8.0f); break;
            case 28: sp8 = sw_species(S->colo3[l], B->strrat * S->colo2[l], S, l, 8.0f); break;
            default: has_spec = 0; memset(&sp8, 0, sizeof sp8); break;
            }
            if (bn == 17 || bn == 21) sp4 = sw_species(colh2o, B->strrat * S->colco2[l], S, l, 4.0f);
            else if (bn == 28) sp4 = sw_species(S->colo3[l], B->strrat * S->colo2[l], S, l, 4.0f);
            else memset(&sp4, 0, sizeof sp4);
            trop_spec[l] = sp8;
            strat_spec[l] = sp4;
            (void)has_spec;
            for (int g = 0; g < ngc; ++g) {
                float taug = 0.0f, taur;
                float cont;
                switch (bn) {
                case 16:
                    if (trop) {
                        float ta = k8(B->ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
                        cont = colh2o * (S->selffac[l] * self_interp(B, S, l, g) + S->forfac[l] * for_interp(B, S, l, g, 1));
                        taug = sp8.sc * ta + cont;
                    } else {
                        taug = S->colch4[l] * k4(B->kb, ngc, jt0, jt10, kjp0, kjp1, f00, f10, f01, f11, g);
                    }
                    taur = colmol * B->rayl;
                    break;
                case 17: case 21:
                    if (trop) {
                        float ta = k8(B->ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
                        cont = colh2o * (S->selffac[l] * self_interp(B, S, l, g) + S->forfac[l] * for_interp(B, S, l, g, 2));
                        taug = sp8.sc * ta + cont;
                    } else {
                        float sa = k8(B->kb, ngc, 5, sp4.js0, jt0, jt10, kjp0, kjp1, sp4.f, g);
                        cont = (colh2o * S->forfac[l]) * for_interp(B, S, l, g, 2);
                        taug = sp8.sc * sa + cont;
                    }
                    taur = colmol * B->rayl;
                    break;
                case 18: case 19:
                    if (trop) {
                        float ta = k8(B->ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
                        cont = colh2o * (S->selffac[l] * self_interp(B, S, l, g) + S->forfac[l] * for_interp(B, S, l, g, 2));
                        taug = sp8.sc * ta + cont;
                    } else {
                        float col = bn == 18 ? S->colch4[l] : S->colco2[l];
                        taug = col * k4(B->kb, ngc, jt0, jt10, kjp0, kjp1, f00, f10, f01, f11, g);
                    }
                    taur = colmol * B->rayl;
                    break;
                case 20:
                    if (trop) {
                        float ta = k4(B->ka, ngc, jt0, jt10, jp0, jp1, f00, f10, f01, f11, g);
                        float inner = (ta + S->selffac[l] * self_interp(B, S, l, g)) + S->forfac[l] * for_interp(B, S, l, g, 2);
                        taug = colh2o * inner + S->colch4[l] * B->absch4[g];
                    } else {
                        float sa = k4(B->kb, ngc, jt0, jt10, kjp0, kjp1, f00, f10, f01, f11, g);
                        float inner = sa + S->forfac[l] * for_interp(B, S, l, g, 2);
                        taug = colh2o * inner + S->colch4[l] * B->absch4[g];
                    }
                    taur = colmol * B->rayl;
                    break;
                case 22: {
                    float o2cont = (4.35e-4f * S->colo2[l]) / (350.0f * 2.0f);
                    if (trop) {
                        float ta = k8(B->ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
                        cont = colh2o * (S->selffac[l] * self_interp(B, S, l, g) + S->forfac[l] * for_interp(B, S, l, g, 2));
                        taug = (sp8.sc * ta + cont) + o2cont;
                    } else {
                        float sa = k4(B->kb, ngc, jt0, jt10, kjp0, kjp1, f00, f10, f01, f11, g);
                        taug = (S->colo2[l] * 1.6f) * sa + o2cont;
                    }
                    taur = colmol * B->rayl;
                    break;
                }
                case 23:
                    if (trop) {
                        float ta = k4(B->ka, ngc, jt0, jt10, jp0, jp1, f00, f10, f01, f11, g);
                        float sum = (B->givfac * ta + S->selffac[l] * self_interp(B, S, l, g)) + S->forfac[l] * for_interp(B, S, l, g, 1);
                        taug = colh2o * sum;
                    }
                    taur = colmol * B->rayl_g[g];
                    break;
                case 24:
                    if (trop) {
                        float ta = k8(B->ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
                        cont = colh2o * (S->selffac[l] * self_interp(B, S, l, g) + S->forfac[l] * for_interp(B, S, l, g, 1));
                        taug = (sp8.sc * ta + S->colo3[l] * B->abso3a[g]) + cont;
                        const float *ra = B->rayla;  /* (ngc, 9) */
                        float r = ra[g * 9 + sp8.js0] + sp8.fs * (ra[g * 9 + sp8.js0 + 1] - ra[g * 9 + sp8.js0]);
                        taur = colmol * r;
                    } else {
                        float sa = k4(B->kb, ngc, jt0, jt10, kjp0, kjp1, f00, f10, f01, f11, g);
                        taug = S->colo2[l] * sa + S->colo3[l] * B->abso3b[g];
                        taur = colmol * B->raylb[g];
                    }
                    break;
                case 25:
                    if (trop) {
                        float ta = k4(B->ka, ngc, jt0, jt10, jp0, jp1, f00, f10, f01, f11, g);
                        taug = colh2o * ta + S->colo3[l] * B->abso3a[g];
                    } else {
                        taug = S->colo3[l] * B->abso3b[g];
                    }
                    taur = colmol * B->rayl_g[g];
                    break;
                case 26:
                    taug = 0.0f;
                    taur = colmol * B->rayl_g[g];
                    break;
                case 27: {
                    float a = trop ? k4(B->ka, ngc, jt0, jt10, jp0, jp1, f00, f10, f01, f11, g)
                                   : k4(B->kb, ngc, jt0, jt10, kjp0, kjp1, f00, f10, f01, f11, g);
                    taug = S->colo3[l] * a;
                    taur = colmol * B->rayl_g[g];
                    break;
                }
                case 28:
                    if (trop) taug = sp8.sc * k8(B->ka, ngc, 9, sp8.js0, jt0, jt10, jp0, jp1, sp8.f, g);
                    else taug = sp8.sc * k8(B->kb, ngc, 5, sp4.js0, jt0, jt10, kjp0, kjp1, sp4.f, g);
                    taur = colmol * B->rayl;
                    break;
                default: /* 29 */
                    if (trop) {
                        float ta = k4(B->ka, ngc, jt0, jt10, jp0, jp1, f00, f10, f01, f11, g);
                        float wat = (ta + S->selffac[l] * self_interp(B, S, l, g)) + S->forfac[l] * for_interp(B, S, l, g, 2);
                        taug = colh2o * wat + S->colco2[l] * B->absco2[g];
                    } else {
                        float sa = k4(B->kb, ngc, jt0, jt10, kjp0, kjp1, f00, f10, f01, f11, g);
                        taug = S->colco2[l] * sa + colh2o * B->absh2o[g];
                    }
                    taur = colmol * B->rayl;
                    break;
                }
                S->taug[l][go + g] = taug;
                S->taur[l][go + g] = taur;
            }
        }
        /* solar source function for the band */
        for (int g = 0; g < ngc; ++g) {
            float sz = 0.0f;
            switch (bn) {
            case 16: case 29:
                sz = laytrop < n ? B->sfluxref[g] : 0.0f;
                break;
            case 17: case 28:
                if (laytrop < n) {
                    int ls = strat_crossing_layer(S, B->layreffr);
                    sz = sflux_interp(B, strat_spec[ls].js0, strat_spec[ls].fs, g);
                }
                break;
            case 18: case 19: case 21: case 22: case 24:
                if (laytrop > 0) {
                    int ls = trop_crossing_layer(S, B->layreffr);
                    sz = sflux_interp(B, trop_spec[ls].js0, trop_spec[ls].fs, g);
                }
                break;
            case 20: case 23: case 25: case 26:
                sz = laytrop > 0 ? B->sfluxref[g] : 0.0f;
                break;
            case 27:
                sz = laytrop < n ? B->scalekur * B->sfluxref[g] : 0.0f;
                break;
            }
            S->sfluxzen[go + g] = sz;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* spcvmc (sw:6788-7094), reftra (sw:3490-3601), vrtqdr (sw:3604-3720)        */
/* ------------------------------------------------------------------------ */
static inline float exp_lookup(const ora_sw_cache *W, float v)
{
    if (v <= 0.06f) return (1.0f - v) + (0.5f * v) * v;
    float tblind = v / (W->bpade + v);
    int it = clampi((int)((float)W->ntbl * tblind + 0.5f), 0, W->ntbl);
    return W->pade_exp[it];
}

typedef struct { float ref, refd, tra, trad; } rt4;

/* FP64 mode (test of the GPU's binary64 variant): the Pade lookup of
 * exp(-v) with binary64 arithmetic; the table is the same binary32 data. */
static double exp_lookup64(const ora_sw_cache *W, double v)
{
    if (v <= 0.06) return (1.0 - v) + (0.5 * v) * v;
    double tblind = v / ((double)W->bpade + v);
    int it = clampi((int)((double)W->ntbl * tblind + 0.5), 0, W->ntbl);
    return (double)W->pade_exp[it];
}

/* FP64 mode's reftra (sw:3490-3601) for a layer whose delta-scaled
 * single-scattering albedo zwo is >= 0.999 or whose optical depth is below
 * 0.1: every operation of both branches in binary64 on the binary32 inputs,
 * the four results rounded once. */
static rt4 reftra64(const ora_sw_cache *W, float zg_in, float mu_in, float zto1_in, float zw_in)
{
    const double zg = (double)zg_in, mu = (double)mu_in, zto1 = (double)zto1_in, zw = (double)zw_in;
    const double eps = 1.0e-8, zwcrit = 0.9999995;
    double ref, refd, tra, trad;
    double zg3 = 3.0 * zg;
    double g1 = (8.0 - zw * (5.0 + zg3)) * 0.25;
    double g2 = 3.0 * (zw * (1.0 - zg)) * 0.25;
    double g3 = (2.0 - zg3 * mu) * 0.25;
    double g4 = 1.0 - g3;
    double sr = zg != 1.0 ? zg / (1.0 - zg) : 0.0;
    double denom = zg != 1.0 ? 1.0 - (1.0 - zw) * sr * sr : 1.0;
    double zwo = (zw > 0.0 && denom != 0.0) ? zw / denom : 0.0;
    double ze2 = zto1 / mu;
    if (ze2 > 500.0) ze2 = 500.0;
    double zem2 = exp_lookup64(W, ze2);
    if (zwo >= zwcrit) {
        double za = g1 * mu;
        double za1 = za - g3;
        double zgt = g1 * zto1;
        ref = (zgt - za1 * (1.0 - zem2)) / (1.0 + zgt);
        tra = 1.0 - ref;
        refd = zgt / (1.0 + zgt);
        trad = 1.0 - refd;
        if (zem2 == 1.0) { ref = 0.0; tra = 1.0; refd = 0.0; trad = 1.0; }
    } else {
        double za1 = g1 * g4 + g2 * g3;
        double za2 = g1 * g3 + g2 * g4;
        double rad = g1 * g1 - g2 * g2;
        double zrk = sqrt(rad > 0.0 ? rad : 0.0);
        double zrp = zrk * mu;
        double zrp1 = 1.0 + zrp, zrm1 = 1.0 - zrp, zrk2 = 2.0 * zrk;
        double zrpp = 1.0 - zrp * zrp;
        double zrkg = zrk + g1;
        double zr1 = zrm1 * (za2 + zrk * g3);
        double zr2 = zrp1 * (za2 - zrk * g3);
        double zr3 = zrk2 * (g3 - za2 * mu);
        double zr4 = zrpp * zrkg;
        double zr5 = zrpp * (zrk - g1);
        double zt1 = zrp1 * (za1 + zrk * g4);
        double zt2 = zrm1 * (za1 - zrk * g4);
        double zt3 = zrk2 * (g4 + za1 * mu);
        double zbeta = (g1 - zrk) / zrkg;
        double ze1 = zrk * zto1;
        if (ze1 > 500.0) ze1 = 500.0;
        double zem1 = exp_lookup64(W, ze1);
        double zep1 = 1.0 / zem1;
        double zep2 = 1.0 / zem2;
        double zdenr = zr4 * zep1 + zr5 * zem1;
        double zdent = zr4 * zep1 + zr5 * zem1;
        if (zdenr >= -eps && zdenr <= eps) {
            ref = eps;
            tra = zem2;
        } else {
            ref = zw * (zr1 * zep1 - zr2 * zem1 - zr3 * zem2) / zdenr;
            tra = zem2 - zem2 * zw * (zt1 * zep1 - zt2 * zem1 - zt3 * zep2) / zdent;
        }
        double zemm = zem1 * zem1;
        double zdend = 1.0 / ((1.0 - zbeta * zemm) * zrkg);
        refd = g2 * (1.0 - zemm) * zdend;
        trad = zrk2 * zem1 * zdend;
    }
    rt4 r = {(float)ref, (float)refd, (float)tra, (float)trad};
    return r;
}

static rt4 reftra(const ora_sw_cache *W, int fp64, int lrt, float zg, float mu, float zto1, float zw)
{
    rt4 r = {0.0f, 0.0f, 1.0f, 1.0f};
    if (!lrt) return r;
    const float eps = 1.0e-8f, zwcrit = 0.9999995f;
    float zg3 = 3.0f * zg;
    float g1 = (8.0f - zw * (5.0f + zg3)) * 0.25f;
    float g2 = 3.0f * (zw * (1.0f - zg)) * 0.25f;
    float g3 = (2.0f - zg3 * mu) * 0.25f;
    float g4 = 1.0f - g3;
    float sr = zg != 1.0f ? zg / (1.0f - zg) : 0.0f;
    float denom = zg != 1.0f ? 1.0f - (1.0f - zw) * sr * sr : 1.0f;
    float zwo = (zw > 0.0f && denom != 0.0f) ? zw / denom : 0.0f;
    if (fp64 && (zwo >= 0.999f || zto1 < 0.1f)) return reftra64(W, zg, mu, zto1, zw);
    if (zwo >= zwcrit) {
        float za = g1 * mu;
        float za1 = za - g3;
        float zgt = g1 * zto1;
        float ze = zto1 / mu;
        if (ze > 500.0f) ze = 500.0f;
        float ex = exp_lookup(W, ze);
        r.ref = (zgt - za1 * (1.0f - ex)) / (1.0f + zgt);
        r.tra = 1.0f - r.ref;
        r.refd = zgt / (1.0f + zgt);
        r.trad = 1.0f - r.refd;
        if (ex == 1.0f) { r.ref = 0.0f; r.tra = 1.0f; r.refd = 0.0f; r.trad = 1.0f; }
        return r;
    }
    float za1 = g1 * g4 + g2 * g3;
    float za2 = g1 * g3 + g2 * g4;
    float rad = g1 * g1 - g2 * g2;
    float zrk = sqrtf(rad > 0.0f ? rad : 0.0f);
    float zrp = zrk * mu;
    float zrp1 = 1.0f + zrp, zrm1 = 1.0f - zrp, zrk2 = 2.0f * zrk;
    float zrpp = 1.0f - zrp * zrp;
    float zrkg = zrk + g1;
    float zr1 = zrm1 * (za2 + zrk * g3);
    float zr2 = zrp1 * (za2 - zrk * g3);
    float zr3 = zrk2 * (g3 - za2 * mu);
    float zr4 = zrpp * zrkg;
    float zr5 = zrpp * (zrk - g1);
    float zt1 = zrp1 * (za1 + zrk * g4);
    float zt2 = zrm1 * (za1 - zrk * g4);
    float zt3 = zrk2 * (g4 + za1 * mu);
    float zt4 = zr4, zt5 = zr5;
    float zbeta = (g1 - zrk) / zrkg;
    float ze1 = zrk * zto1;
    if (ze1 > 500.0f) ze1 = 500.0f;
    float ze2 = zto1 / mu;
    if (ze2 > 500.0f) ze2 = 500.0f;
    float zem1 = exp_lookup(W, ze1);
    float zep1 = 1.0f / zem1;
    float zem2 = exp_lookup(W, ze2);
    float zep2 = 1.0f / zem2;
    float zdenr = zr4 * zep1 + zr5 * zem1;
    float zdent = zt4 * zep1 + zt5 * zem1;
    int small = (zdenr >= -eps) && (zdenr <= eps);
    if (small) {
        r.ref = eps;
        r.tra = zem2;
    } else {
        r.ref = zw * (zr1 * zep1 - zr2 * zem1 - zr3 * zem2) / zdenr;
        r.tra = zem2 - zem2 * zw * (zt1 * zep1 - zt2 * zem1 - zt3 * zep2) / zdent;
    }
    float zemm = zem1 * zem1;
    float zdend = 1.0f / ((1.0f - zbeta * zemm) * zrkg);
    r.refd = g2 * (1.0f - zemm) * zdend;
    r.trad = zrk2 * zem1 * zdend;
    return r;
}

/* vrtqdr for one g-point; arrays indexed top-down 0..n (n = surface) */
static void vrtqdr(int n, const float *pref, const float *prefd, const float *ptra, const float *ptrad,
                   const float *pdbt, const float *ptdbt, float *pfd, float *pfu)
{
    float prup[MAX_LAY + 1], prupd[MAX_LAY + 1], ztdn[MAX_LAY + 1], prdnd[MAX_LAY + 1];
    prup[n] = pref[n];
    prupd[n] = prefd[n];
    for (int i = n - 1; i >= 0; --i) {
        float zreflect = 1.0f / (1.0f - prupd[i + 1] * prefd[i]);
        prup[i] = pref[i] + ptrad[i] * ((ptra[i] - pdbt[i]) * prupd[i + 1] + pdbt[i] * prup[i + 1]) * zreflect;
        prupd[i] = prefd[i] + ptrad[i] * ptrad[i] * prupd[i + 1] * zreflect;
    }
    ztdn[0] = 1.0f;
    prdnd[0] = 0.0f;
    ztdn[1] = ptra[0];
    prdnd[1] = prefd[0];
    for (int i = 1; i < n; ++i) {
        float zreflect = 1.0f / (1.0f - prefd[i] * prdnd[i]);
        ztdn[i + 1] = ptdbt[i] * ptra[i] + ptrad[i] * ((ztdn[i] - ptdbt[i]) + ptdbt[i] * pref[i] * prdnd[i]) * zreflect;
        prdnd[i + 1] = prefd[i] + ptrad[i] * ptrad[i] * prdnd[i] * zreflect;
    }
    for (int k = 0; k <= n; ++k) {
        float zreflect = 1.0f / (1.0f - prdnd[k] * prupd[k]);
        pfu[k] = (ptdbt[k] * prup[k] + (ztdn[k] - ptdbt[k]) * prupd[k]) * zreflect;
        pfd[k] = ptdbt[k] + (ztdn[k] - ptdbt[k] + ptdbt[k] * prup[k] * prdnd[k]) * zreflect;
    }
}

/* Direct (albp) and diffuse (albd) surface albedo of a band (0-based): the
 * Noah-MP fields for columns with xland < 1.5 when all four are given
 * (sw:2519-2530), visible in bands 25-28 and near infrared in bands 16-24 and
 * 29 (sw:2120-2127); `albedo` otherwise. */
static void sw_band_albedo(const ora_in *in, int col, int band, float *albp, float *albd)
{
    *albp = in->albedo[col];
    *albd = in->albedo[col];
    if (in->alswvisdir && in->alswvisdif && in->alswnirdir && in->alswnirdif && in->xland[col] < 1.5f) {
        const int vis = band >= 9 && band <= 12;
        *albp = vis ? in->alswvisdir[col] : in->alswnirdir[col];
        *albd = vis ? in->alswvisdif[col] : in->alswnirdif[col];
    }
}

static void sw_spcvmc(const ora_sw_cache *W, const ora_in *in, int col, sw_col *S, int clear_only)
{
    const int n = S->nlay;
    const float mu = fmaxf(in->coszr[col], 1.0e-10f);
    const float repclc = 1.0e-12f;
    /* accumulators, top-down levels */
    float sfu[MAX_LAY + 1], sfd[MAX_LAY + 1], scu[MAX_LAY + 1], scd[MAX_LAY + 1], sfdir[MAX_LAY + 1], scdir[MAX_LAY + 1];
    for (int k = 0; k <= n; ++k) { sfu[k] = 0; sfd[k] = 0; scu[k] = 0; scd[k] = 0; sfdir[k] = 0; scdir[k] = 0; }
    for (int g = 0; g < SW_NGPT; ++g) {
        int band = 0;
        while (g >= W->band[band].gofs + W->band[band].ngc) ++band;
        float albp, albd;
        sw_band_albedo(in, col, band, &albp, &albd);
        float zrefc[MAX_LAY + 1], zrefdc[MAX_LAY + 1], ztrac[MAX_LAY + 1], ztradc[MAX_LAY + 1];
        float zref[MAX_LAY + 1], zrefd[MAX_LAY + 1], ztra[MAX_LAY + 1], ztrad[MAX_LAY + 1];
        float zdbtc[MAX_LAY + 1], zdbt[MAX_LAY + 1], ztdbtc[MAX_LAY + 1], ztdbt[MAX_LAY + 1];
        float ztdbtc_nd[MAX_LAY + 1], ztdbt_nd[MAX_LAY + 1];
        ztdbtc[0] = 1.0f; ztdbt[0] = 1.0f; ztdbtc_nd[0] = 1.0f; ztdbt_nd[0] = 1.0f;
        for (int r = 0; r < n; ++r) {
            const int l = n - 1 - r;              /* reversed: r = 0 is the top layer */
            const float cloud = (float)S->cldf[g][l];
            const float clear = 1.0f - cloud;
            const float taur = S->taur[l][g], taug = S->taug[l][g];
            float ztau = (taur + taug) + 0.0f;
            float zom = taur + 0.0f * 1.0f;
            float zgr = 0.0f * 1.0f * 0.0f / zom;
            zom = zom / ztau;
            float dbtc_nd = exp_lookup(W, ztau / mu);
            ztdbtc_nd[r + 1] = ztdbtc_nd[r] * dbtc_nd;
            if (!clear_only) {
                float tauorig = ztau + S->taormc[g][l];
                float dbtmo_nd = exp_lookup(W, tauorig / mu);
                float dbt_nd = clear * dbtc_nd + cloud * dbtmo_nd;
                ztdbt_nd[r + 1] = ztdbt_nd[r] * dbt_nd;
            }
            float zf = zgr * zgr;
            float zwf = zom * zf;
            float ztauc = (1.0f - zwf) * ztau;
            float zomcc = (zom - zwf) / (1.0f - zwf);
            float zgcc = (zgr - zf) / (1.0f - zf);
            rt4 c = reftra(W, S->fp64_reftra, 1, zgcc, mu, ztauc, zomcc);
            zrefc[r] = c.ref; zrefdc[r] = c.refd; ztrac[r] = c.tra; ztradc[r] = c.trad;
            float dbtc = exp_lookup(W, ztauc / mu);
            zdbtc[r] = dbtc;
            ztdbtc[r + 1] = ztdbtc[r] * dbtc;
            if (!clear_only) {
                const float tc = S->taucmc[g][l], wc = S->ssacmc[g][l], gc = S->asmcmc[g][l];
                float ztauo = ztauc + tc;
                float zomco = ztauc * zomcc + tc * wc;
                float zgco = (tc * wc * gc + ztauc * zomcc * zgcc) / zomco;
                zomco = zomco / ztauo;
                rt4 o = reftra(W, S->fp64_reftra, cloud > repclc, zgco, mu, ztauo, zomco);
                zref[r] = clear * c.ref + cloud * o.ref;
                zrefd[r] = clear * c.refd + cloud * o.refd;
                ztra[r] = clear * c.tra + cloud * o.tra;
                ztrad[r] = clear * c.trad + cloud * o.trad;
                float dbtmo = exp_lookup(W, ztauo / mu);
                float dbt = clear * dbtc + cloud * dbtmo;
                zdbt[r] = dbt;
                ztdbt[r + 1] = ztdbt[r] * dbt;
            }
        }
        zrefc[n] = albp; zrefdc[n] = albd; ztrac[n] = 0.0f; ztradc[n] = 0.0f; zdbtc[n] = 0.0f;
        float pfd_c[MAX_LAY + 1], pfu_c[MAX_LAY + 1], pfd_t[MAX_LAY + 1], pfu_t[MAX_LAY + 1];
        vrtqdr(n, zrefc, zrefdc, ztrac, ztradc, zdbtc, ztdbtc, pfd_c, pfu_c);
        const float *pfd_tot = pfd_c, *pfu_tot = pfu_c, *tdbt_nd = ztdbtc_nd;
        if (!clear_only) {
            zref[n] = albp; zrefd[n] = albd; ztra[n] = 0.0f; ztrad[n] = 0.0f; zdbt[n] = 0.0f;
            vrtqdr(n, zref, zrefd, ztra, ztrad, zdbt, ztdbt, pfd_t, pfu_t);
            pfd_tot = pfd_t;
            pfu_tot = pfu_t;
            tdbt_nd = ztdbt_nd;
        }
        float zincflx = ((S->adjflux * S->sfluxzen[g]) * mu) * 1.0f;
        for (int k = 0; k <= n; ++k) {
            sfu[k] = sfu[k] + pfu_tot[k] * zincflx;
            sfd[k] = sfd[k] + pfd_tot[k] * zincflx;
            scu[k] = scu[k] + pfu_c[k] * zincflx;
            scd[k] = scd[k] + pfd_c[k] * zincflx;
            sfdir[k] = sfdir[k] + tdbt_nd[k] * zincflx;
            scdir[k] = scdir[k] + ztdbtc_nd[k] * zincflx;
        }
    }
    for (int k = 0; k <= n; ++k) {
        S->bbfu[k] = sfu[n - k]; S->bbfd[k] = sfd[n - k];
        S->bbcu[k] = scu[n - k]; S->bbcd[k] = scd[n - k];
        S->bbfddir[k] = sfdir[n - k]; S->bbcddir[k] = scdir[n - k];
    }
    /* heating rates (sw:2285-2301) */
    const float heatfac = (9.8066f * 8.6400e4f) / (1004.5f * 1.0e2f);
    for (int l = 0; l < n; ++l) {
        float zdpgcp = heatfac / S->pdp[l];
        float n1 = S->bbfd[l + 1] - S->bbfu[l + 1], n0 = S->bbfd[l] - S->bbfu[l];
        float c1 = S->bbcd[l + 1] - S->bbcu[l + 1], c0 = S->bbcd[l] - S->bbcu[l];
        S->swhr[l] = (n1 - n0) * zdpgcp;
        S->swhrc[l] = (c1 - c0) * zdpgcp;
        if (l >= S->fp64_from) {
            /* FP64 mode: net fluxes, their difference and dF/dp in binary64 */
            S->swhr[l] = ora_heating64(heatfac, S->bbfu[l], S->bbfd[l], S->bbfu[l + 1], S->bbfd[l + 1],
                                       S->plev[l], S->plev[l + 1]);
            S->swhrc[l] = ora_heating64(heatfac, S->bbcu[l], S->bbcd[l], S->bbcu[l + 1], S->bbcd[l + 1],
                                        S->plev[l], S->plev[l + 1]);
        }
    }
    S->swhr[n - 1] = 0.0f;
    S->swhrc[n - 1] = 0.0f;
}

/* ------------------------------------------------------------------------ */
typedef struct { const ora_cache *C; const ora_in *in; ora_out *out; } sw_job;

static int sw_one_column(void *ctx, int col)
{
    sw_job *J = (sw_job *)ctx;
    const ora_in *in = J->in;
    ora_out *out = J->out;
    const int nk = in->nk, nlay = nk + 1;
    const float coszen = in->coszr[col];
    float *r3[2] = {out->rthraten + (size_t)col * nk, out->rthratenc + (size_t)col * nk};
    if (!(coszen > 0.0f)) {
        /* night: every output is masked to zero (sw:2667-2671) */
        for (int k = 0; k < nk; ++k) { r3[0][k] = 0.0f; r3[1][k] = 0.0f; }
        out->up_top[col] = out->upc_top[col] = out->dn_top[col] = out->dnc_top[col] = 0.0f;
        out->up_sfc[col] = out->upc_sfc[col] = out->dn_sfc[col] = out->dnc_sfc[col] = 0.0f;
        out->swddir[col] = out->swddni[col] = out->swddif[col] = out->swddirc[col] = out->swddnic[col] = 0.0f;
        return 0;
    }
    sw_col *S = (sw_col *)malloc(sizeof(sw_col));
    if (!S) return 1;
    const int icld = in->icloud == 0 ? 0 : in->cldovrlp;
    sw_prepare(J->C, in, col, S);
    sw_inatm(in, S);
    if (sw_clouds(J->C, in, col, S, icld) != 0) { free(S); return 2; }
    sw_setcoef(&J->C->sw, S);
    sw_taumol(&J->C->sw, S);
    sw_spcvmc(&J->C->sw, in, col, S, icld == 0);
    const float *pi3d = in->pi3d + (size_t)col * nk;
    for (int k = 0; k < nk; ++k) {
        r3[0][k] = (S->swhr[k] / 86400.0f) / pi3d[k];
        r3[1][k] = (S->swhrc[k] / 86400.0f) / pi3d[k];
    }
    out->up_top[col] = S->bbfu[nlay];
    out->upc_top[col] = S->bbcu[nlay];
    out->dn_top[col] = S->bbfd[nlay];
    out->dnc_top[col] = S->bbcd[nlay];
    out->up_sfc[col] = S->bbfu[0];
    out->upc_sfc[col] = S->bbcu[0];
    out->dn_sfc[col] = S->bbfd[0];
    out->dnc_sfc[col] = S->bbcd[0];
    out->swddir[col] = S->bbfddir[0];
    out->swddni[col] = S->bbfddir[0] / coszen;
    out->swddif[col] = S->bbfd[0] - S->bbfddir[0];
    out->swddirc[col] = S->bbcddir[0];
    out->swddnic[col] = S->bbcddir[0] / coszen;
    if (out->taug)
        for (int l = 0; l < nlay; ++l)
            for (int g = 0; g < SW_NGPT; ++g) {
                out->taug[((size_t)col * nlay + l) * SW_NGPT + g] = S->taug[l][g];
                out->fracs_or_taur[((size_t)col * nlay + l) * SW_NGPT + g] = S->taur[l][g];
            }
    if (out->cldfmc)
        for (int g = 0; g < SW_NGPT; ++g)
            for (int l = 0; l < nlay; ++l) {
                out->cldfmc[((size_t)col * SW_NGPT + g) * nlay + l] = (float)S->cldf[g][l];
                out->taucmc[((size_t)col * SW_NGPT + g) * nlay + l] = S->taucmc[g][l];
            }
    if (out->uflx)
        for (int lev = 0; lev <= nlay; ++lev) {
            out->uflx[(size_t)col * (nlay + 1) + lev] = S->bbfu[lev];
            out->dflx[(size_t)col * (nlay + 1) + lev] = S->bbfd[lev];
            out->uflxc[(size_t)col * (nlay + 1) + lev] = S->bbcu[lev];
            out->dflxc[(size_t)col * (nlay + 1) + lev] = S->bbcd[lev];
        }
    if (out->hr)
        for (int l = 0; l < nlay; ++l) {
            out->hr[(size_t)col * nlay + l] = S->swhr[l];
            out->hrc[(size_t)col * nlay + l] = S->swhrc[l];
        }
    free(S);
    return 0;
}

int ora_sw_columns(const ora_tables *t, const ora_in *in, ora_out *out, int nthreads)
{
    if (in->nk < 4 || in->nk + 1 > MAX_LAY) return -1;
    sw_job J = {ora_cache_of(t), in, out};
    return ora_parallel_for(in->ncol, nthreads, sw_one_column, &J);
}

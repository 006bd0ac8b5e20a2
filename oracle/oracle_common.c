/*
 * Oracle: pieces shared by the LW and SW restatements (test infrastructure).
 * Reference file: src/wrf_jax/physics/module_ra_rrtmg_common.py ("common").
 */
#include "oracle_internal.h"

#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* table blob (format written by wrf-jax_b200/tables.py)                    */
/* ------------------------------------------------------------------------ */
typedef struct {
    char name[48];
    uint32_t dtype, ndim, shape[4];
    uint64_t offset, nbytes;
    uint64_t words;   /* nbytes / 4 as stored in the blob */
} blob_entry;

struct ora_tables {
    unsigned char *raw;
    size_t size;
    uint32_t count;
    blob_entry *entries;
    ora_cache cache;
};

const void *ora_table(const ora_tables *t, const char *name, int *n_out)
{
    for (uint32_t i = 0; i < t->count; ++i) {
        if (strncmp(t->entries[i].name, name, 48) == 0) {
            if (n_out) *n_out = (int)t->entries[i].words;
            return t->raw + t->entries[i].offset;
        }
    }
    if (n_out) *n_out = 0;
    return NULL;
}

const ora_cache *ora_cache_of(const ora_tables *t) { return &t->cache; }

#ifdef ORA_WIDE_TABLES
/* Binary64 build: `float` is the 8-byte binary64 type, so every binary32
 * entry (dtype 0) is copied once into an array of it (exact); other entries
 * are copied as they are.  Entries start on 8-byte boundaries. */
static int widen_tables(ora_tables *t)
{
    size_t total = 0;
    for (uint32_t i = 0; i < t->count; ++i) {
        const blob_entry *e = &t->entries[i];
        const size_t bytes = e->dtype == 0 ? (size_t)e->words * sizeof(float) : (size_t)e->nbytes;
        total += (bytes + 7) / 8 * 8;
    }
    unsigned char *wide = (unsigned char *)calloc(total ? total : 1, 1);
    if (!wide) return -1;
    size_t pos = 0;
    for (uint32_t i = 0; i < t->count; ++i) {
        blob_entry *e = &t->entries[i];
        const unsigned char *src = t->raw + e->offset;
        size_t bytes;
        if (e->dtype == 0) {
            float *dst = (float *)(wide + pos);
            for (uint64_t k = 0; k < e->words; ++k) {
                ora_binary32 v;
                memcpy(&v, src + 4 * k, 4);
                dst[k] = v;
            }
            bytes = (size_t)e->words * sizeof(float);
        } else {
            memcpy(wide + pos, src, (size_t)e->nbytes);
            bytes = (size_t)e->nbytes;
        }
        e->offset = pos;
        e->nbytes = bytes;
        pos += (bytes + 7) / 8 * 8;
    }
    free(t->raw);
    t->raw = wide;
    t->size = total;
    return 0;
}
#endif

ora_tables *ora_tables_load(const char *path)
{
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    ora_tables *t = (ora_tables *)calloc(1, sizeof(*t));
    t->raw = (unsigned char *)malloc((size_t)size);
    t->size = (size_t)size;
    if (fread(t->raw, 1, (size_t)size, f) != (size_t)size || memcmp(t->raw, "RRTMGB2\0", 8) != 0) {
        fclose(f);
        ora_tables_free(t);
        return NULL;
    }
    fclose(f);
    uint32_t version;
    memcpy(&version, t->raw + 8, 4);
    memcpy(&t->count, t->raw + 12, 4);
    t->entries = (blob_entry *)calloc(t->count, sizeof(blob_entry));
    const unsigned char *p = t->raw + 16;
    for (uint32_t i = 0; i < t->count; ++i, p += 88) {
        memcpy(t->entries[i].name, p, 48);
        memcpy(&t->entries[i].dtype, p + 48, 4);
        memcpy(&t->entries[i].ndim, p + 52, 4);
        memcpy(t->entries[i].shape, p + 56, 16);
        memcpy(&t->entries[i].offset, p + 72, 8);
        memcpy(&t->entries[i].nbytes, p + 80, 8);
        t->entries[i].words = t->entries[i].nbytes / 4;
        if (t->entries[i].offset > t->size || t->entries[i].nbytes > t->size - t->entries[i].offset) {
            ora_tables_free(t);
            return NULL;
        }
    }
#ifdef ORA_WIDE_TABLES
    if (widen_tables(t) != 0) {
        ora_tables_free(t);
        return NULL;
    }
#endif
    if (ora_cache_init(t, &t->cache) != 0) {
        ora_tables_free(t);
        return NULL;
    }
    return t;
}

void ora_tables_free(ora_tables *t)
{
    if (!t) return;
    free(t->entries);
    free(t->raw);
    free(t);
}

/* ------------------------------------------------------------------------ */
/* ozone climatology work profile (common:343-355)                          */
/* ------------------------------------------------------------------------ */
static void o3_work_profile(const ora_tables *t, float o3wrk[31], float ppwrkh[32])
{
    const float *o3sum = (const float *)ora_table(t, "o3sum", NULL);
    const float *ppsum = (const float *)ora_table(t, "ppsum", NULL);
    const float *o3win = (const float *)ora_table(t, "o3win", NULL);
    const float *ppwin = (const float *)ora_table(t, "ppwin", NULL);
    o3wrk[0] = 0.5f * (o3sum[0] + o3win[0]);
    for (int i = 0; i < 30; ++i) {
        float slope = (o3win[i + 1] - o3win[i]) / (ppwin[i + 1] - ppwin[i]);
        float interp = o3win[i] + slope * (ppsum[i + 1] - ppwin[i]);
        o3wrk[i + 1] = 0.5f * (interp + o3sum[i + 1]);
    }
    /* ppwrkh (common:366-372) */
    ppwrkh[0] = 1100.0f;
    for (int i = 0; i < 30; ++i) ppwrkh[i + 1] = 0.5f * (ppsum[i + 1] + ppsum[i]);
    ppwrkh[31] = 0.0f;
}

int ora_cache_init(const ora_tables *t, ora_cache *c)
{
    memset(c, 0, sizeof(*c));
    o3_work_profile(t, c->o3wrk, c->ppwrkh);
    c->retab = (const float *)ora_table(t, "retab", NULL);
    c->pprof = (const float *)ora_table(t, "lw_buffer_pprof", &c->nprof);
    c->tprof = (const float *)ora_table(t, "lw_buffer_tprof", NULL);
    if (!c->retab || !c->pprof || !c->tprof) return -1;
    return ora_lw_cache_init(t, &c->lw) | ora_sw_cache_init(t, &c->sw);
}

/* o3data/inirad (common:357-410): pressure-weighted climatological ozone for
 * layers 0..nout-1 bounded by plev[0..nout] (hPa, decreasing). */
void ora_o3data(const ora_cache *c, const float *plev, int nout, float *o3)
{
    for (int l = 0; l < nout; ++l) {
        float pa = plev[l], pb = plev[l + 1];
        float total = 0.0f;
        for (int b = 0; b < 31; ++b) {
            float pb1 = fmaxf(pa - c->ppwrkh[b], 0.0f);
            float pb2 = fmaxf(pa - c->ppwrkh[b + 1], 0.0f);
            float pt1 = fmaxf(pb - c->ppwrkh[b], 0.0f);
            float pt2 = fmaxf(pb - c->ppwrkh[b + 1], 0.0f);
            float overlap = ((pb2 - pb1) - pt2) + pt1;
            total = total + overlap * c->o3wrk[b];
        }
        o3[l] = total / (pa - pb);
    }
}

/* ------------------------------------------------------------------------ */
/* KISS generator (common:964-1005)                                          */
/* ------------------------------------------------------------------------ */
void ora_kiss_step(uint32_t s[4], ora_binary32 *ran)
{
    s[0] = 69069u * s[0] + 1327217885u;
    uint32_t x = s[1];
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    s[1] = x;
    s[2] = 18000u * (s[2] & 65535u) + (s[2] >> 16);
    s[3] = 30903u * (s[3] & 65535u) + (s[3] >> 16);
    uint32_t kiss = s[0] + s[1] + (s[2] << 16) + s[3];
    ora_binary32 k = (ora_binary32)(int32_t)kiss;
    *ran = k * 2.328306e-10f + 0.5f;
}

void ora_kiss_seeds(const ora_binary32 *pmid4, uint32_t s[4])
{
    for (int i = 0; i < 4; ++i) {
        ora_binary32 frac = pmid4[i] - truncf(pmid4[i]);
        s[i] = (uint32_t)(int32_t)(frac * 1000000000.0f);
    }
}

/* McICA maximum-random overlap (common:1092-1153) for one column.
 * cld: (nlay) cloud fraction.  cloudy: (nsub, nlay) output 0/1. */
void ora_mcica_overlap2(const float *play, const float *cld_in, int nlay, int nsub,
                        int change_seed, unsigned char *cloudy, ora_binary32 *cdf_work)
{
    /* binary32 in every build: the layer pressures and cloud fractions are
     * binary32 values (rounded to it in the binary64 build) */
    ora_binary32 pmid[4];
    for (int i = 0; i < 4; ++i) pmid[i] = (ora_binary32)play[i] * 100.0f;
    uint32_t s[4];
    ora_kiss_seeds(pmid, s);
    ora_binary32 r;
    for (int i = 0; i < change_seed; ++i) ora_kiss_step(s, &r);
    for (int d = 0; d < nsub * nlay; ++d) {
        ora_kiss_step(s, &r);
        cdf_work[d] = r;          /* index = sub * nlay + lay */
    }
    for (int sub = 0; sub < nsub; ++sub) {
        ora_binary32 *cdf = cdf_work + (size_t)sub * nlay;
        for (int l = 1; l < nlay; ++l) {
            const ora_binary32 cl = (ora_binary32)cld_in[l - 1];
            ora_binary32 cprev = cl < 1.0e-20f ? 0.0f : cl;
            ora_binary32 thr = 1.0f - cprev;
            cdf[l] = (cdf[l - 1] > thr) ? cdf[l - 1] : cdf[l] * thr;
        }
        for (int l = 0; l < nlay; ++l) {
            const ora_binary32 cl = (ora_binary32)cld_in[l];
            ora_binary32 c = cl < 1.0e-20f ? 0.0f : cl;
            cloudy[(size_t)sub * nlay + l] = cdf[l] >= 1.0f - c;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* cloud radii and in-cloud paths (common:793-961, 1332-1380)                */
/* ------------------------------------------------------------------------ */
static float retab_interp(const float *retab, float temp, int hi)
{
    int tint = (int)temp;
    int index = (int)(temp - 179.0f);
    if (index < 1) index = 1;
    if (index > hi) index = hi;
    float corr = temp - (float)tint;
    return retab[index - 1] * (1.0f - corr) + retab[index] * corr;
}

void ora_cloud_flags(int has_reqc, int has_reqi, int has_reqs, int icloud,
                     int *inflg, int *iceflg, int *liqflg)
{
    *inflg = 2; *iceflg = 3; *liqflg = 1;
    if (icloud != 0) {
        if (has_reqc) *inflg = 3;
        if (has_reqi) { *inflg = 4; *iceflg = 4; }
        if (has_reqs) { *inflg = 5; *iceflg = 5; }
        if (!has_reqs && has_reqi && has_reqc) { *inflg = 5; *iceflg = 5; }
    }
}

/* One column, nk layers.  Inputs already max-clipped (qc,qi,qs >= 0). */
void ora_cloud_paths(const ora_cache *c, const ora_in *in, int col, const float *tlay,
                     const float *pdel, ora_cloud *out)
{
    const int nk = in->nk;
    int inflg, iceflg, liqflg;
    ora_cloud_flags(in->has_reqc, in->has_reqi, in->has_reqs, in->icloud, &inflg, &iceflg, &liqflg);
    const float xland = in->xland[col], xice = in->xice[col], snow = in->snow[col];
    const float gravmks = 9.8066f;
    for (int k = 0; k < nk; ++k) {
        size_t i = (size_t)col * nk + k;
        float t = in->t3d[i];
        float cldfra = in->cldfra[i];
        float qc = fmaxf(in->qc[i], 0.0f), qi = fmaxf(in->qi[i], 0.0f), qs = fmaxf(in->qs[i], 0.0f);
        float recloud = 5.0f, reice = 10.0f, resnow = 10.0f;
        /* prepare_cloud_radii (common:801-874) */
        if (in->icloud != 0) {
            if (in->has_reqc) {
                recloud = fmaxf(2.5f, in->re_cloud[i] * 1.0e6f);
                int cloudy_min = (recloud <= 2.5f) && (cldfra > 0.0f);
                if (cloudy_min && (xland - 1.5f > 0.0f)) recloud = 10.5f;
                if (cloudy_min && (xland - 1.5f < 0.0f)) recloud = 7.5f;
            }
            if (in->has_reqi) {
                reice = fmaxf(5.0f, in->re_ice[i] * 1.0e6f);
                if ((reice <= 5.0f) && (cldfra > 0.0f))
                    reice = fmaxf(retab_interp(c->retab, t, 75), 5.0f);
            }
            if (in->has_reqs) resnow = fmaxf(10.0f, in->re_snow[i] * 1.0e6f);
            if (!in->has_reqs && in->has_reqi && in->has_reqc) {
                resnow = fmaxf(10.0f, in->re_ice[i] * 1.0e6f);
                qs = qi;
                qi = 0.0f;
                reice = 10.0f;
            }
        }
        /* prepare_cloud_path_inputs (common:877-961) */
        float temp = tlay[k];
        float dp = pdel[k];
        float denom = fmaxf(0.01f, cldfra);
        float gicewp = (qi + qs) * dp * 100.0f / gravmks * 1000.0f;
        float gliqwp = qc * dp * 100.0f / gravmks * 1000.0f;
        float cicewp = gicewp / denom;
        float cliqwp = gliqwp / denom;
        if (iceflg >= 4) {
            gicewp = qi * dp * 100.0f / gravmks * 1000.0f;
            cicewp = gicewp / denom;
        }
        float csnowp = 0.0f, res_adj = resnow;
        if (iceflg == 5) {
            float smf = 0.99f;
            if (res_adj > 130.0f) {
                float lim = (130.0f / res_adj) * (130.0f / res_adj);
                smf = fminf(0.99f, lim);
                res_adj = 130.0f;
            }
            float gsnowp = qs * smf * dp * 100.0f / gravmks * 1000.0f;
            csnowp = gsnowp / denom;
        }
        /* relcalc (common:1332-1365) with landm = 2 - xland, icefrac = xice,
         * snowh = 0.001 * snow */
        const float tmelt = 273.16f, rocean = 14.0f, rice = 14.0f, rland = 8.0f;
        float landm = 2.0f - xland;
        float snowh = 0.001f * snow;
        float rel = rland + (rocean - rland) * fminf(1.0f, fmaxf(0.0f, (tmelt - temp) * 0.05f));
        rel = rel + (rocean - rel) * fminf(1.0f, fmaxf(0.0f, snowh * 10.0f));
        rel = rel + (rocean - rel) * fminf(1.0f, fmaxf(0.0f, 1.0f - landm));
        rel = rel + (rice - rel) * fminf(1.0f, fmaxf(0.0f, xice));
        float rei = retab_interp(c->retab, temp, 94);   /* reicalc (common:1368-1380) */
        if (inflg >= 3) rel = recloud;
        if (iceflg >= 4) rei = reice;
        if (iceflg == 3) rei = fminf(140.0f, rei * 1.0315f);
        out->cldfrac[k] = cldfra;
        out->clwp[k] = cliqwp;
        out->ciwp[k] = cicewp;
        out->cswp[k] = (inflg == 5) ? csnowp : 0.0f;
        out->rel[k] = rel;
        out->rei[k] = rei;
        out->res[k] = (inflg == 5) ? res_adj : 10.0f;
    }
    out->inflg = inflg;
    out->iceflg = iceflg;
    out->liqflg = liqflg;
}

/* ------------------------------------------------------------------------ */
/* column-parallel loop on pthreads                                          */
/* ------------------------------------------------------------------------ */
typedef struct {
    int n, next, status;
    int (*fn)(void *, int);
    void *ctx;
    pthread_mutex_t lock;
} par_state;

static void *par_worker(void *arg)
{
    par_state *P = (par_state *)arg;
    for (;;) {
        pthread_mutex_lock(&P->lock);
        int i = P->next++;
        pthread_mutex_unlock(&P->lock);
        if (i >= P->n) break;
        int r = P->fn(P->ctx, i);
        if (r) {
            pthread_mutex_lock(&P->lock);
            P->status |= r;
            pthread_mutex_unlock(&P->lock);
        }
    }
    return NULL;
}

int ora_parallel_for(int n, int nthreads, int (*fn)(void *, int), void *ctx)
{
    par_state P = {n, 0, 0, fn, ctx, PTHREAD_MUTEX_INITIALIZER};
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    int started = 0;
    for (int i = 1; i < nthreads; ++i)
        if (pthread_create(&th[started], NULL, par_worker, &P) == 0) ++started;
    par_worker(&P);
    for (int i = 0; i < started; ++i) pthread_join(th[i], NULL);
    return P.status ? -P.status : 0;
}

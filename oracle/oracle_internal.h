/* Oracle internals shared between oracle_common.c, oracle_lw.c, oracle_sw.c. */
#ifndef RRTMG_ORACLE_INTERNAL_H
#define RRTMG_ORACLE_INTERNAL_H

#include "oracle.h"
#include <math.h>
#include <stddef.h>

#define LW_NBND 16
#define LW_NGPT 140
#define SW_NBND 14
#define SW_NGPT 112
#define MAX_LAY 512

typedef struct {
    const float *fracrefa, *fracrefb, *ka, *kb, *selfref, *forref;
    const float *ka_mn2, *kb_mn2, *ka_mn2o, *kb_mn2o, *ka_mo3, *kb_mo3;
    const float *ka_mco2, *kb_mco2, *ka_mco, *ka_mo2, *kb_mo2;
    const float *ccl4, *cfc11adj, *cfc12, *cfc22adj;
    int ngc, gofs, ka_rows, kb_rows;
} ora_lw_band;

typedef struct {
    ora_lw_band band[LW_NBND];
    const float *preflog, *tref, *chi_mls, *totplnk, *totplk16;
    const float *absice0, *absice1, *absice2, *absice3, *absliq1;
    float absliq0;
    const float *pade_tau, *pade_exp, *pade_tfn;
    float bpade;
    int ntbl;
} ora_lw_cache;

typedef struct {
    const float *ka, *kb, *selfref, *forref, *sfluxref, *rayla, *raylb, *rayl_g;
    const float *absch4, *abso3a, *abso3b, *absh2o, *absco2;
    float rayl, strrat, strrat1, givfac, scalekur;
    int layreffr, ngc, gofs, ka_rows, kb_rows, forref_rows, sflux_cols;
} ora_sw_band;

typedef struct {
    ora_sw_band band[SW_NBND];
    const float *preflog, *tref;
    const float *extliq1, *ssaliq1, *asyliq1, *extice2, *ssaice2, *asyice2;
    const float *extice3, *ssaice3, *asyice3, *fdlice3;
    const float *abari, *bbari, *cbari, *dbari, *ebari, *fbari;
    const float *pade_exp;
    float bpade;
    int ntbl;
} ora_sw_cache;

typedef struct {
    float o3wrk[31], ppwrkh[32];
    const float *retab, *pprof, *tprof;
    int nprof;
    ora_lw_cache lw;
    ora_sw_cache sw;
} ora_cache;

typedef struct {
    float cldfrac[MAX_LAY], clwp[MAX_LAY], ciwp[MAX_LAY], cswp[MAX_LAY];
    float rel[MAX_LAY], rei[MAX_LAY], res[MAX_LAY];
    int inflg, iceflg, liqflg;
} ora_cloud;

const ora_cache *ora_cache_of(const ora_tables *t);
/* run fn(ctx, i) for i in [0, n) on nthreads pthreads; returns -(OR of nonzero results) */
int ora_parallel_for(int n, int nthreads, int (*fn)(void *, int), void *ctx);
int ora_cache_init(const ora_tables *t, ora_cache *c);
int ora_lw_cache_init(const ora_tables *t, ora_lw_cache *c);
int ora_sw_cache_init(const ora_tables *t, ora_sw_cache *c);
void ora_o3data(const ora_cache *c, const float *plev, int nout, float *o3);
void ora_mcica_overlap2(const float *play, const float *cld_in, int nlay, int nsub,
                        int change_seed, unsigned char *cloudy, ora_binary32 *cdf_work);
void ora_cloud_flags(int has_reqc, int has_reqi, int has_reqs, int icloud,
                     int *inflg, int *iceflg, int *liqflg);
void ora_cloud_paths(const ora_cache *c, const ora_in *in, int col, const float *tlay,
                     const float *pdel, ora_cloud *out);

/* Pa -> hPa as the reference's REAL division (common:70-82): binary64
 * quotient rounded once to binary32, identical to a binary32 division. */
static inline float ora_pa_to_hpa(float p) { return (float)((double)p / 100.0); }

/* jnp.clip of an int index to [lo, hi] */
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* JAX gather semantics for a computed row index: negative wraps once, then clamp. */
static inline int jrow(int r, int n) { if (r < 0) r += n; return clampi(r, 0, n - 1); }

static inline float interpf(float lo, float hi, float f) { return lo + f * (hi - lo); }

/* FP64 mode's heating rate of a layer (LW: lw:5702-5712, SW: sw:2285-2301
 * with zdpgcp = heatfac / dp): the net fluxes at the layer's bottom (0) and
 * top (1), their difference and the division by the pressure thickness are
 * binary64 operations on the binary32 fluxes and pressures; one rounding to
 * binary32 at the end.  up - dn is the LW net flux; the SW passes (dn, up). */
static inline float ora_heating64(float heatfac, float up0, float dn0, float up1, float dn1,
                                  float plev0, float plev1)
{
    const double f0 = (double)up0 - (double)dn0;
    const double f1 = (double)up1 - (double)dn1;
    const double dp = (double)plev0 - (double)plev1;
    return (float)((double)heatfac * (f0 - f1) / dp);
}

#endif

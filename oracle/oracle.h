/*
 * CPU oracle for the RRTMG LW+SW radiation path of WRF-JAX (test infrastructure).
 *
 * This is a plain-C restatement of the reference's algorithm, statement by
 * statement, used ONLY by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg as the checker.  The product path never links it.
 *
 * Arithmetic contract (matches the reference's WRF default-REAL rounding,
 * src/wrf_jax/core/real_arithmetic.py:194-212 and module_ra_rrtmg_lw.py:51-105):
 *   every binary operation is one IEEE binary32 operation, round to nearest,
 *   no fused multiply-add (built with -ffp-contract=off); logf/expf/powf are
 *   glibc's, which the reference reproduces bit for bit
 *   (src/wrf_jax/core/wrf_math.py:120-280).
 */
#ifndef RRTMG_ORACLE_H
#define RRTMG_ORACLE_H

#include <stdint.h>

/* The type of the parts every build keeps in binary32: the McICA random
 * stream and its cloud decisions, so that all builds sample the same
 * subcolumns.  The binary64 build (fp64.h) defines it before it widens
 * `float`. */
#ifndef ORA_BINARY32_DEFINED
#define ORA_BINARY32_DEFINED 1
typedef float ora_binary32;
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- table blob -------------------------------------------------------- */
typedef struct ora_tables ora_tables;
ora_tables *ora_tables_load(const char *path);
void ora_tables_free(ora_tables *t);
/* pointer to a named float/int array; NULL if absent */
const void *ora_table(const ora_tables *t, const char *name, int *n_out);

/* ---- KISS random stream (common.py:964-1090) ----------------------------- */
void ora_kiss_step(uint32_t s[4], ora_binary32 *ran);
void ora_kiss_seeds(const ora_binary32 *pmid4, uint32_t s[4]);

/* ---- WRF-layout batch inputs ------------------------------------------- */
typedef struct {
    int ncol, nk;
    /* (ncol, nk) arrays, level fastest */
    const float *p3d, *pi3d, *t3d, *qv, *qc, *qi, *qs, *cldfra, *o3;
    const float *re_cloud, *re_ice, *re_snow;
    /* (ncol, nk+1) */
    const float *p8w, *t8w;
    /* (ncol,) */
    const float *tsk, *emiss, *albedo, *coszr, *xland, *xice, *snow;
    double p_top;                         /* Pa */
    float co2, n2o, ch4, cfc11, cfc12;   /* volume mixing ratios */
    float solcon;
    int has_reqc, has_reqi, has_reqs, icloud, cldovrlp;
    /* 1: the two steps the GPU's FP64 mode evaluates in binary64 (SW reftra
     * of layers whose delta-scaled single-scattering albedo is >= 0.999 or
     * whose optical depth is below 0.1; the heating rate of every layer from
     * the fifth-highest model layer up) are evaluated in binary64 here too;
     * 0: binary32 throughout (the reference) */
    int fp64_steps;
    /* optional (ncol,) Noah-MP albedos for sf_surface_physics == 8 (all four or
     * NULL): used for columns with xland < 1.5 (sw:2519-2530) */
    const float *alswvisdir, *alswvisdif, *alswnirdir, *alswnirdif;
} ora_in;

typedef struct {
    /* (ncol, nk) */
    float *rthraten, *rthratenc;
    /* (ncol,) : top/bottom fluxes */
    float *up_top, *upc_top, *dn_top, *dnc_top, *up_sfc, *upc_sfc, *dn_sfc, *dnc_sfc;
    /* SW only (ncol,) */
    float *swddir, *swddni, *swddif, *swddirc, *swddnic;
    /* optional diagnostics, NULL to skip; nlay = LW or SW layer count */
    float *taug, *fracs_or_taur;   /* (ncol, nlay, ngpt) */
    float *cldfmc, *taucmc;        /* (ncol, ngpt, nlay) */
    float *uflx, *dflx, *uflxc, *dflxc;   /* (ncol, nlay+1) */
    float *hr, *hrc;               /* (ncol, nlay) K/day */
} ora_out;

int ora_lw_nlayers(double p_top, int nk);
int ora_lw_columns(const ora_tables *t, const ora_in *in, ora_out *out, int nthreads);
int ora_sw_columns(const ora_tables *t, const ora_in *in, ora_out *out, int nthreads);
/* Test knob: move the LW cloud-absorptance expf and minor-gas powf results by
 * the given numbers of ulps (0, 0 = glibc, the default); process-wide. */
void ora_set_libm_perturbation(int exp_ulps, int pow_ulps);

#ifdef __cplusplus
}
#endif
#endif

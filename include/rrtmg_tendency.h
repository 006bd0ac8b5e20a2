/*
 * rrtmg_tendency: the radiation heating applied to the model's potential
 * temperature tendency, fused into one pass over the 3-D arrays.
 *
 * Replaces, for the radiation term, three reference steps:
 *   rthraten  = rthratenlw + rthratensw           (src/wrf_jax/runtime.py:7946)
 *   rthraten *= c1[k] * mut[i,j] + c2[k]          (calculate_phy_tend, src/wrf_jax/dyn_em/module_em.py:462,
 *                                                  multiply_3d 585-602, applied at 621-622; over the tile)
 *   rt_tendf += rthraten                          (phy_ra_ten -> add_a2a,
 *                                                  src/wrf_jax/physics/module_physics_addtendc.py:542, 173;
 *                                                  over the tile less the specified / nested boundary rows)
 * Each product and sum is one binary32 operation in the reference's order, so
 * results are bit-identical.
 *
 * Arrays are float32 device pointers in WRF memory order: 3-D fields
 * (ime-ims+1, kme-kms+1, jme-jms+1) row-major, c1/c2 (kme-kms+1), mut
 * (ime-ims+1, jme-jms+1).  Calls are asynchronous on the given stream.
 */
#ifndef RRTMG_TENDENCY_H
#define RRTMG_TENDENCY_H

#include "rrtmg_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* WRF index bounds (inclusive, Fortran numbering) and the lateral boundary
 * flags of the a2a region (module_physics_addtendc.py:131-170). */
typedef struct {
    int ids, ide, jds, jde, kds, kde;   /* domain */
    int ims, ime, jms, jme, kms, kme;   /* memory */
    int its, ite, jts, jte, kts, kte;   /* tile */
    int specified, nested, periodic_x;
} rrtmg_tendency_bounds;

/* The fused chain.  rthratensw may be NULL (rthraten = rthratenlw as given);
 * couple = 0 skips the mass coupling (c1, c2, mut may then be NULL); rthraten
 * (the coupled sum, written over the whole array) and rt_tendf (updated in
 * place) may each be NULL, not both.  RRTMG_BAD_ARG for inconsistent bounds
 * (memory extents < 1, more than 2^31 elements) or missing pointers. */
rrtmg_status rrtmg_radiation_tendency(const rrtmg_tendency_bounds *bounds, const float *rthratenlw,
                                      const float *rthratensw, const float *c1, const float *c2,
                                      const float *mut, int couple, float *rthraten, float *rt_tendf,
                                      void *stream);

/* phy_ra_ten alone (module_physics_addtendc.py:542): rt_tendf += rthraten over
 * the a2a region, in place. */
rrtmg_status rrtmg_phy_ra_ten(const rrtmg_tendency_bounds *bounds, float *rt_tendf, const float *rthraten,
                              void *stream);

#ifdef __cplusplus
}
#endif
#endif /* RRTMG_TENDENCY_H */

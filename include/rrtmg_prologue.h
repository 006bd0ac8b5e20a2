/*
 * rrtmg_prologue: the radiation inputs WRF-JAX derives on every radiation step
 * before its RRTMG calls, computed on the GPU.
 *
 * Replaces the prologue of _radiation_driver_stage (src/wrf_jax/runtime.py:7733-7766):
 *   _cal_cldfra1_np / _cal_cldfra1_jax   cloud fraction        (runtime.py:5896, :5967)
 *   _calc_coszen_np / _calc_coszen_jax   cos solar zenith      (runtime.py:6207, :6246)
 *   _cam_o3rad_jax -> _cam_o3rad_arrays  CAM ozone             (runtime.py:5804, :5822)
 * The per-step scalars (declination, solar constant, the equation of time,
 * ozone month weights) stay host work as in the reference; helpers below
 * compute them.
 *
 * Conventions are those of rrtmg_b200.h: float32 arrays in the WRF runtime
 * layout (nx, nk, ny) / (nx, ny), column c = i*ny + j, device pointers the
 * caller owns, asynchronous on the given stream, ordered status codes.
 * Results: ozone and cos zenith are bit-identical to the reference's numpy
 * path (the same binary32 operations; the SVML sin/cos emulation the
 * reference applies to whole groups of four west-east rows, glibc sinf/cosf
 * for the remaining rows).  Cloud fraction calls CUDA expf/powf where the
 * reference calls numpy's (host path) or XLA's (device path) exp and power,
 * so it agrees to a few units in the last place, except where such a
 * difference crosses the 0.01 cut or the saturation test.
 */
#ifndef RRTMG_PROLOGUE_H
#define RRTMG_PROLOGUE_H

#include "rrtmg_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-step scalars of the prologue. */
typedef struct {
    float tloctm0;      /* gmt + (fmod(xtime, 1440) + equation of time) / 60, hours
                           (runtime.py:6224-6234) */
    float sin_declin;   /* sin and cos of the solar declination (runtime.py:6240-6241) */
    float cos_declin;
    int month_lo;       /* CAM ozone months around the date, 0-based (runtime.py:5717-5750) */
    int month_hi;
    float fact_lo;      /* their interpolation weights */
    float fact_hi;
} rrtmg_prologue_scalars;

/* Declination [rad] and solar constant [W m-2] of a day of the year
 * (_radconst, runtime.py:5667-5690), binary32 with the host libm's sinf,
 * cosf and asinf (the reference calls numpy's float32 functions, which can
 * differ from libm in the last place). */
rrtmg_status rrtmg_radconst(double julian, float *declin, float *solcon);

/* The scalars from the calendar: julian day (fractional, 0-based), minutes
 * since the start of the run at which the zenith angle is wanted, start hour
 * (GMT) and declination (runtime.py:6220-6241, 5717-5750).  Binary32 with the
 * host libm's sinf/cosf for the equation of time and the declination. */
rrtmg_status rrtmg_prologue_scalars_from_calendar(double julian, double xtime, double gmt, double declin,
                                                  rrtmg_prologue_scalars *out);

/* CAM ozone climatology of a case, copied to the context's device (replaces
 * the cached loader _load_cam_ozone_tables, runtime.py:5697-5714): plev_pa
 * (levsiz) pressures in Pa and lat (latsiz) latitudes in degrees, both
 * ascending; ozone (12, latsiz, levsiz) volume mixing ratios, row-major.
 * Limits: 2 <= levsiz <= 128, 2 <= latsiz <= 256, latsiz * levsiz <= 12288.
 * Replaces a climatology set earlier; calls already queued keep the old one. */
rrtmg_status rrtmg_set_ozone_climatology(rrtmg_ctx *ctx, const float *plev_pa, int levsiz,
                                         const float *lat, int latsiz, const float *ozone);

typedef struct {
    const float *qv3d, *qc3d, *qi3d, *qs3d;   /* (nx, nk, ny) kg/kg */
    const float *t3d, *p3d;                   /* (nx, nk, ny) K, Pa */
    const float *xlat, *xlong;                /* (nx, ny) degrees */
} rrtmg_prologue_in;

typedef struct {
    float *cldfra3d;          /* (nx, nk, ny) cal_cldfra1, or NULL */
    float *o33d;              /* (nx, nk, ny) ozone volume mixing ratio, or NULL */
    float *coszr;             /* (nx, ny) cos solar zenith, or NULL */
    int *condensate_present;  /* device int: 1 if any qc, qi or qs of the nk levels
                                 has a nonzero magnitude, else 0 (the reference's
                                 cloud presence test, runtime.py:5110-5121); or NULL */
} rrtmg_prologue_out;

/* All requested outputs in one launch; inputs an output does not need may be
 * NULL (cldfra3d: the q and t fields and p3d; o33d: xlat and p3d; coszr: xlat
 * and xlong).  o33d needs a climatology (rrtmg_set_ozone_climatology). */
rrtmg_status rrtmg_radiation_prologue(rrtmg_ctx *ctx, int nx, int nk, int ny,
                                      const rrtmg_prologue_scalars *scalars,
                                      const rrtmg_prologue_in *in, rrtmg_prologue_out *out, void *stream);

/* One output each, mirroring the reference's three functions. */
rrtmg_status rrtmg_cal_cldfra1(rrtmg_ctx *ctx, int nx, int nk, int ny, const float *qv, const float *qc,
                               const float *qi, const float *qs, const float *t_phy, const float *p_phy,
                               float *cldfra, void *stream);
rrtmg_status rrtmg_calc_coszen(rrtmg_ctx *ctx, int nx, int ny, const float *xlat, const float *xlong,
                               const rrtmg_prologue_scalars *scalars, float *coszen, void *stream);
rrtmg_status rrtmg_cam_o3rad(rrtmg_ctx *ctx, int nx, int nk, int ny, const float *xlat, const float *p3d,
                             const rrtmg_prologue_scalars *scalars, float *o33d, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* RRTMG_PROLOGUE_H */

/*
 * rrtmg_b200: C-ABI of the B200 RRTMG longwave + shortwave radiation path.
 *
 * Drop-in for the two jitted column kernels WRF-JAX's radiation stage calls:
 *   rrtmg_lwrad_wrf_columns  (src/wrf_jax/physics/module_ra_rrtmg_lw.py:6789)
 *   rrtmg_swrad_wrf_columns  (src/wrf_jax/physics/module_ra_rrtmg_sw.py:2386)
 * dispatched from _run_radiation_sides / _run_paired_rrtmg
 * (src/wrf_jax/runtime.py:5422, :433, jitted at runtime.py:406-414).
 *
 * Conventions
 *   - Arrays are float32 in the WRF-JAX runtime layout: 3-D fields
 *     (west_east, bottom_top, south_north) = (nx, nk, ny) row-major, level-
 *     interface fields (nx, nk+1, ny), 2-D fields (nx, ny).  Column c = i*ny + j.
 *     (module_ra_rrtmg_sw.py:2435-2438, module_ra_rrtmg_lw.py:6572-6589)
 *   - Every array pointer is a DEVICE pointer the caller owns; outputs are
 *     written in place, inputs are never modified (the reference's calls are
 *     pure functions returning new arrays).
 *   - The library owns the lookup tables (uploaded once by rrtmg_create) and
 *     its per-call scratch (stream-ordered allocations on the call's stream).
 *   - Calls are asynchronous on the given cudaStream_t (passed as void*; NULL =
 *     legacy default stream).  One context may serve several streams and host
 *     threads concurrently.
 *   - Status codes are ordered: OK < BAD_ARG < UNSUPPORTED_OPTION < CUDA < TIMEOUT.
 *     Option combinations the reference rejects with NotImplementedError
 *     (module_ra_rrtmg_lw.py:5750-5753, module_ra_rrtmg_sw.py:1438-1441) return
 *     RRTMG_UNSUPPORTED_OPTION.
 */
#ifndef RRTMG_B200_H
#define RRTMG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    RRTMG_OK = 0,
    RRTMG_BAD_ARG = 1,
    RRTMG_UNSUPPORTED_OPTION = 2,
    RRTMG_CUDA = 3,
    RRTMG_TIMEOUT = 4
} rrtmg_status;

typedef struct rrtmg_ctx rrtmg_ctx;

/* Static keywords and scalars of one call (runtime.py:383-404 lists the
 * reference's static keywords; the gas scalars are runtime.py:5627-5664). */
typedef struct {
    int nx, ny, nk;          /* domain: nx*ny columns, nk mass levels */
    double p_top;            /* model top pressure, Pa (LW buffer layers) */
    float co2vmr, n2ovmr, ch4vmr, cfc11vmr, cfc12vmr;   /* volume mixing ratios */
    float solcon;            /* solar constant, W m-2 (SW) */
    int has_reqc, has_reqi, has_reqs;                   /* effective-radius inputs present */
    int icloud;              /* 0: no cloud microphysics radii (SW runs clear) */
    int cldovrlp;            /* 0 clear, >= 1 McICA maximum-random overlap */
    /* 0 (default): binary32 throughout, bit for bit the reference's results.
     * 1: FP64 mode; no counterpart in the reference.  Two steps run in binary64:
     * the SW delta-Eddington reflectance/transmittance (reftra,
     * module_ra_rrtmg_sw.py:3490-3601) of every layer whose delta-scaled
     * single-scattering albedo is >= 0.999 (the conservative branch, sw:2829,
     * and the nearly conservative layers where g1^2 - g2^2 cancels) or whose
     * optical depth is below 0.1 (where its terms cancel to O(tau)), and the
     * flux-difference heating rate dF/dp (lw:5706-5709, sw:2285-2300) of the
     * five highest model layers and every layer above them. */
    int fp64_steps;
} rrtmg_config;

/* Keyword arrays of rrtmg_lwrad_wrf_columns (module_ra_rrtmg_lw.py:6789-6822).
 * dz8w is accepted for signature parity and not read (the reference deletes it). */
typedef struct {
    const float *p3d, *p8w, *pi3d, *t3d, *t8w, *tsk, *dz8w;
    const float *qv3d, *qc3d, *qi3d, *qs3d, *cldfra3d, *o33d;
    const float *emiss, *xland, *xice, *snow;
    const float *re_cloud, *re_ice, *re_snow;
} rrtmg_lw_in;

/* Fields of RrtmgLwWrfColumnResult (module_ra_rrtmg_lw.py:499-518). */
typedef struct {
    float *rthratenlw, *rthratenlwc;                       /* (nx, nk, ny) K/s of theta */
    float *lwupt, *lwuptc, *lwuptcln, *lwdnt, *lwdntc, *lwdntcln;
    float *lwupb, *lwupbc, *lwupbcln, *lwdnb, *lwdnbc, *lwdnbcln;
    float *glw, *olr, *lwcf;                               /* (nx, ny) W m-2 */
} rrtmg_lw_out;

/* Keyword arrays of rrtmg_swrad_wrf_columns (module_ra_rrtmg_sw.py:2386-2420).
 * The four (nx, ny) albedo fields of the Noah-MP land model are optional: pass
 * all four for sf_surface_physics == 8 (module_ra_rrtmg_sw.py:2519-2530), NULL
 * otherwise.  With all four given, a column with xland < 1.5 takes its direct
 * and diffuse surface albedos from alswvisdir / alswvisdif in bands 25-28 and
 * from alswnirdir / alswnirdif in bands 16-24 and 29 (sw:2120-2127); the other
 * columns, and every column without them, use `albedo` for both. */
typedef struct {
    const float *p3d, *p8w, *pi3d, *t3d, *t8w, *tsk, *dz8w;
    const float *qv3d, *qc3d, *qi3d, *qs3d, *cldfra3d, *o33d;
    const float *albedo, *coszr, *xland, *xice, *snow;
    const float *re_cloud, *re_ice, *re_snow;
    const float *alswvisdir, *alswvisdif, *alswnirdir, *alswnirdif;
} rrtmg_sw_in;

/* Fields of RrtmgSwWrfColumnResult (module_ra_rrtmg_sw.py:617-642). */
typedef struct {
    float *rthratensw, *rthratenswc;                       /* (nx, nk, ny) */
    float *swupt, *swuptc, *swuptcln, *swdnt, *swdntc, *swdntcln;
    float *swupb, *swupbc, *swupbcln, *swdnb, *swdnbc, *swdnbcln;
    float *swcf, *gsw, *swddir, *swddni, *swddif, *swdownc, *swddnic, *swddirc;
    float *coszr;                                          /* (nx, ny) */
} rrtmg_sw_out;

/* Build a context on `device` from a table blob written by the package's
 * tables.py (replaces the lru-cached table loaders runtime.py:441-466). */
rrtmg_status rrtmg_create(const char *table_blob_path, int device, rrtmg_ctx **out);
rrtmg_status rrtmg_create_from_memory(const void *blob, size_t nbytes, int device, rrtmg_ctx **out);
void rrtmg_destroy(rrtmg_ctx *ctx);

/* LW: replaces _rrtmg_lwrad_wrf_columns_jit (runtime.py:406-409). */
rrtmg_status rrtmg_lwrad(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_lw_in *in,
                         rrtmg_lw_out *out, void *stream);
/* SW: replaces _rrtmg_swrad_wrf_columns_jit (runtime.py:410-414). */
rrtmg_status rrtmg_swrad(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_sw_in *in,
                         rrtmg_sw_out *out, void *stream);

/* LW / SW over the first *live_count columns of a domain, the count read on
 * the GPU when the kernels run (live_count: device memory, written earlier on
 * the same stream); no counterpart in the reference.  Columns c = i * ny + j
 * at or past the count are skipped and their outputs left as they were; the
 * results of the others are those of rrtmg_lwrad / rrtmg_swrad.  The
 * radiation surrogate uses it to re-solve the columns its gate
 * rejects without reading their number on the host. */
rrtmg_status rrtmg_lwrad_live(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_lw_in *in,
                              rrtmg_lw_out *out, const int *live_count, void *stream);
rrtmg_status rrtmg_swrad_live(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_sw_in *in,
                              rrtmg_sw_out *out, const int *live_count, void *stream);

/* LW / SW with the per-call scratch in a caller's workspace instead of the
 * context's stream-ordered pool; no counterpart in the reference.  For
 * callers whose framework owns device memory, such as an XLA custom call,
 * which receives the workspace as one more result buffer from XLA's
 * allocator.  rrtmg_lw_workspace_bytes / rrtmg_sw_workspace_bytes return the
 * bytes a call with this config needs under the context's current schedule
 * (0 for an invalid config); they also build the context's McICA jump table
 * for the config's layer count, the one allocation a first call would
 * otherwise make, so call them during set-up.  The workspace is device memory
 * on the context's device, 256-byte aligned, at least that many bytes, and
 * must not be used by anything else until the call's work on `stream` is
 * done.  Results are those of rrtmg_lwrad / rrtmg_swrad bit for bit. */
size_t rrtmg_lw_workspace_bytes(rrtmg_ctx *ctx, const rrtmg_config *cfg);
size_t rrtmg_sw_workspace_bytes(rrtmg_ctx *ctx, const rrtmg_config *cfg);
rrtmg_status rrtmg_lwrad_ws(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_lw_in *in, rrtmg_lw_out *out,
                            void *workspace, size_t workspace_bytes, void *stream);
rrtmg_status rrtmg_swrad_ws(rrtmg_ctx *ctx, const rrtmg_config *cfg, const rrtmg_sw_in *in, rrtmg_sw_out *out,
                            void *workspace, size_t workspace_bytes, void *stream);

/* LW with no allocation inside the call; no counterpart in the reference.
 * Same arguments and results as rrtmg_lwrad, but the McICA scratch lives in
 * fixed file-scope device arrays (32 MiB of mask words) instead of a per-call
 * stream-ordered allocation.  Limit: nlay * 5 * nx * ny <= 8,388,608 mask words
 * (nlay = rrtmg_lw_nlayers(p_top, nk)); larger domains get RRTMG_BAD_ARG.
 * The first call on each device looks up the scratch's address; make it
 * before any stream capture begins.  The scratch is shared by all contexts
 * and streams of a device: calls that overlap in time on one device race. */
rrtmg_status rrtmg_lwrad_static_scratch(rrtmg_ctx *ctx, const rrtmg_config *cfg,
                                        const rrtmg_lw_in *in, rrtmg_lw_out *out, void *stream);

/* Per-column status of the last call (the per-column status of the C-ABI;
 * the reference itself checks nothing at run time, so bad inputs propagate
 * silently into its outputs).  While enabled on a context, every rrtmg_lwrad /
 * rrtmg_swrad call ends with one more launch on its stream that writes a
 * bitmask per column into the context's status array for that side (0 = LW,
 * 1 = SW); the *_live and *_static_scratch calls do not.  Bits: */
#define RRTMG_COL_NONFINITE_INPUT   0x1u  /* a NaN or infinity in an input of the column */
#define RRTMG_COL_NONFINITE_OUTPUT  0x2u  /* a NaN or infinity in a result of the column */
#define RRTMG_COL_PRESSURE_ORDER    0x4u  /* p8w not decreasing upward, or p3d outside its interfaces */
#define RRTMG_COL_TEMPERATURE_RANGE 0x8u  /* t3d, t8w or tsk outside [160, 340) K: the tables clamp */
#define RRTMG_COL_FRACTION_RANGE    0x10u /* cldfra, emiss or albedo outside [0, 1], or coszr > 1 */
rrtmg_status rrtmg_column_status_enable(rrtmg_ctx *ctx, int enable);
/* Copies the status words of the last enabled call of `side` into dev_status
 * (device memory, ncol = nx * ny words of that call, column c = i * ny + j),
 * asynchronously on `stream`, ordered after that call when both use the same
 * stream.  RRTMG_BAD_ARG when no call was recorded or ncol differs. */
rrtmg_status rrtmg_last_column_errors(rrtmg_ctx *ctx, int side, uint32_t *dev_status, int ncol, void *stream);

/* Per-phase timing; no counterpart in the reference.  While enabled, every
 * rrtmg_lwrad / rrtmg_swrad call records CUDA events on its stream between
 * its phases, for up to 256 calls per side: the McICA masks, then per column
 * chunk the optics launches (LW: column set-up, layer set-up, gas optics; SW:
 * day list with the first chunk, column set-up, layer optics, solar source)
 * and the sweep launch.  rrtmg_timing_read waits for the recorded calls and
 * writes, oldest first, three durations in milliseconds per call to
 * ms[3 * i + k]: McICA, the optics phases summed over the chunks, the sweeps
 * summed; side 0 = LW, 1 = SW.  It returns the number of calls written (at
 * most max_calls), or -1. */
rrtmg_status rrtmg_timing_enable(rrtmg_ctx *ctx, int enable);
int rrtmg_timing_read(rrtmg_ctx *ctx, int side, float *ms, int max_calls);

/* Launch schedule of a context; no counterpart in the reference.  Columns per
 * launch of the LW band-group/finish pair and of the SW column kernel, the
 * largest domains (columns) that run the g-point split SW and LW schedules
 * (one thread per column and g-point; the LW one keeps 1,376 bytes of layer
 * optics per column and layer).  Defaults: 131072, 131072, 4096, 2048;
 * limits 1024..16777216, 1024..16777216, 0..16384, 0..8192.  Results do not
 * depend on the schedule.  The autotuner of the ensemble runner sets it. */
typedef struct {
    int lw_chunk_columns;
    int sw_chunk_columns;
    int sw_split_max_columns;
    int lw_split_max_columns;
} rrtmg_schedule;
rrtmg_status rrtmg_set_schedule(rrtmg_ctx *ctx, const rrtmg_schedule *schedule);
rrtmg_status rrtmg_get_schedule(const rrtmg_ctx *ctx, rrtmg_schedule *schedule);

/* Number of LW layers used for a model top and level count
 * (rrtmg_lw_nlayers, module_ra_rrtmg_common.py:1243-1247). */
int rrtmg_lw_nlayers(double p_top, int nk);

/* Human-readable text of the last error recorded on this context (or of the
 * last failed rrtmg_create when ctx is NULL). */
const char *rrtmg_last_error(const rrtmg_ctx *ctx);
const char *rrtmg_status_string(rrtmg_status status);

#ifdef __cplusplus
}
#endif
#endif /* RRTMG_B200_H */

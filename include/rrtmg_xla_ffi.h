/*
 * rrtmg_b200 as XLA custom calls: FFI handlers for jax.ffi.
 *
 * The reference's radiation stage calls its two jitted keyword kernels from
 * JAX (_run_radiation_sides, src/wrf_jax/runtime.py:5422; the traced time loop
 * places the radiation step at src/wrf_jax/trajectory.py:2573).  These
 * handlers let that JAX code call the B200 path inside a compiled program:
 * register them with
 *     jax.ffi.register_ffi_target("rrtmg_lwrad", jax.ffi.pycapsule(lib.rrtmg_ffi_lwrad), platform="CUDA")
 * (INTEGRATION.md shows the whole binding).  They follow XLA's FFI C ABI
 * (xla/ffi/api/c_api.h, API version 0.1): XLA passes a call frame and the
 * handler returns NULL on success or an error it created with XLA's API.
 *
 * Operands, in order (all float32, WRF layout as in rrtmg_b200.h):
 *   LW: the 20 arrays of rrtmg_lw_in;   SW: the 21 arrays of rrtmg_sw_in,
 *       then optionally the four Noah-MP albedos (sf_surface_physics == 8).
 * Results, in order: the 17 (LW) / 23 (SW) arrays of rrtmg_lw_out /
 *   rrtmg_sw_out, then one uint8 workspace of at least
 *   rrtmg_ffi_lw_workspace_bytes / rrtmg_ffi_sw_workspace_bytes bytes (XLA
 *   allocates it, so the handler allocates no device memory of its own).
 * Attributes (scalars, by name): LW p_top (f64), co2vmr n2ovmr ch4vmr
 *   cfc11vmr cfc12vmr (f32); SW solcon co2vmr n2ovmr ch4vmr (f32); both
 *   has_reqc has_reqi has_reqs icloud cldovrlp fp64_steps (s32).
 * Tables: one context per device, created at the first call on that device
 *   from the blob named by rrtmg_ffi_set_table_blob or, if unset, the
 *   RRTMG_TABLE_BLOB environment variable.  The workspace-size queries create
 *   it too; call them while setting up, before any capture.
 * The handlers do not declare command-buffer compatibility.
 */
#ifndef RRTMG_XLA_FFI_H
#define RRTMG_XLA_FFI_H

#include <stddef.h>

#include "rrtmg_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct XLA_FFI_CallFrame XLA_FFI_CallFrame;
typedef struct XLA_FFI_Error XLA_FFI_Error;

XLA_FFI_Error *rrtmg_ffi_lwrad(XLA_FFI_CallFrame *call_frame);
XLA_FFI_Error *rrtmg_ffi_swrad(XLA_FFI_CallFrame *call_frame);

/* Table blob for the handlers' contexts (copied; set before the first call). */
rrtmg_status rrtmg_ffi_set_table_blob(const char *path);
/* Workspace bytes of one call on `device` (0 on error; see rrtmg_last_error(NULL)). */
size_t rrtmg_ffi_lw_workspace_bytes(int device, const rrtmg_config *cfg);
size_t rrtmg_ffi_sw_workspace_bytes(int device, const rrtmg_config *cfg);

#ifdef __cplusplus
}
#endif
#endif /* RRTMG_XLA_FFI_H */

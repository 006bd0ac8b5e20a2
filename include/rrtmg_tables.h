/*
 * rrtmg_tables: the reference's own RRTMG data files read natively.
 *
 * RRTMG_LW_DATA and RRTMG_SW_DATA (src/wrf_jax/physics/data/rrtmg/) are
 * Fortran unformatted sequential files, big-endian, one record per band
 * (16 LW bands, 14 SW bands).  These calls parse them and reduce every band's
 * tables from 16 to its compressed g-points in binary32 (WRF's cmbgb, as the
 * reference's loaders do: module_ra_rrtmg_lw.py:554-950,
 * module_ra_rrtmg_sw.py:800-1170, module_ra_rrtmg_common.py:530-789), with no
 * Python step, and put the result in place of the absorption tables of a
 * table blob.  The rest of the blob (cloud, Pade and setcoef tables, the
 * g-point maps and weights, constants) is taken from the base blob as it is.
 * Replaces the lru-cached loaders load_rrtmg_lw/sw_compressed_lookup_tables.
 */
#ifndef RRTMG_TABLES_H
#define RRTMG_TABLES_H

#include "rrtmg_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Write a blob: the base blob with its lwN.* / swN.* absorption tables
 * rebuilt from the two data files.  RRTMG_BAD_ARG (text in
 * rrtmg_last_error(NULL)) for unreadable or malformed files. */
rrtmg_status rrtmg_blob_with_wrf_data(const char *base_blob_path, const char *lw_data_path,
                                      const char *sw_data_path, const char *out_blob_path);

/* rrtmg_create on that blob, built in memory. */
rrtmg_status rrtmg_create_with_wrf_data(const char *base_blob_path, const char *lw_data_path,
                                        const char *sw_data_path, int device, rrtmg_ctx **out);

#ifdef __cplusplus
}
#endif
#endif /* RRTMG_TABLES_H */

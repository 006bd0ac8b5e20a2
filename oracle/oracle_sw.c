/* Oracle: RRTMG shortwave restatement (test infrastructure only). */
#include "oracle_internal.h"

int ora_sw_cache_init(const ora_tables *t, ora_sw_cache *c) { (void)t; (void)c; return 0; }
int ora_sw_columns(const ora_tables *t, const ora_in *in, ora_out *out, int nthreads)
{
    (void)t; (void)in; (void)out; (void)nthreads;
    return -99;
}

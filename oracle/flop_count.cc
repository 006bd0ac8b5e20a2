/* Counter storage and read-out of the counted oracle build (flop_count.h). */
#include "flop_count.h"

thread_local ora_flop_counts ora_flops = {0, 0, 0, 0, 0, 0, 0};

extern "C" void ora_flop_counts_take(unsigned long long out[7]) {
    out[0] = ora_flops.add;
    out[1] = ora_flops.mul;
    out[2] = ora_flops.div;
    out[3] = ora_flops.sqrt;
    out[4] = ora_flops.exp;
    out[5] = ora_flops.log;
    out[6] = ora_flops.pow;
    ora_flops = ora_flop_counts{0, 0, 0, 0, 0, 0, 0};
}

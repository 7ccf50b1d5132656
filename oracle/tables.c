/* Exposes the seeded synthetic parameter generator to the Python test harness
 * (test infrastructure). The generator itself is the product's table source. */
#include "../lasp-d3_b200/csrc/d3_synth_params.h"

void oracle_synth_tables(int extended, float *c6ab, float *r0ab, float *rcov, float *r2r4) {
    if (extended)
        d3_synth_fill(D3_SYNTH_SEED, D3_NE_EXTENDED, D3_NREF_EXTENDED, 1, c6ab, r0ab, rcov, r2r4);
    else
        d3_synth_fill(D3_SYNTH_SEED, D3_NE_ORIGINAL, D3_NREF_ORIGINAL, 0, c6ab, r0ab, rcov, r2r4);
}

/*
 * Table definitions linked into the reference's CUDA build (oracle/_ref). The arrays
 * are filled once when the library loads, from the same seeded generator the engine
 * uses, so the reference and the engine see bit-identical parameters.
 * Test infrastructure only.
 */
#include "../../lasp-d3_b200/csrc/d3_synth_params.h"

#ifdef USE_EXTENDED_PARAMETERS
#define NE D3_NE_EXTENDED
#define NR D3_NREF_EXTENDED
#define EXT 1
#else
#define NE D3_NE_ORIGINAL
#define NR D3_NREF_ORIGINAL
#define EXT 0
#endif

extern "C" {
float c6ab_ref[NE][NE][NR][NR][3];
float r0ab[NE][NE];
float rcov[NE];
float r2r4[NE];
}

namespace {
struct FillTables {
    FillTables() { d3_synth_fill(D3_SYNTH_SEED, NE, NR, EXT, &c6ab_ref[0][0][0][0][0], &r0ab[0][0], rcov, r2r4); }
} fill_tables_at_load;
} // namespace

/*
 * Stand-in for the reference's missing src/gen_constants_extended.h (7-reference,
 * 103-element layout selected by USE_EXTENDED_PARAMETERS, src/constants_include.h:9-18).
 * Declarations only; ref_tables.cpp defines and fills them. Test infrastructure.
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
extern float c6ab_ref[103][103][7][7][3];
extern float r0ab[103][103];
extern float rcov[103];
extern float r2r4[103];
#ifdef __cplusplus
}
#endif

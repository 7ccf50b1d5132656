/*
 * Stand-in for the reference's missing src/gen_constants_original.h (listed in its
 * .MISSING_LARGE_BLOBS). It only DECLARES the four tables with the layout the
 * reference indexes in src/d3_buffer.cu:193-277; ref_tables.cpp defines them and
 * fills them at load time from the seeded synthetic generator. Test infrastructure:
 * used only to build the reference's own CUDA code as a checker.
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
extern float c6ab_ref[95][95][5][5][3];
extern float r0ab[95][95];
extern float rcov[95];
extern float r2r4[95];
#ifdef __cplusplus
}
#endif

/*
 * Seeded synthetic DFT-D3 parameter tables in the reference's table layout.
 *
 * The real Grimme D3 reference tables (c6ab / r0ab / rcov / r2r4) are third-party
 * data that are not available here. This generator produces a table with the SAME
 * layout and the same structural invariants, so the engine, the FP64 oracle and the
 * reference's own CUDA build can all be compiled against one identical table:
 *
 *   c6ab[e_i][e_j][a][b][3] = { C6ref, CNref(e_i, a), CNref(e_j, b) }
 *       - CNref depends only on (element, reference index), as in the real table,
 *         so the Gaussian weights factor per atom;
 *       - a reference that an element does not have is marked by -1 in all three
 *         slots (the reference kernel tests `CNref > -1`, src/d3_kernel.cu:725-728);
 *       - c6ab[i][j][a][b][0] == c6ab[j][i][b][a][0] (symmetric C6);
 *   r0ab[e_i][e_j]  symmetric, bohr (zero-damping and ATM radii);
 *   rcov[e]         covalent radius already multiplied by K2 = 4/3, bohr
 *                   (src/d3_kernel.cu:560 uses it without K2);
 *   r2r4[e]         sqrt(Q) so that C8 = 3 C6 r2r4_i r2r4_j (src/d3_kernel.cu:1050-1054).
 *
 * Table index e maps to atomic number Z as Z = e (5-reference layout, 95 entries,
 * index 0 unused by real atoms) or Z = e + 1 (7-reference "extended" layout, 103
 * entries), following IDX_ELEM in the reference's src/d3_buffer.cu:11-19.
 *
 * Only integer hashing, +, -, *, / and sqrt are used (all correctly rounded in
 * IEEE-754), so every compiler produces bit-identical tables.
 */
#ifndef D3_SYNTH_PARAMS_H
#define D3_SYNTH_PARAMS_H

#include <math.h>
#include <stdint.h>

#define D3_SYNTH_SEED 0x44335F42323030ULL /* "D3_B200" */

#define D3_NE_ORIGINAL 95
#define D3_NREF_ORIGINAL 5
#define D3_NE_EXTENDED 103
#define D3_NREF_EXTENDED 7

static inline uint64_t d3s_mix(uint64_t x) {
    /* splitmix64 finaliser */
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

/* uniform double in [0, 1) from a tuple of small integers */
static inline double d3s_u(uint64_t seed, uint64_t a, uint64_t b, uint64_t c, uint64_t d) {
    uint64_t h = d3s_mix(seed ^ d3s_mix(a + 0x1000ULL * d3s_mix(b + 0x100000ULL * d3s_mix(c + 0x7000000ULL * d3s_mix(d)))));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

static inline int d3s_period(int Z) {
    if (Z <= 2) return 1;
    if (Z <= 10) return 2;
    if (Z <= 18) return 3;
    if (Z <= 36) return 4;
    if (Z <= 54) return 5;
    if (Z <= 86) return 6;
    return 7;
}

/* number of valid references for element with atomic number Z (1..nref) */
static inline int d3s_nref_of(uint64_t seed, int Z, int nref) {
    if (Z <= 0) return 1;
    int n = 1 + (int)(d3s_u(seed, 11, (uint64_t)Z, 0, 0) * (double)nref);
    if (n > nref) n = nref;
    return n;
}

static inline double d3s_cnref(uint64_t seed, int Z, int a) {
    double cn = 0.0;
    for (int k = 1; k <= a; ++k) cn += 0.6 + 0.8 * d3s_u(seed, 12, (uint64_t)Z, (uint64_t)k, 0);
    return cn;
}

/* per-(element, reference) C6 base value, hartree*bohr^6 */
static inline double d3s_c6base(uint64_t seed, int Z, int a) {
    int p = d3s_period(Z);
    double g = 1.0 + 1.6 * (double)(p - 1);
    double c0 = 2.5 * g * g * (0.8 + 0.4 * d3s_u(seed, 13, (uint64_t)Z, 0, 0));
    double shrink = 1.0 - 0.08 * (double)a * d3s_u(seed, 14, (uint64_t)Z, (uint64_t)a, 0);
    return c0 * shrink;
}

static inline double d3s_rcov(uint64_t seed, int Z) {
    int p = d3s_period(Z);
    double r_ang = 0.30 + 0.22 * (double)(p - 1) + 0.15 * d3s_u(seed, 15, (uint64_t)Z, 0, 0);
    return r_ang * (4.0 / 3.0) / 0.52917726; /* K2-scaled, bohr */
}

static inline double d3s_r2r4(uint64_t seed, int Z) {
    int p = d3s_period(Z);
    return 2.0 + 1.2 * (double)(p - 1) + 1.5 * d3s_u(seed, 16, (uint64_t)Z, 0, 0);
}

static inline double d3s_r0(uint64_t seed, int Z) {
    int p = d3s_period(Z);
    return 3.5 + 0.9 * (double)(p - 1) + 0.8 * d3s_u(seed, 17, (uint64_t)Z, 0, 0);
}

/*
 * Fill tables for `ne` element slots and `nref` references.
 * extended == 0: slot e is atomic number e; extended != 0: slot e is atomic number e + 1.
 * c6ab: ne*ne*nref*nref*3 floats; r0ab: ne*ne; rcov, r2r4: ne.
 */
static inline void d3_synth_fill(uint64_t seed, int ne, int nref, int extended, float *c6ab, float *r0ab,
                                 float *rcov, float *r2r4) {
    for (int e = 0; e < ne; ++e) {
        int Z = extended ? e + 1 : e;
        rcov[e] = (float)d3s_rcov(seed, Z);
        r2r4[e] = (float)d3s_r2r4(seed, Z);
    }
    for (int ei = 0; ei < ne; ++ei) {
        int Zi = extended ? ei + 1 : ei;
        int ni = d3s_nref_of(seed, Zi, nref);
        for (int ej = 0; ej < ne; ++ej) {
            int Zj = extended ? ej + 1 : ej;
            int nj = d3s_nref_of(seed, Zj, nref);
            int zlo = Zi < Zj ? Zi : Zj, zhi = Zi < Zj ? Zj : Zi;
            double r0 = 0.5 * (d3s_r0(seed, Zi) + d3s_r0(seed, Zj)) *
                        (0.95 + 0.1 * d3s_u(seed, 18, (uint64_t)zlo, (uint64_t)zhi, 0));
            r0ab[ei * ne + ej] = (float)r0;
            for (int a = 0; a < nref; ++a) {
                for (int b = 0; b < nref; ++b) {
                    float *t = c6ab + ((((uint64_t)ei * ne + ej) * nref + a) * nref + b) * 3;
                    if (a >= ni || b >= nj) {
                        t[0] = -1.0f;
                        t[1] = -1.0f;
                        t[2] = -1.0f;
                        continue;
                    }
                    /* symmetric under (Zi,a) <-> (Zj,b) */
                    uint64_t k1 = (uint64_t)Zi * 16 + (uint64_t)a, k2 = (uint64_t)Zj * 16 + (uint64_t)b;
                    uint64_t klo = k1 < k2 ? k1 : k2, khi = k1 < k2 ? k2 : k1;
                    double c = sqrt(d3s_c6base(seed, Zi, a) * d3s_c6base(seed, Zj, b)) *
                               (0.9 + 0.2 * d3s_u(seed, 19, klo, khi, 0));
                    t[0] = (float)c;
                    t[1] = (float)d3s_cnref(seed, Zi, a);
                    t[2] = (float)d3s_cnref(seed, Zj, b);
                }
            }
        }
    }
}

#endif /* D3_SYNTH_PARAMS_H */

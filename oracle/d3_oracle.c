/*
 * FP64 CPU oracle for the LASP-D3 energy/force/stress path.
 *
 * TEST INFRASTRUCTURE. This file is the checker for the engine and the timed CPU
 * baseline of bench.py; nothing in the product links, loads or calls it.
 *
 * It restates, in double precision, the formulas of the reference's
 * src/d3_kernel.cu with the reference's enumeration and cutoff semantics:
 *   - image box: every pair (i, j, T) with T in [-n_k, n_k]^3 (ALL_ITERATE,
 *     src/d3_kernel.cu:632-667, bias decoding :652-654), n_k from
 *     calculate_cell_repeats (src/d3_buffer.cu:63-84), positions NOT wrapped;
 *   - CN: 0 < r^2 <= rc_CN^2 (src/d3_kernel.cu:626,662), term 1/(1+exp(-K1((Ri+Rj)/r-1)))
 *     with rcov already scaled by K2 (:544-574);
 *   - C6: reference-weighted Gaussian average with the max-exponent shift and the
 *     `CNref > -1` validity test (:709-881);
 *   - damping: zero (alpha 14/16) and Becke-Johnson (:359-424);
 *   - two-body: 0 < r^2 < rc^2 over ordered pairs, E/2 per ordered pair, dE/dCN of the
 *     central atom, force scalar and virial (:902-986, :1105-1154);
 *   - ATM: a >= b >= c in index order, images of b and c, every side in
 *     [1e-12, rc_ATM^2], scale 1/6 / 1/2 / 1 (:1235-1478), E/3 to each atom;
 *   - chain rule: 0 < r^2 <= rc_CN^2, (dE/dCN_i + dE/dCN_j) dCN_ij/dr (:1511-1556, :1624-1667).
 * Units: bohr and hartree inside; the caller converts (src/d3.cu:204-219).
 *
 * One reference behaviour is selectable: the reference scales ATM energies, dE/dCN
 * and stress by the 1/2, 1/6 repeated-index factors but not the ATM forces
 * (src/d3_kernel.cu:1422-1441). atm_force_scaled = 0 reproduces that; 1 applies the
 * factor to forces as well (forces then equal -dE/dx).
 *
 * Parameter tables come in per-handle form (element slots in the order of the
 * handle's sorted unique element list, src/d3_buffer.cu:193-277).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define K1 16.0
#define K3 4.0

typedef struct {
    int ne, nref;
    const float *c6ab; /* [ne][ne][nref][nref][3] */
    const float *r0ab; /* [ne][ne] */
    const float *rcov; /* [ne] */
    const float *r2r4; /* [ne] */
    double s6, s8, p1, p2; /* zero: p1 = sr6, p2 = sr8; BJ: p1 = a1, p2 = a2 */
    int damping;            /* 0 zero, 1 BJ */
    double rc, rc_cn, rc_atm;
    int use_atm;
    int atm_force_scaled;
    int c6_mode; /* 0 literal per-pair 2-D loop, 1 factorised per-atom weights */
    int smooth_cn; /* tanh^3 CN cutoff (reference's SMOOTH_CUTOFF_CN), 0 = off */
} oracle_params;

typedef struct {
    double *energy; /* [n] per-atom, hartree, reference sign (positive = binding) */
    double *forces; /* [n][3] hartree/bohr, F = +dE/dx in the reference's sign */
    double *virial; /* [9] hartree/bohr^3 (already divided by signed V) */
    double *cn;     /* [n] */
    double *dedcn;  /* [n] */
} oracle_out;

/* ------------------------------------------------------------------------ */
/* C6 with dC6/dCN_1 and dC6/dCN_2, literal form (src/d3_kernel.cu:709-798)  */
static void c6_literal(const oracle_params *p, int t1, int t2, double cn1, double cn2, double *c6, double *d1,
                       double *d2) {
    const int nr = p->nref;
    const float *base = p->c6ab + ((size_t)t1 * p->ne + t2) * nr * nr * 3;
    double mx = -INFINITY;
    for (int a = 0; a < nr; ++a)
        for (int b = 0; b < nr; ++b) {
            const float *e = base + (a * nr + b) * 3;
            if (e[1] > -1.0f && e[2] > -1.0f) {
                double da = cn1 - e[1], db = cn2 - e[2];
                double arg = -K3 * (da * da + db * db);
                if (arg > mx) mx = arg;
            }
        }
    double Z = 0, W = 0, dz1 = 0, dz2 = 0, dw1 = 0, dw2 = 0;
    for (int a = 0; a < nr; ++a)
        for (int b = 0; b < nr; ++b) {
            const float *e = base + (a * nr + b) * 3;
            if (e[1] > -1.0f && e[2] > -1.0f) {
                double da = cn1 - e[1], db = cn2 - e[2];
                double L = exp(-K3 * (da * da + db * db) - mx);
                double l1 = -2.0 * K3 * da * L, l2 = -2.0 * K3 * db * L;
                Z += e[0] * L;
                W += L;
                dz1 += e[0] * l1;
                dz2 += e[0] * l2;
                dw1 += l1;
                dw2 += l2;
            }
        }
    *c6 = W > 0.0 ? Z / W : 0.0;
    *d1 = W * W > 0.0 ? (dz1 * W - Z * dw1) / (W * W) : 0.0;
    *d2 = W * W > 0.0 ? (dz2 * W - Z * dw2) / (W * W) : 0.0;
}

/* factorised form: per-atom normalised weights w and dw (same mathematics) */
typedef struct {
    double w[8], dw[8];
} atom_weights;

static void atom_weights_of(const oracle_params *p, int t, double cn, atom_weights *aw) {
    const int nr = p->nref;
    /* CNref of element t at reference a: column 1 of c6ab[t][t][a][0] (depends on (t, a) only) */
    double mx = -INFINITY;
    double cr[8];
    int valid[8];
    for (int a = 0; a < nr; ++a) {
        const float *e = p->c6ab + ((((size_t)t * p->ne + t) * nr + a) * nr + 0) * 3;
        cr[a] = e[1];
        valid[a] = e[1] > -1.0f;
        if (valid[a]) {
            double d = cn - cr[a];
            double arg = -K3 * d * d;
            if (arg > mx) mx = arg;
        }
    }
    double sw = 0, sdw = 0, w[8], dw[8];
    for (int a = 0; a < nr; ++a) {
        if (valid[a]) {
            double d = cn - cr[a];
            w[a] = exp(-K3 * d * d - mx);
            dw[a] = -2.0 * K3 * d * w[a];
        } else {
            w[a] = 0;
            dw[a] = 0;
        }
        sw += w[a];
        sdw += dw[a];
    }
    for (int a = 0; a < nr; ++a) {
        if (sw > 0) {
            aw->w[a] = w[a] / sw;
            aw->dw[a] = dw[a] / sw - aw->w[a] * (sdw / sw);
        } else {
            aw->w[a] = 0;
            aw->dw[a] = 0;
        }
    }
}

static void c6_factorised(const oracle_params *p, int t1, int t2, const atom_weights *w1, const atom_weights *w2,
                          double *c6, double *d1, double *d2) {
    const int nr = p->nref;
    const float *base = p->c6ab + ((size_t)t1 * p->ne + t2) * nr * nr * 3;
    double c = 0, g1 = 0, g2 = 0;
    for (int a = 0; a < nr; ++a) {
        double v = 0, dv = 0;
        for (int b = 0; b < nr; ++b) {
            double cref = base[(a * nr + b) * 3];
            if (w2->w[b] != 0.0 || w2->dw[b] != 0.0) {
                v += cref * w2->w[b];
                dv += cref * w2->dw[b];
            }
        }
        c += w1->w[a] * v;
        g1 += w1->dw[a] * v;
        g2 += w1->w[a] * dv;
    }
    *c6 = c;
    *d1 = g1;
    *d2 = g2;
}

typedef struct {
    const oracle_params *p;
    const atom_weights *aw; /* per atom when c6_mode == 1 */
    const int *types;
    const double *cn;
} c6_ctx;

static inline void pair_c6(const c6_ctx *c, int64_t i, int64_t j, double *c6, double *d1, double *d2) {
    if (c->p->c6_mode == 1)
        c6_factorised(c->p, c->types[i], c->types[j], &c->aw[i], &c->aw[j], c6, d1, d2);
    else
        c6_literal(c->p, c->types[i], c->types[j], c->cn[i], c->cn[j], c6, d1, d2);
}

/* damping functions and derivatives (src/d3_kernel.cu:359-424) */
static void damping(int type, double r, double R0, double p1, double p2, double *f6, double *f8, double *df6,
                    double *df8) {
    if (type == 0) {
        double b6 = p1 * R0 / r, b8 = p2 * R0 / r;
        double b6_2 = b6 * b6, b6_4 = b6_2 * b6_2, b6_8 = b6_4 * b6_4, b6_14 = b6_8 * b6_4 * b6_2, b6_15 = b6_14 * b6;
        double b8_2 = b8 * b8, b8_4 = b8_2 * b8_2, b8_8 = b8_4 * b8_4, b8_16 = b8_8 * b8_8, b8_17 = b8_16 * b8;
        *f6 = 1.0 / (1.0 + 6.0 * b6_14);
        *f8 = 1.0 / (1.0 + 6.0 * b8_16);
        *df6 = 6.0 * 14.0 * (*f6) * (*f6) * b6_15 / p1 / R0;
        *df8 = 6.0 * 16.0 * (*f8) * (*f8) * b8_17 / p2 / R0;
    } else {
        double A = p1 * R0 + p2;
        double A2 = A * A, A4 = A2 * A2, A6 = A4 * A2, A8 = A4 * A4;
        double r2 = r * r, r4 = r2 * r2, r5 = r4 * r, r6 = r4 * r2, r7 = r6 * r, r8 = r4 * r4;
        *f6 = r6 / (r6 + A6);
        *f8 = r8 / (r8 + A8);
        *df6 = 6.0 * A6 * r5 / ((r6 + A6) * (r6 + A6));
        *df8 = 8.0 * A8 * r7 / ((r8 + A8) * (r8 + A8));
    }
    if (!isfinite(*f6)) *f6 = 0;
    if (!isfinite(*df6)) *df6 = 0;
    if (!isfinite(*f8)) *f8 = 0;
    if (!isfinite(*df8)) *df8 = 0;
}

static double cell_volume(const double *h) {
    return h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) + h[2] * (h[3] * h[7] - h[4] * h[6]);
}

static inline void image_shift(const double *h, int64_t bx, int64_t by, int64_t bz, double *s) {
    s[0] = bx * h[0] + by * h[3] + bz * h[6];
    s[1] = bx * h[1] + by * h[4] + bz * h[7];
    s[2] = bx * h[2] + by * h[5] + bz * h[8];
}

typedef struct {
    int64_t n_img;
    double *shift; /* [n_img][3] */
} image_set;

static void make_images(const double *h, const int64_t *mcb, image_set *im) {
    int64_t tot = mcb[0] * mcb[1] * mcb[2];
    im->n_img = tot;
    im->shift = (double *)malloc(sizeof(double) * 3 * tot);
    for (int64_t b = 0; b < tot; ++b) {
        int64_t x = (b % mcb[0]) - mcb[0] / 2;
        int64_t y = ((b / mcb[0]) % mcb[1]) - mcb[1] / 2;
        int64_t z = (b / (mcb[0] * mcb[1]) % mcb[2]) - mcb[2] / 2;
        image_shift(h, x, y, z, im->shift + 3 * b);
    }
}

static double cn_term(const oracle_params *p, double r, double rsum, double *dcn_over_r) {
    double e = exp(-K1 * (rsum / r - 1.0));
    if (p->smooth_cn) {
        double t = tanh(p->rc_cn - r);
        double sc = t * t * t;
        double dsc = 3.0 * t * t * (1.0 - t * t) * (-1.0);
        *dcn_over_r = 1.0 / ((1.0 + e) * (1.0 + e)) * (-K1) * e * rsum / (r * r * r) * sc + dsc * 1.0 / (1.0 + e) / r;
        return 1.0 / (1.0 + e) * sc;
    }
    *dcn_over_r = 1.0 / ((1.0 + e) * (1.0 + e)) * (-K1) * e * rsum / (r * r * r);
    return 1.0 / (1.0 + e);
}

/* ------------------------------------------------------------------------ */
/* per-atom pieces of the evaluation, shared by the full evaluation and the  */
/* per-atom term export                                                      */

/* CN of atom i over every atom and image (src/d3_kernel.cu:582-683) */
static double cn_of_atom(const oracle_params *p, int64_t n, const double *pos, const int *types,
                         const image_set *im, int64_t i) {
    const double rcn2 = p->rc_cn * p->rc_cn;
    double acc = 0;
    double ri = p->rcov[types[i]];
    for (int64_t j = 0; j < n; ++j) {
        double rs = ri + p->rcov[types[j]];
        for (int64_t b = 0; b < im->n_img; ++b) {
            double dx = pos[3 * i] - (pos[3 * j] + im->shift[3 * b]);
            double dy = pos[3 * i + 1] - (pos[3 * j + 1] + im->shift[3 * b + 1]);
            double dz = pos[3 * i + 2] - (pos[3 * j + 2] + im->shift[3 * b + 2]);
            double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 <= rcn2 && d2 > 0.0) {
                double dd;
                acc += cn_term(p, sqrt(d2), rs, &dd);
            }
        }
    }
    return acc;
}

/* growable half list of one apex: entry atoms and image positions */
typedef struct {
    int64_t cap, m;
    int64_t *lj;
    double *lv;
} atm_list;

static void atm_list_build(atm_list *L, int64_t n, const double *pos, const image_set *im, double ra2, int64_t a) {
    /* L_a: (b, T_b) with b <= a, 1e-12 <= r_ab^2 <= rc_atm^2, ordered by (b, image) */
    (void)n;
    L->m = 0;
    for (int64_t b = 0; b <= a; ++b)
        for (int64_t t = 0; t < im->n_img; ++t) {
            double px = pos[3 * b] + im->shift[3 * t], py = pos[3 * b + 1] + im->shift[3 * t + 1],
                   pz = pos[3 * b + 2] + im->shift[3 * t + 2];
            double rx = pos[3 * a] - px, ry = pos[3 * a + 1] - py, rz = pos[3 * a + 2] - pz;
            double d2 = rx * rx + ry * ry + rz * rz;
            if (d2 > ra2 || d2 < 1e-12) continue;
            if (L->m == L->cap) {
                L->cap = L->cap ? 2 * L->cap : 1024;
                L->lj = (int64_t *)realloc(L->lj, sizeof(int64_t) * L->cap);
                L->lv = (double *)realloc(L->lv, sizeof(double) * 3 * L->cap);
            }
            L->lj[L->m] = b;
            L->lv[3 * L->m] = px;
            L->lv[3 * L->m + 1] = py;
            L->lv[3 * L->m + 2] = pz;
            ++L->m;
        }
}

/* every triplet of apex a (src/d3_kernel.cu:1235-1478): energy E/3 to each atom, dE/dCN,
   forces into E[n], G[n], F[3n] and the virial into Vv[9] */
static void atm_apex(const oracle_params *p, const c6_ctx *cc, const double *pos, const int *types, double V,
                     const atm_list *L, int64_t a, double *E, double *G, double *F, double *Vv) {
    const double ra2 = p->rc_atm * p->rc_atm;
    const int64_t m = L->m;
    const int64_t *lj = L->lj;
    const double *lv = L->lv;
    const double *xa = pos + 3 * a;
    for (int64_t ib = 0; ib < m; ++ib) {
        int64_t b = lj[ib];
        double c6ab, dab_a, dab_b;
        pair_c6(cc, a, b, &c6ab, &dab_a, &dab_b);
        double r0ab = p->r0ab[types[a] * p->ne + types[b]];
        double rab[3] = {xa[0] - lv[3 * ib], xa[1] - lv[3 * ib + 1], xa[2] - lv[3 * ib + 2]};
        for (int64_t ic = 0; ic < m; ++ic) {
            int64_t c = lj[ic];
            if (c > b) break; /* entries are ordered by atom index */
            double rac[3] = {xa[0] - lv[3 * ic], xa[1] - lv[3 * ic + 1], xa[2] - lv[3 * ic + 2]};
            double rbc[3] = {lv[3 * ib] - lv[3 * ic], lv[3 * ib + 1] - lv[3 * ic + 1], lv[3 * ib + 2] - lv[3 * ic + 2]};
            double d_ac2 = rac[0] * rac[0] + rac[1] * rac[1] + rac[2] * rac[2];
            double d_bc2 = rbc[0] * rbc[0] + rbc[1] * rbc[1] + rbc[2] * rbc[2];
            if (d_ac2 > ra2 || d_bc2 > ra2 || d_ac2 < 1e-12 || d_bc2 < 1e-12) continue;
            double scale;
            if (c == b && b == a)
                scale = 1.0 / 6.0;
            else if (c == b || c == a || b == a)
                scale = 0.5;
            else
                scale = 1.0;
            double c6ac, dac_a, dac_c, c6bc, dbc_b, dbc_c;
            pair_c6(cc, a, c, &c6ac, &dac_a, &dac_c);
            pair_c6(cc, b, c, &c6bc, &dbc_b, &dbc_c);
            double r0ac = p->r0ab[types[a] * p->ne + types[c]];
            double r0bc = p->r0ab[types[b] * p->ne + types[c]];

            double ab2 = rab[0] * rab[0] + rab[1] * rab[1] + rab[2] * rab[2];
            double ab = sqrt(ab2), ab3 = ab2 * ab, ab4 = ab2 * ab2;
            double ac2 = d_ac2, ac = sqrt(ac2), ac3 = ac2 * ac, ac4 = ac2 * ac2;
            double bc2 = d_bc2, bc = sqrt(bc2), bc3 = bc2 * bc, bc4 = bc2 * bc2;
            double rsq = ab2 * ac2 * bc2, r = sqrt(rsq);
            double t1 = ab2 + ac2 - bc2, t2 = ab2 - ac2 + bc2, t3 = -ab2 + ac2 + bc2;
            double cosine = t1 * t2 * t3 / (8.0 * rsq);
            double ang = (1.0 + 3.0 * cosine) / (rsq * r);
            double dang_ab = 3.0 / 8.0 *
                             (ab3 * ab3 + ab4 * (ac2 + bc2) + ab2 * (3.0 * bc2 * bc2 + 2.0 * bc2 * ac2 + 3.0 * ac2 * ac2) -
                              5.0 * (bc2 - ac2) * (bc2 - ac2) * (bc2 + ac2)) /
                             (rsq * rsq * r);
            double dang_ac = 3.0 / 8.0 *
                             (ac3 * ac3 + ac4 * (bc2 + ab2) + ac2 * (3.0 * bc2 * bc2 + 2.0 * bc2 * ab2 + 3.0 * ab2 * ab2) -
                              5.0 * (bc2 - ab2) * (bc2 - ab2) * (bc2 + ab2)) /
                             (rsq * rsq * r);
            double dang_bc = 3.0 / 8.0 *
                             (bc3 * bc3 + bc4 * (ac2 + ab2) + bc2 * (3.0 * ac2 * ac2 + 2.0 * ac2 * ab2 + 3.0 * ab2 * ab2) -
                              5.0 * (ac2 - ab2) * (ac2 - ab2) * (ac2 + ab2)) /
                             (rsq * rsq * r);
            double C9 = -sqrt(c6ab * c6ac * c6bc);
            double dC9_ab = -0.5 * C9 / c6ab, dC9_ac = -0.5 * C9 / c6ac, dC9_bc = -0.5 * C9 / c6bc;
            double dC9a = dC9_ab * dab_a + dC9_ac * dac_a;
            double dC9b = dC9_ab * dab_b + dC9_bc * dbc_b;
            double dC9c = dC9_ac * dac_c + dC9_bc * dbc_c;
            double ravg = pow(ab2 * ac2 * bc2, 1.0 / 6.0);
            double r0 = pow(r0ab * r0ac * r0bc, 1.0 / 3.0);
            double x16 = pow(4.0 / 3.0 * r0 / ravg, 16.0);
            double fd = 1.0 / (1.0 + 6.0 * x16);
            double dfd = 2.0 * 16.0 * x16 * fd * fd;
            double e3 = C9 * ang * fd * scale / 3.0;
            E[a] += e3;
            E[b] += e3;
            E[c] += e3;
            G[a] += -dC9a * ang * fd * scale;
            G[b] += -dC9b * ang * fd * scale;
            G[c] += -dC9c * ang * fd * scale;
            double fs = p->atm_force_scaled ? scale : 1.0;
            double fab = -C9 * (dang_ab * fd - ang * dfd) / ab2;
            double fac = -C9 * (dang_ac * fd - ang * dfd) / ac2;
            double fbc = -C9 * (dang_bc * fd - ang * dfd) / bc2;
            for (int k = 0; k < 3; ++k) {
                for (int l = 0; l < 3; ++l)
                    Vv[k * 3 + l] += (-1.0 * fab * rab[k] * rab[l] + -1.0 * fac * rac[k] * rac[l] +
                                      -1.0 * fbc * rbc[k] * rbc[l]) /
                                     V * scale;
                F[3 * a + k] += (fab * rab[k] + fac * rac[k]) * fs;
                F[3 * b + k] += (-fab * rab[k] + fbc * rbc[k]) * fs;
                F[3 * c + k] += (-fac * rac[k] - fbc * rbc[k]) * fs;
            }
        }
    }
}

/* two-body terms of central atom i over its ordered pairs (src/d3_kernel.cu:997-1197):
   energy (E/2 per ordered pair), dE/dCN_i, force and virial */
static void twobody_atom(const oracle_params *p, const c6_ctx *cc, int64_t n, const double *pos, const int *types,
                         const image_set *im, double V, int64_t i, double *e_out, double *g_out, double *f_acc,
                         double *v_acc) {
    const double rc2 = p->rc * p->rc, s8 = p->s8, p1 = p->p1, p2 = p->p2;
    double e_acc = 0, g_acc = 0;
    for (int k = 0; k < 3; ++k) f_acc[k] = 0;
    for (int k = 0; k < 9; ++k) v_acc[k] = 0;
    int ti = types[i];
    for (int64_t j = 0; j < n; ++j) {
        int tj = types[j];
        double c6, d1, d2;
        pair_c6(cc, i, j, &c6, &d1, &d2);
        double rr_i = p->r2r4[ti], rr_j = p->r2r4[tj];
        double c8 = 3.0 * c6 * rr_i * rr_j, dc8 = 3.0 * d1 * rr_i * rr_j;
        double R0 = p->damping == 1 ? sqrt(3.0 * rr_i * rr_j) : (double)p->r0ab[ti * p->ne + tj];
        for (int64_t b = 0; b < im->n_img; ++b) {
            double dx = pos[3 * i] - (pos[3 * j] + im->shift[3 * b]);
            double dy = pos[3 * i + 1] - (pos[3 * j + 1] + im->shift[3 * b + 1]);
            double dz = pos[3 * i + 2] - (pos[3 * j + 2] + im->shift[3 * b + 2]);
            double d2r = dx * dx + dy * dy + dz * dz;
            if (!(d2r < rc2 && d2r > 0.0)) continue;
            double r = sqrt(d2r);
            double r3 = d2r * r, r4 = d2r * d2r, r6 = r3 * r3, r7 = r6 * r, r8 = r4 * r4, r9 = r8 * r, r10 = r6 * r4;
            double f6, f8, df6, df8;
            damping(p->damping, r, R0, p1, p2, &f6, &f8, &df6, &df8);
            double E6 = p->s6 * (c6 / r6) * f6, E8 = s8 * (c8 / r8) * f8;
            e_acc += (E6 + E8) / 2.0;
            g_acc += p->s6 * f6 * d1 / r6 + s8 * f8 * dc8 / r8;
            double fsc = p->s6 * c6 * f6 * (-6.0) / r8 + s8 * c8 * f8 * (-8.0) / r10 + p->s6 * c6 * df6 / r7 +
                         s8 * c8 * df8 / r9;
            double d[3] = {dx, dy, dz};
            for (int k = 0; k < 3; ++k) {
                f_acc[k] += fsc * d[k];
                for (int l = 0; l < 3; ++l) v_acc[k * 3 + l] += -1.0 * d[k] * fsc * d[l] / 2.0 / V;
            }
        }
    }
    *e_out = e_acc;
    *g_out = g_acc;
}

/* chain-rule force and virial of atom i (src/d3_kernel.cu:1571-1698); v_acc not yet
   divided by the volume */
static void chain_atom(const oracle_params *p, int64_t n, const double *pos, const int *types, const image_set *im,
                       const double *dedcn, int64_t i, double *f_acc, double *v_acc) {
    const double rcn2 = p->rc_cn * p->rc_cn;
    double ri = p->rcov[types[i]], gi = dedcn[i];
    for (int k = 0; k < 3; ++k) f_acc[k] = 0;
    for (int k = 0; k < 9; ++k) v_acc[k] = 0;
    for (int64_t j = 0; j < n; ++j) {
        double rs = ri + p->rcov[types[j]], g = gi + dedcn[j];
        for (int64_t b = 0; b < im->n_img; ++b) {
            double dx = pos[3 * i] - (pos[3 * j] + im->shift[3 * b]);
            double dy = pos[3 * i + 1] - (pos[3 * j + 1] + im->shift[3 * b + 1]);
            double dz = pos[3 * i + 2] - (pos[3 * j + 2] + im->shift[3 * b + 2]);
            double d2r = dx * dx + dy * dy + dz * dz;
            if (!(d2r <= rcn2 && d2r > 0.0)) continue;
            double dcn;
            cn_term(p, sqrt(d2r), rs, &dcn);
            double dE = g * dcn;
            double d[3] = {dx, dy, dz};
            for (int k = 0; k < 3; ++k) {
                f_acc[k] += dE * d[k];
                for (int l = 0; l < 3; ++l) v_acc[k * 3 + l] += (-1.0 * d[k] * dE * d[l]) / 2.0;
            }
        }
    }
}

/*
 * Full evaluation. pos: [n][3] bohr (unwrapped, in the caller's order), types: handle
 * slot per atom, cell: 3x3 rows = lattice vectors (bohr), mcb: image counts per
 * direction (odd). `subset`, when not NULL, restricts the central atoms of the
 * two-body, ATM-apex and chain-rule loops to subset[0..n_subset) (CN is always
 * computed for every atom); used only to time a bounded sample.
 */
int oracle_compute(const oracle_params *p, int64_t n, const double *pos, const int *types, const double *cell,
                   const int64_t *mcb, const int64_t *subset, int64_t n_subset, int nthreads, oracle_out *out) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    image_set im;
    make_images(cell, mcb, &im);
    const double V = cell_volume(cell);
    const double ra2 = p->rc_atm * p->rc_atm;
    int64_t ncent = subset ? n_subset : n;

    memset(out->energy, 0, sizeof(double) * n);
    memset(out->forces, 0, sizeof(double) * 3 * n);
    memset(out->virial, 0, sizeof(double) * 9);
    memset(out->dedcn, 0, sizeof(double) * n);

    /* ---- CN (every atom) ---- */
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < n; ++i) out->cn[i] = cn_of_atom(p, n, pos, types, &im, i);

    atom_weights *aw = NULL;
    if (p->c6_mode == 1) {
        aw = (atom_weights *)malloc(sizeof(atom_weights) * n);
        for (int64_t i = 0; i < n; ++i) atom_weights_of(p, types[i], out->cn[i], &aw[i]);
    }
    c6_ctx cc = {p, aw, types, out->cn};

    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    /* per-thread scatter buffers for ATM (energy, dE/dCN, forces) */
    double *th_e = (double *)calloc((size_t)nth * n, sizeof(double));
    double *th_g = (double *)calloc((size_t)nth * n, sizeof(double));
    double *th_f = (double *)calloc((size_t)nth * n * 3, sizeof(double));
    double *th_v = (double *)calloc((size_t)nth * 9, sizeof(double));

    /* ---- ATM (src/d3_kernel.cu:1199-1509) ---- */
    if (p->use_atm) {
#pragma omp parallel
        {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            double *E = th_e + (size_t)tid * n, *G = th_g + (size_t)tid * n, *F = th_f + (size_t)tid * n * 3;
            double *Vv = th_v + (size_t)tid * 9;
            atm_list L = {0, 0, NULL, NULL};
#pragma omp for schedule(dynamic, 1)
            for (int64_t s = 0; s < ncent; ++s) {
                int64_t a = subset ? subset[s] : (n - 1 - s);
                atm_list_build(&L, n, pos, &im, ra2, a);
                atm_apex(p, &cc, pos, types, V, &L, a, E, G, F, Vv);
            }
            free(L.lj);
            free(L.lv);
        }
    }

    /* ---- two-body (src/d3_kernel.cu:997-1197) ---- */
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *Vv = th_v + (size_t)tid * 9;
#pragma omp for schedule(dynamic, 4)
        for (int64_t s = 0; s < ncent; ++s) {
            int64_t i = subset ? subset[s] : s;
            double e_acc, g_acc, f_acc[3], v_acc[9];
            twobody_atom(p, &cc, n, pos, types, &im, V, i, &e_acc, &g_acc, f_acc, v_acc);
            out->energy[i] += e_acc;
            out->dedcn[i] += g_acc;
            for (int k = 0; k < 3; ++k) out->forces[3 * i + k] += f_acc[k];
            for (int k = 0; k < 9; ++k) Vv[k] += v_acc[k];
        }
    }

    /* gather ATM scatter buffers before the chain rule (dE/dCN must be complete) */
    for (int t = 0; t < nth; ++t) {
        for (int64_t i = 0; i < n; ++i) {
            out->energy[i] += th_e[(size_t)t * n + i];
            out->dedcn[i] += th_g[(size_t)t * n + i];
            for (int k = 0; k < 3; ++k) out->forces[3 * i + k] += th_f[((size_t)t * n + i) * 3 + k];
        }
    }

    /* ---- chain rule (src/d3_kernel.cu:1571-1698) ---- */
    double *th_v2 = (double *)calloc((size_t)nth * 9, sizeof(double));
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *Vv = th_v2 + (size_t)tid * 9;
#pragma omp for schedule(dynamic, 4)
        for (int64_t s = 0; s < ncent; ++s) {
            int64_t i = subset ? subset[s] : s;
            double f_acc[3], v_acc[9];
            chain_atom(p, n, pos, types, &im, out->dedcn, i, f_acc, v_acc);
            for (int k = 0; k < 3; ++k) out->forces[3 * i + k] += f_acc[k];
            for (int k = 0; k < 9; ++k) Vv[k] += v_acc[k] / V;
        }
    }
    for (int t = 0; t < nth; ++t)
        for (int k = 0; k < 9; ++k) out->virial[k] += th_v[t * 9 + k] + th_v2[t * 9 + k];

    free(th_e);
    free(th_g);
    free(th_f);
    free(th_v);
    free(th_v2);
    free(aw);
    free(im.shift);
    return 0;
}

/*
 * Per-atom terms of each pass for the atoms subset[0..n_subset), in the column layout
 * of the engine's diagnostic export (31 doubles per atom, hartree and bohr):
 *   [0] two-body energy, [1] its dE/dCN, [2..4] force, [5..10] virial (xx yy zz xy xz yz);
 *   [11] a third of the energy of every triplet whose apex (largest index) is the atom,
 *   [12] the apex's dE/dCN from those triplets, [13..15] its force from them, [16..21]
 *   their virial; [22..24] chain-rule force and [25..30] virial given dedcn_in (the
 *   complete dE/dCN of every atom; skipped when NULL).
 * cn_out receives the CN of every atom. Used by the parity tests on boxes too large for a
 * full oracle evaluation.
 */
int oracle_terms(const oracle_params *p, int64_t n, const double *pos, const int *types, const double *cell,
                 const int64_t *mcb, const int64_t *subset, int64_t n_subset, const double *dedcn_in, int nthreads,
                 double *cn_out, double *terms) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    image_set im;
    make_images(cell, mcb, &im);
    const double V = cell_volume(cell);
    const double ra2 = p->rc_atm * p->rc_atm;
    static const int vidx[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < n; ++i) cn_out[i] = cn_of_atom(p, n, pos, types, &im, i);
    atom_weights *aw = NULL;
    if (p->c6_mode == 1) {
        aw = (atom_weights *)malloc(sizeof(atom_weights) * n);
        for (int64_t i = 0; i < n; ++i) atom_weights_of(p, types[i], cn_out[i], &aw[i]);
    }
    c6_ctx cc = {p, aw, types, cn_out};
    memset(terms, 0, sizeof(double) * 31 * (size_t)n_subset);
#pragma omp parallel
    {
        double *E = (double *)calloc((size_t)n, sizeof(double)), *G = (double *)calloc((size_t)n, sizeof(double));
        double *F = (double *)calloc((size_t)n * 3, sizeof(double));
        atm_list L = {0, 0, NULL, NULL};
#pragma omp for schedule(dynamic, 1)
        for (int64_t s = 0; s < n_subset; ++s) {
            const int64_t i = subset[s];
            double *t = terms + 31 * (size_t)s;
            double f[3], v[9];
            twobody_atom(p, &cc, n, pos, types, &im, V, i, &t[0], &t[1], f, v);
            for (int k = 0; k < 3; ++k) t[2 + k] = f[k];
            for (int k = 0; k < 6; ++k) t[5 + k] = v[3 * vidx[k][0] + vidx[k][1]];
            if (p->use_atm) {
                double Vv[9] = {0};
                atm_list_build(&L, n, pos, &im, ra2, i);
                atm_apex(p, &cc, pos, types, V, &L, i, E, G, F, Vv);
                /* the apex's share, then clear what the apex's triplets touched */
                double etot = E[i];
                E[i] = 0;
                for (int64_t q = 0; q < L.m; ++q) {
                    const int64_t b = L.lj[q];
                    etot += E[b];
                    E[b] = 0;
                }
                t[11] = etot / 3.0;
                t[12] = G[i];
                for (int k = 0; k < 3; ++k) t[13 + k] = F[3 * i + k];
                for (int k = 0; k < 6; ++k) t[16 + k] = Vv[3 * vidx[k][0] + vidx[k][1]];
                G[i] = 0;
                F[3 * i] = F[3 * i + 1] = F[3 * i + 2] = 0;
                for (int64_t q = 0; q < L.m; ++q) {
                    const int64_t b = L.lj[q];
                    G[b] = 0;
                    F[3 * b] = F[3 * b + 1] = F[3 * b + 2] = 0;
                }
            }
            if (dedcn_in) {
                chain_atom(p, n, pos, types, &im, dedcn_in, i, f, v);
                for (int k = 0; k < 3; ++k) t[22 + k] = f[k];
                for (int k = 0; k < 6; ++k) t[25 + k] = v[3 * vidx[k][0] + vidx[k][1]] / V;
            }
        }
        free(E);
        free(G);
        free(F);
        free(L.lj);
        free(L.lv);
    }
    free(aw);
    free(im.shift);
    return 0;
}

/*
 * Exact work counts of the reference's enumeration over every atom (integers):
 * counts[0] CN ordered pairs (i, j, T) with 0 < r^2 <= rc_CN^2; counts[1] two-body
 * ordered pairs with 0 < r^2 < rc^2; counts[2] ATM triplets: over every apex a,
 * unordered pairs of distinct entries of its half list (b <= a, 1e-12 <= r_ab^2 <=
 * rc_ATM^2) whose own distance is in [1e-12, rc_ATM^2] (0 when ATM is off).
 */
int oracle_counts(const oracle_params *p, int64_t n, const double *pos, const double *cell, const int64_t *mcb,
                  int nthreads, int64_t *counts) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    image_set im;
    make_images(cell, mcb, &im);
    const double rc2 = p->rc * p->rc, rcn2 = p->rc_cn * p->rc_cn, ra2 = p->rc_atm * p->rc_atm;
    int64_t ncn = 0, n2 = 0, n3 = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : ncn, n2)
    for (int64_t i = 0; i < n; ++i)
        for (int64_t j = 0; j < n; ++j)
            for (int64_t b = 0; b < im.n_img; ++b) {
                double dx = pos[3 * i] - (pos[3 * j] + im.shift[3 * b]);
                double dy = pos[3 * i + 1] - (pos[3 * j + 1] + im.shift[3 * b + 1]);
                double dz = pos[3 * i + 2] - (pos[3 * j + 2] + im.shift[3 * b + 2]);
                double d2 = dx * dx + dy * dy + dz * dz;
                ncn += (d2 <= rcn2 && d2 > 0.0);
                n2 += (d2 < rc2 && d2 > 0.0);
            }
    if (p->use_atm) {
#pragma omp parallel reduction(+ : n3)
        {
            atm_list L = {0, 0, NULL, NULL};
#pragma omp for schedule(dynamic, 1)
            for (int64_t a = 0; a < n; ++a) {
                atm_list_build(&L, n, pos, &im, ra2, a);
                const double *lv = L.lv;
                for (int64_t ib = 1; ib < L.m; ++ib) {
                    const double bx = lv[3 * ib], by = lv[3 * ib + 1], bz = lv[3 * ib + 2];
                    int64_t c = 0;
                    for (int64_t ic = 0; ic < ib; ++ic) {
                        double dx = bx - lv[3 * ic], dy = by - lv[3 * ic + 1], dz = bz - lv[3 * ic + 2];
                        double d2 = dx * dx + dy * dy + dz * dz;
                        c += (d2 <= ra2 && d2 >= 1e-12);
                    }
                    n3 += c;
                }
            }
            free(L.lj);
            free(L.lv);
        }
    }
    counts[0] = ncn;
    counts[1] = n2;
    counts[2] = n3;
    free(im.shift);
    return 0;
}

/*
 * Image box of the reference (calculate_cell_repeats, src/d3_buffer.cu:63-84, with
 * the float-operand inverse of matrix_inverse<float,double>, :22-42) and its
 * workload decision (set_cell, :431-477). cell_f: bohr, float, rows = vectors.
 * Returns 1 for CELL_LIST, 0 for ALL_ITERATE; mcb receives the image counts.
 */
static void inverse_float_ops(const float m[3][3], double inv[3][3]) {
    /* every product and difference is evaluated in float, as in the reference's
       instantiation with T1 = float (the result is widened to double) */
    float det_f = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                  m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    double det = det_f;
    double id = 1.0 / det;
    inv[0][0] = (double)(float)(m[1][1] * m[2][2] - m[1][2] * m[2][1]) * id;
    inv[0][1] = (double)(float)(m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id;
    inv[0][2] = (double)(float)(m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
    inv[1][0] = (double)(float)(m[1][2] * m[2][0] - m[1][0] * m[2][2]) * id;
    inv[1][1] = (double)(float)(m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id;
    inv[1][2] = (double)(float)(m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
    inv[2][0] = (double)(float)(m[1][0] * m[2][1] - m[1][1] * m[2][0]) * id;
    inv[2][1] = (double)(float)(m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id;
    inv[2][2] = (double)(float)(m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
}

int oracle_cell_box(const float *cell_f, float rc, float rc_cn, int64_t *mcb, int64_t *num_grid) {
    float m[3][3];
    for (int i = 0; i < 9; ++i) m[i / 3][i % 3] = cell_f[i];
    double inv[3][3];
    inverse_float_ops(m, inv);
    double larger = rc_cn > rc ? rc_cn : rc;
    int mode = 1;
    for (int i = 0; i < 3; ++i) {
        double vn = sqrt(inv[i][0] * inv[i][0] + inv[i][1] * inv[i][1] + inv[i][2] * inv[i][2]);
        double h = 1.0 / vn;
        uint64_t g = (uint64_t)floor(h / larger);
        num_grid[i] = (int64_t)g;
        if (g <= 2) mode = 0;
    }
    float cut = (float)larger;
    for (int i = 0; i < 3; ++i) {
        /* row norms of transpose(inv) = column norms of inv */
        double nrm = sqrt(inv[0][i] * inv[0][i] + inv[1][i] * inv[1][i] + inv[2][i] * inv[2][i]);
        mcb[i] = ((int64_t)(int)(cut * nrm) + 1) * 2 + 1;
    }
    return mode;
}

/*
 * Cell-list assignment of construct_grids (src/d3_buffer.cu:496-607): grid index
 * and supercell shift per atom, from float coordinates (bohr) and the float-op inverse.
 */
void oracle_grid_assign(const float *cell_f, int64_t n, const float *pos_f, const int64_t *num_grid,
                        int64_t *grid_index, int64_t *super_idx) {
    float m[3][3];
    for (int i = 0; i < 9; ++i) m[i / 3][i % 3] = cell_f[i];
    double inv[3][3];
    inverse_float_ops(m, inv);
    for (int64_t i = 0; i < n; ++i) {
        uint64_t g[3];
        for (int j = 0; j < 3; ++j) {
            double fr = inv[0][j] * (double)pos_f[3 * i] + inv[1][j] * (double)pos_f[3 * i + 1] +
                        inv[2][j] * (double)pos_f[3 * i + 2];
            int64_t s = (int64_t)floor(fr);
            double w = fr - floor(fr);
            g[j] = (uint64_t)(w * (double)num_grid[j]);
            if (g[j] == (uint64_t)num_grid[j]) {
                s += 1;
                g[j] = 0;
            }
            super_idx[3 * i + j] = s;
        }
        grid_index[i] = (int64_t)(g[0] + g[1] * num_grid[0] + g[2] * num_grid[0] * num_grid[1]);
    }
}

/*
 * Learned ATM surrogate (no reference counterpart: the checker of the engine's
 * surrogate descriptors and of its force / stress chain).
 *
 * Descriptor of atom i, channel c, radial function k:
 *     G[i][c*nrbf + k] = sum over (j, T) with 0 < r^2 <= rc_atm^2 and chan[types[j]] = c of
 *                        C6_ij exp(-(r - mu0 - k dmu)^2 inv2s2) (1 + cos(pi r / rc_atm)) / 2
 * with this oracle's CN and C6. Given dEdG (derivative of an energy E = sum_i E_i(G_i),
 * hartree, the oracle's sign), accumulates the gradient +dE/dx into forces[n][3], the
 * virial (divided by V) into virial[9] and dE/dCN into dedcn[n], then applies the CN
 * chain rule. Any output may be NULL; dEdG NULL skips the backward part.
 */
int oracle_surrogate(const oracle_params *p, int64_t n, const double *pos, const int *types, const double *cell,
                     const int64_t *mcb, const int *chan, int nch, int nrbf, double mu0, double dmu, double inv2s2,
                     double *G, const double *dEdG, double *forces, double *virial, double *cn_out, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    image_set im;
    make_images(cell, mcb, &im);
    const double V = cell_volume(cell);
    const double rcn2 = p->rc_cn * p->rc_cn, ra2 = p->rc_atm * p->rc_atm;
    const double rca = p->rc_atm, pi = 3.14159265358979323846;
    const int nf = nch * nrbf;
    double *cn = (double *)calloc((size_t)n, sizeof(double));
    double *dedcn = (double *)calloc((size_t)n, sizeof(double));
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < n; ++i) {
        double acc = 0, ri = p->rcov[types[i]];
        for (int64_t j = 0; j < n; ++j) {
            double rs = ri + p->rcov[types[j]];
            for (int64_t b = 0; b < im.n_img; ++b) {
                double dx = pos[3 * i] - (pos[3 * j] + im.shift[3 * b]);
                double dy = pos[3 * i + 1] - (pos[3 * j + 1] + im.shift[3 * b + 1]);
                double dz = pos[3 * i + 2] - (pos[3 * j + 2] + im.shift[3 * b + 2]);
                double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 <= rcn2 && d2 > 0.0) {
                    double dd;
                    acc += cn_term(p, sqrt(d2), rs, &dd);
                }
            }
        }
        cn[i] = acc;
    }
    if (cn_out) memcpy(cn_out, cn, sizeof(double) * n);
    atom_weights *aw = NULL;
    if (p->c6_mode == 1) {
        aw = (atom_weights *)malloc(sizeof(atom_weights) * n);
        for (int64_t i = 0; i < n; ++i) atom_weights_of(p, types[i], cn[i], &aw[i]);
    }
    c6_ctx cc = {p, aw, types, cn};
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    double *th_v = (double *)calloc((size_t)nth * 9, sizeof(double));
    if (G) memset(G, 0, sizeof(double) * n * nf);
    if (forces) memset(forces, 0, sizeof(double) * 3 * n);
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *Vv = th_v + (size_t)tid * 9;
#pragma omp for schedule(dynamic, 4)
        for (int64_t i = 0; i < n; ++i) {
            const int ci = chan[types[i]];
            double f_acc[3] = {0, 0, 0}, v_acc[9] = {0}, g_acc = 0;
            for (int64_t j = 0; j < n; ++j) {
                const int cj = chan[types[j]];
                if (cj < 0) continue;
                double c6 = 0, d1 = 0, d2c = 0;
                int have_c6 = 0;
                for (int64_t b = 0; b < im.n_img; ++b) {
                    double dx = pos[3 * i] - (pos[3 * j] + im.shift[3 * b]);
                    double dy = pos[3 * i + 1] - (pos[3 * j + 1] + im.shift[3 * b + 1]);
                    double dz = pos[3 * i + 2] - (pos[3 * j + 2] + im.shift[3 * b + 2]);
                    double d2 = dx * dx + dy * dy + dz * dz;
                    if (!(d2 <= ra2 && d2 > 0.0)) continue;
                    if (!have_c6) {
                        pair_c6(&cc, i, j, &c6, &d1, &d2c);
                        have_c6 = 1;
                    }
                    const double r = sqrt(d2);
                    const double fc = 0.5 * (1.0 + cos(pi * r / rca));
                    const double dfc = -0.5 * (pi / rca) * sin(pi * r / rca);
                    double sa = 0, sb = 0;
                    for (int k = 0; k < nrbf; ++k) {
                        const double u = r - (mu0 + k * dmu);
                        const double ph = exp(-u * u * inv2s2);
                        const double psi = ph * fc;
                        if (G && ci >= 0) G[(size_t)i * nf + (size_t)cj * nrbf + k] += c6 * psi;
                        if (dEdG && ci >= 0) {
                            const double dpsi = ph * (dfc - 2.0 * u * inv2s2 * fc);
                            const double gg = dEdG[(size_t)i * nf + (size_t)cj * nrbf + k] +
                                              dEdG[(size_t)j * nf + (size_t)ci * nrbf + k];
                            sa += gg * dpsi;
                            sb += gg * psi;
                        }
                    }
                    if (dEdG && ci >= 0) {
                        const double a = c6 * sa / r; /* dE/dr_ij / r over both descriptors */
                        const double d[3] = {dx, dy, dz};
                        for (int k = 0; k < 3; ++k) {
                            f_acc[k] += a * d[k];
                            for (int l = 0; l < 3; ++l) v_acc[k * 3 + l] += -d[k] * a * d[l] / 2.0;
                        }
                        g_acc += sb * d1; /* dE/dC6_ij dC6_ij/dCN_i */
                    }
                }
            }
            if (forces)
                for (int k = 0; k < 3; ++k) forces[3 * i + k] += f_acc[k];
            dedcn[i] = g_acc;
            for (int k = 0; k < 9; ++k) Vv[k] += v_acc[k] / V;
        }
    }
    if (dEdG) {
        /* CN chain rule: (dE/dCN_i + dE/dCN_j) dCN_ij/dr over CN pairs */
#pragma omp parallel
        {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            double *Vv = th_v + (size_t)tid * 9;
#pragma omp for schedule(dynamic, 4)
            for (int64_t i = 0; i < n; ++i) {
                double ri = p->rcov[types[i]], gi = dedcn[i];
                double f_acc[3] = {0, 0, 0}, v_acc[9] = {0};
                for (int64_t j = 0; j < n; ++j) {
                    double rs = ri + p->rcov[types[j]], g = gi + dedcn[j];
                    for (int64_t b = 0; b < im.n_img; ++b) {
                        double dx = pos[3 * i] - (pos[3 * j] + im.shift[3 * b]);
                        double dy = pos[3 * i + 1] - (pos[3 * j + 1] + im.shift[3 * b + 1]);
                        double dz = pos[3 * i + 2] - (pos[3 * j + 2] + im.shift[3 * b + 2]);
                        double d2r = dx * dx + dy * dy + dz * dz;
                        if (!(d2r <= rcn2 && d2r > 0.0)) continue;
                        double dcn;
                        cn_term(p, sqrt(d2r), rs, &dcn);
                        double dE = g * dcn;
                        double d[3] = {dx, dy, dz};
                        for (int k = 0; k < 3; ++k) {
                            f_acc[k] += dE * d[k];
                            for (int l = 0; l < 3; ++l) v_acc[k * 3 + l] += (-1.0 * d[k] * dE * d[l]) / 2.0;
                        }
                    }
                }
                if (forces)
                    for (int k = 0; k < 3; ++k) forces[3 * i + k] += f_acc[k];
                for (int k = 0; k < 9; ++k) Vv[k] += v_acc[k] / V;
            }
        }
    }
    if (virial) {
        memset(virial, 0, sizeof(double) * 9);
        for (int t = 0; t < nth; ++t)
            for (int k = 0; k < 9; ++k) virial[k] += th_v[t * 9 + k];
    }
    free(th_v);
    free(cn);
    free(dedcn);
    free(aw);
    free(im.shift);
    return 0;
}

// ATM three-body kernel, precision form, block-pair schedule: every triplet visited once.
// Included by d3_engine.cu after k_atm32 (same per-entry set-up, weights and outputs).
//
// Per apex a (persistent CTAs take apexes from a work counter, largest lists first):
//  1. The entries of the half list are counting-sorted by the Hilbert-curve position of their
//     cell in a 16^3 grid over [-rc, rc]^3 around the apex, so 32 consecutive entries ("a
//     block") are close in space.
//     Per-entry set-up (FP64 C6 of the apex pair, its CN derivatives, damping ratio) is
//     written once per apex, in sorted order, to this CTA's slot of a global scratch array.
//  2. Block pairs (A, B), B >= A, whose bounding boxes are within rc_ATM of each other are
//     walked by the warps (rows A taken from a counter, in order). Lane L owns entry x = A[L];
//     at step s it pairs with y = B[(L + s) mod 32], so no two lanes of the warp touch the
//     same y in a step. Diagonal blocks take steps 1..16 (step 16 on lanes 0..15 only), so
//     every unordered pair of entries is visited exactly once.
//  3. The y block (positions, per-entry constants, and for every partner type the entry's
//     C6 row, derivative row and r0^2, from the YD32 table) is copied to shared memory by
//     cp.async while the previous block pair is visited (two buffers per warp). A lane takes
//     four steps per iteration as two packed f32x2 pairs (steps s, s+1 and s+2, s+3: their
//     partners sit side by side in one 16-byte slot), so every FP32 add / mul / fma of the
//     triplet term serves two visits. x-side sums stay in the lane's registers for the whole
//     row; y-side sums travel with their y (shifted four lanes down per iteration), so after
//     the last step the four sets in lane L belong to four consecutive y's and are gathered
//     by three shuffles into one entry's sums, added to that entry's accumulators (L2
//     atomics on this CTA's global slot, one per quantity per block pair).
//  4. Per entry e at the end: energy share SE/3, dE/dCN 0.5 (lam_ea SE + SD) and its force
//     F_e (FP64 atomics to the entry atom, as k_atm32); the apex gets SE/6, 0.5 lam_ae SE,
//     the force -sum F_e (each triplet term depends on relative positions only) and the
//     virial sum v_e (x) F_e, plus in the weighted form the corrections for the visits
//     whose energy weight w differs from the force weight wf.
// With f1, f2, f3 the force scalars of sides a-x, a-y, x-y of a triplet (mirror symmetry of
// k_atm: f2 of visit (x, y) is f1 of the mirrored visit), the quantities per entry are
//   SE = sum w E, SD = sum w E lam_{e,other}, F = sum wf ((f_apex-side + f3) v_e - f3 v_other);
// x lanes keep F as SF = sum wf (f_apex-side + f3) and W = sum wf f3 v_other (v_x is fixed
// along the row), y sums carry -F itself (five travelling quantities).
// C6_xy = Y_y[t_x] . w_x, dC6_xy/dCN_x = Y_y[t_x] . dw_x, dC6_xy/dCN_y = D_y[t_x] . w_x
// with the x entry's own weights in registers and the y entry's rows at the x type read
// from the staged block (the reverse factorisation halves the shared-memory bytes per
// visit against staging the x rows for every partner type).
// Profiles on the 10,000-atom box (ncu, one launch): shared-memory data pipe 85 % of peak
// with the x rows staged per type -> 49 % with the y rows; long-scoreboard stalls of the
// synchronous y gather removed by the cp.async double buffer; warp instructions -22 % with
// the packed pairs, which leaves the kernel bound by the latency of the packed chains
// (2 warps of 243 registers per scheduler, four independent chains).

// longest list this kernel takes (longer lists: k_atm32): chosen per launch, a multiple of
// 512 in [ATMB_MCAP_MIN, ATMB_MCAP_MAX], as large as the shared memory left by the warps allows
constexpr int ATMB_MCAP_MIN = 4096, ATMB_MCAP_MAX = 8192;
constexpr int ATMB_GRID = 16;     // spatial grid per dimension for the entry sort
constexpr int ATMB_CELLS = ATMB_GRID * ATMB_GRID * ATMB_GRID;
constexpr int ATMB_MAXW = 8;      // warps per CTA at most with two y buffers per warp
constexpr int ATMB_MAXW1 = 12;    // warps per CTA at most with one y buffer per warp (168
                                  // registers per thread: three warps per scheduler)
constexpr int ATMB_CTAS_PER_SM = 2; // preferred CTAs per SM (of four warps each)

// global scratch per CTA (float4 units): per-entry records sA, sB, sJ and the per-entry
// accumulators [6][mcap] floats
__host__ __device__ inline size_t atmb_scratch_per_cta(int mcap) { return 3 * (size_t)mcap + (6 * (size_t)mcap + 3) / 4; }

// shared memory: fixed part + per-warp staging
__host__ __device__ inline size_t atmb_smem_fixed(int ne, int NR, int mcap) {
    size_t b = (size_t)mcap * sizeof(int);                    // atom of each sorted entry
    b += 2 * (size_t)(mcap / 32) * sizeof(float4);            // block bounding boxes
    b += (size_t)((ne * ne + 3) & ~3) * sizeof(float);        // r0^2
    b += (size_t)((ne * NR + 1) & ~1) * sizeof(double);       // apex C6 rows
    return (b + 15) & ~(size_t)15;
}
// per warp: two buffers (the block pair being visited and the next one, filled by
// cp.async meanwhile), each the staged y block: the rows of its entries for every partner
// type as float4 [type][row quad][lane] (lanes read consecutive 16-byte words whatever the
// x type, so the reads are free of bank conflicts) and positions / per-entry constants
__host__ __device__ inline size_t atmb_buf_quads(int ne, int NR) { return 32 * ((size_t)ne * (atmb_row_floats(NR) / 4) + 2); }
// plus the lanes' FP64 carries (the weighted form's cross terms of the apex virial, row sums
// of the x entry), [15][lane]
// and the current block's positions / per-entry constants with entries k, k + 1 side by
// side ([4][32] float4)
constexpr int ATMB_NCARRY = 15;
__host__ __device__ inline size_t atmb_smem_warp(int ne, int NR, int nbuf = 2) {
    return nbuf * atmb_buf_quads(ne, NR) * sizeof(float4) + ATMB_NCARRY * 32 * sizeof(double) + 4 * 32 * sizeof(float4);
}

// a lane's view of FP64 carries kept in shared memory ([q][32] doubles): they change once
// per block pair, so they need not hold registers through the visits
struct AtmbCarry {
    double *p;
    __device__ __forceinline__ double &operator[](int q) const { return p[q * 32]; }
};

// 16-byte global -> shared copy that bypasses registers (cached in L2 only)
__device__ __forceinline__ void atmb_cp16(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void atmb_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's groups are still in flight
template <int N>
__device__ __forceinline__ void atmb_cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Position of cell (x, y, z) of the 16^3 grid along a Hilbert curve (Skilling's transform
// of the axes to the transposed Hilbert index, then bit interleaving). Consecutive entries in
// this order stay spatially adjacent (no jumps), so 32 consecutive entries form tighter
// blocks than in Morton order: a simulation of uniform apex spheres gives 0.57-0.62 of the
// visit slots of surviving block pairs in range, against 0.53-0.57 with Morton order on 8^3.
__device__ __forceinline__ int atmb_hilbert(int x, int y, int z) {
    int X[3] = {x, y, z};
    constexpr int M = ATMB_GRID >> 1;
#pragma unroll
    for (int Q = M; Q > 1; Q >>= 1) {
        const int P = Q - 1;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (X[i] & Q) {
                X[0] ^= P;
            } else {
                const int t = (X[0] ^ X[i]) & P;
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    X[1] ^= X[0];
    X[2] ^= X[1];
    int t = 0;
#pragma unroll
    for (int Q = M; Q > 1; Q >>= 1)
        if (X[2] & Q) t ^= Q - 1;
    int h = 0;
#pragma unroll
    for (int b = 3; b >= 0; --b)
#pragma unroll
        for (int i = 0; i < 3; ++i) h = (h << 1) | (((X[i] ^ t) >> b) & 1);
    return h;
}

// one row of the table (atmb_row_floats(NR) floats as float4 quads): C6 row Y, r0^2 of the
// type pair, derivative row D, atom index bits
template <int NR>
struct AtmbRow {
    float Y[NR], D[NR], r0sq;
    int j;
    __device__ __forceinline__ void load(const float4 *r, int k) {
        const float4 q0 = r[k], q1 = r[32 + k], q2 = r[64 + k];
        Y[0] = q0.x;
        Y[1] = q0.y;
        Y[2] = q0.z;
        Y[3] = q0.w;
        Y[4] = q1.x;
        if constexpr (NR == 5) {
            r0sq = q1.y;
            D[0] = q1.z;
            D[1] = q1.w;
            D[2] = q2.x;
            D[3] = q2.y;
            D[4] = q2.z;
            j = __float_as_int(q2.w);
        } else {
            const float4 q3 = r[96 + k];
            Y[5] = q1.y;
            Y[6] = q1.z;
            r0sq = q1.w;
            D[0] = q2.x;
            D[1] = q2.y;
            D[2] = q2.z;
            D[3] = q2.w;
            D[4] = q3.x;
            D[5] = q3.y;
            D[6] = q3.z;
            j = __float_as_int(q3.w);
        }
    }
};

// padding partner rows: unit C6 row and r0^2, zero derivative row, atom bits -1
template <int NR>
struct AtmbRowFill {
    __device__ __forceinline__ static void padding(float4 *r) {
        if constexpr (NR == 5) {
            r[0] = make_float4(1.f, 1.f, 1.f, 1.f);
            r[32] = make_float4(1.f, 1.f, 0.f, 0.f);
            r[64] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
        } else {
            r[0] = make_float4(1.f, 1.f, 1.f, 1.f);
            r[32] = make_float4(1.f, 1.f, 1.f, 1.f);
            r[64] = make_float4(0.f, 0.f, 0.f, 0.f);
            r[96] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
        }
    }
};

// packed pairs of references: NR = 5 as (0,1) (2,3) + 4, NR = 7 as (0,1) (2,3) (4,5) + 6
template <int NR>
struct AtmbVec {
    float2 p[(NR - 1) / 2];
    float l;
};

// sum_b r[b] v[b]: pairs of references in packed multiply-adds, the last one and the
// halves of the pair sum as scalars
template <int NR>
__device__ __forceinline__ float atmb_dot2(const float *r, const AtmbVec<NR> &v) {
    float2 acc = __fmul2_rn(make_float2(r[0], r[1]), v.p[0]);
    acc = __ffma2_rn(make_float2(r[2], r[3]), v.p[1], acc);
    if constexpr (NR == 7) acc = __ffma2_rn(make_float2(r[4], r[5]), v.p[2], acc);
    return fmaf(r[NR - 1], v.l, acc.x) + acc.y;
}

// per-row constants of the x entry as (v, v) pairs for the packed arithmetic of two visits;
// gq carries the factor (4/3)^16, c1 = -0.75 d1, d1x3 = 3 d1; w, dw its own C6 weights and
// their CN derivatives
template <int NR>
struct AtmbX2 {
    float2 vx, vy, vz, d1, ir1, id1, sq, gq, c1, d1x3;
    AtmbVec<NR> w, dw;
    int jx;
    bool qa;
};

// y sums of one entry over a block pair: SE = sum w E, SD = sum w E lam, and minus the
// entry's force from these visits, NF = -sum wf ((f_apex-side + f3) v_e - f3 v_other)
// (weighted form also SC = sum (w - wf)(f_apex-side + f3): where the energy weight w of a
// visit differs from its force weight wf, the apex virial gets SC v (x) v per entry)
template <bool SIMPLE>
struct AtmbSide {
    float SE, SD, NFx, NFy, NFz, SC;
    // add the y sums that lane src holds
    __device__ __forceinline__ void add_from(const AtmbSide &o, int src) {
        SE += __shfl_sync(0xffffffffu, o.SE, src);
        SD += __shfl_sync(0xffffffffu, o.SD, src);
        NFx += __shfl_sync(0xffffffffu, o.NFx, src);
        NFy += __shfl_sync(0xffffffffu, o.NFy, src);
        NFz += __shfl_sync(0xffffffffu, o.NFz, src);
        if (!SIMPLE) SC += __shfl_sync(0xffffffffu, o.SC, src);
    }
    __device__ __forceinline__ void flush(float *acc, int mcap, int e, int m) {
        if (e < m && (SE != 0.f || SD != 0.f || NFx != 0.f || NFy != 0.f || NFz != 0.f)) {
            atomicAdd(&acc[0 * mcap + e], SE);
            atomicAdd(&acc[1 * mcap + e], SD);
            atomicAdd(&acc[2 * mcap + e], -NFx);
            atomicAdd(&acc[3 * mcap + e], -NFy);
            atomicAdd(&acc[4 * mcap + e], -NFz);
            if (!SIMPLE && SC != 0.f) atomicAdd(&acc[5 * mcap + e], SC);
        }
    }
};

// packed y sums of one block pair (component x for one visit of a pair, y for the other),
// travelling with their y
template <bool SIMPLE>
struct AtmbYSums2 {
    float2 SE, SD, NFx, NFy, NFz, SC;
    // take those of lane src
    __device__ __forceinline__ void shift(int src) {
        float2 *v[6] = {&SE, &SD, &NFx, &NFy, &NFz, &SC};
#pragma unroll
        for (int q = 0; q < (SIMPLE ? 5 : 6); ++q) {
            v[q]->x = __shfl_sync(0xffffffffu, v[q]->x, src);
            v[q]->y = __shfl_sync(0xffffffffu, v[q]->y, src);
        }
    }
    // one component as a scalar side
    __device__ __forceinline__ AtmbSide<SIMPLE> part(int c) const {
        AtmbSide<SIMPLE> o{};
        o.SE = c ? SE.y : SE.x;
        o.SD = c ? SD.y : SD.x;
        o.NFx = c ? NFx.y : NFx.x;
        o.NFy = c ? NFy.y : NFy.x;
        o.NFz = c ? NFz.y : NFz.x;
        o.SC = c ? SC.y : SC.x;
        return o;
    }
};

// packed x sums of one block pair: SE, SD as above, SF = sum wf (f_apex-side + f3),
// W = sum wf f3 v_other (the entry's force is SF v_x - W); weighted form: SC as above and
// U = sum (w - wf) f3 v_other (the cross terms of the apex virial that the force weights
// miss)
template <bool SIMPLE>
struct AtmbXSums2 {
    float2 SE, SD, SF, Wx, Wy, Wz, Ux, Uy, Uz, SC;
};

// Two (possible) visits of entry x, with the staged partners k0 and k1 = k0 + 1 (mod 32)
// of two consecutive steps, in packed f32x2 arithmetic (component x: k0, y: k1): triplet
// terms, x-side sums into xt, y-side sums into ys, virial corrections where the energy and
// force weights differ. P0 = (x, x', y, y'), P1 = (z, z', d2, d2') of the two partners.
// Branch-free: an out-of-range pair (act false) runs on finite stand-in values (lanes
// without entry and padding partners sit at far, distinct points with positive C6 rows)
// with zero weights. With P = t1 t2 t3 (t1 = d1 + d2 - d3 ...), the angular term is
// A = (1 + 3/8 P / (d1 d2 d3)) / (r1 r2 r3)^3 and its side derivatives
// dA/dr_k / r_k = q52 G_k, G_k = 15/8 P + 3 d1 d2 d3 - 3/4 d_k (T - 2 t_ij),
// T = t12 + t13 + t23 (t_ij the product of the two t's without t_k). Signs are carried in
// the constants (f32x2 has add, mul and fma only): nw = -w, Em = -E, ndfd = -dfd.
template <int NR, bool SIMPLE>
__device__ __forceinline__ void atmb_visit2(const AtmbX2<NR> &X, int k0, float2 d3in, bool act0, bool act1,
                                            const float4 P0, const float4 P1, const float4 *yQ0, const float4 *yQ1,
                                            const float4 *yrow, int a, float third, bool force_scaled,
                                            AtmbXSums2<SIMPLE> &xt, AtmbYSums2<SIMPLE> &ys) {
    const int k1 = (k0 + 1) & 31;
    const float2 ONE = make_float2(1.0f, 1.0f), M1 = make_float2(-1.0f, -1.0f), M2 = make_float2(-2.0f, -2.0f);
    const float2 d3 = make_float2(act0 ? d3in.x : X.d1.x, act1 ? d3in.y : X.d1.x);
    const float4 Q0 = yQ0[k0], Q1 = yQ1[k0]; // (ir, ir', id2, id2'), (s, s', g, g')
    AtmbRow<NR> R0, R1; // the partners' rows at the x entry's type
    R0.load(yrow, k0);
    R1.load(yrow, k1);
    const float2 ir3 = make_float2(sfu_rsqrt(d3.x), sfu_rsqrt(d3.y));
    const float2 id3 = __fmul2_rn(ir3, ir3);
    // C6_xy = Y_y[t_x] . w_x, its derivatives dw_x and through D_y[t_x] = dw_y C
    const float2 c6 = make_float2(atmb_dot2<NR>(R0.Y, X.w), atmb_dot2<NR>(R1.Y, X.w));
    const float2 dcx = make_float2(atmb_dot2<NR>(R0.Y, X.dw), atmb_dot2<NR>(R1.Y, X.dw)); // dC6_xy/dCN_x
    const float2 dcy = make_float2(atmb_dot2<NR>(R0.D, X.w), atmb_dot2<NR>(R1.D, X.w));   // dC6_xy/dCN_y
    const float2 is3 = make_float2(sfu_rsqrt(c6.x), sfu_rsqrt(c6.y));
    const float2 s3 = __fmul2_rn(c6, is3);
    const float2 is3q = __fmul2_rn(is3, is3);
    const float2 lam_xy = __fmul2_rn(dcx, is3q), lam_yx = __fmul2_rn(dcy, is3q);
    // (r0_xy^2 / d3)^(8/3)
    const float2 lgu = __fmul2_rn(make_float2(sfu_log2(R0.r0sq * id3.x), sfu_log2(R1.r0sq * id3.y)),
                                  make_float2(8.0f / 3.0f, 8.0f / 3.0f));
    const float2 g3 = make_float2(sfu_exp2(lgu.x), sfu_exp2(lgu.y));
    // reference scale factors (src/d3_kernel.cu:1282-1290) as pair weights; SIMPLE: no
    // atom appears twice in the list (cell heights > 2 rc_ATM), every weight is 1
    float2 nw, wf;
    if (SIMPLE) {
        wf = make_float2(act0 ? 1.0f : 0.0f, act1 ? 1.0f : 0.0f);
        nw = make_float2(act0 ? -1.0f : 0.0f, act1 ? -1.0f : 0.0f);
    } else {
        const bool same0 = (X.jx == R0.j), same1 = (X.jx == R1.j);
        const bool img0 = X.qa | (R0.j == a), img1 = X.qa | (R1.j == a);
        const float w0 = act0 ? (same0 ? (X.qa ? third : 1.0f) : (img0 ? 0.5f : 1.0f)) : 0.0f;
        const float w1 = act1 ? (same1 ? (X.qa ? third : 1.0f) : (img1 ? 0.5f : 1.0f)) : 0.0f;
        nw = make_float2(-w0, -w1);
        wf = make_float2(act0 ? (force_scaled ? w0 : (same0 ? 2.0f : 1.0f)) : 0.0f,
                         act1 ? (force_scaled ? w1 : (same1 ? 2.0f : 1.0f)) : 0.0f);
    }
    const float2 d1 = X.d1, d2 = make_float2(P1.z, P1.w);
    const float2 irsq = __fmul2_rn(__fmul2_rn(X.id1, make_float2(Q0.z, Q0.w)), id3);
    const float2 ir9 = __fmul2_rn(__fmul2_rn(__fmul2_rn(irsq, X.ir1), make_float2(Q0.x, Q0.y)), ir3);
    const float2 t1 = __ffma2_rn(d3, M1, __fadd2_rn(d1, d2)); // d1 + d2 - d3
    const float2 t2 = __fadd2_rn(__ffma2_rn(d2, M1, d1), d3); // d1 - d2 + d3
    const float2 t3 = __fadd2_rn(__ffma2_rn(d1, M1, d2), d3); // -d1 + d2 + d3
    const float2 t12 = __fmul2_rn(t1, t2), t13 = __fmul2_rn(t1, t3), t23 = __fmul2_rn(t2, t3);
    const float2 P = __fmul2_rn(t12, t3);
    const float2 T = __fadd2_rn(__fadd2_rn(t12, t13), t23);
    const float2 Aang = __fmul2_rn(__ffma2_rn(__fmul2_rn(make_float2(0.375f, 0.375f), P), irsq, ONE), ir9);
    const float2 q52 = __fmul2_rn(ir9, irsq);
    const float2 base = __ffma2_rn(make_float2(1.875f, 1.875f), P, __fmul2_rn(__fmul2_rn(X.d1x3, d2), d3));
    const float2 G1 = __ffma2_rn(X.c1, __ffma2_rn(M2, t12, T), base);
    const float2 G2 = __ffma2_rn(__fmul2_rn(make_float2(-0.75f, -0.75f), d2), __ffma2_rn(M2, t13, T), base);
    const float2 G3 = __ffma2_rn(__fmul2_rn(make_float2(-0.75f, -0.75f), d3), __ffma2_rn(M2, t23, T), base);
    const float2 x16 = __fmul2_rn(__fmul2_rn(X.gq, make_float2(Q1.z, Q1.w)), g3);
    const float2 den = __ffma2_rn(make_float2(6.0f, 6.0f), x16, ONE);
    const float2 fd = make_float2(sfu_rcp(den.x), sfu_rcp(den.y));
    const float2 ndfd = __fmul2_rn(__fmul2_rn(__fmul2_rn(make_float2(-32.0f, -32.0f), x16), fd), fd);
    const float2 nC9 = __fmul2_rn(__fmul2_rn(X.sq, make_float2(Q1.x, Q1.y)), s3); // -C9
    const float2 nC9fd = __fmul2_rn(nC9, fd);
    const float2 Em = __fmul2_rn(nC9fd, Aang); // -E
    const float2 Ap = __fmul2_rn(nC9fd, q52), nBp = __fmul2_rn(__fmul2_rn(nC9, Aang), ndfd);
    const float2 f1 = __fmul2_rn(__ffma2_rn(Ap, G1, nBp), X.id1);
    const float2 f2 = __fmul2_rn(__ffma2_rn(Ap, G2, nBp), make_float2(Q0.z, Q0.w));
    const float2 f3 = __fmul2_rn(__ffma2_rn(Ap, G3, nBp), id3);
    const float2 wE = __fmul2_rn(nw, Em);
    const float2 wf3 = __fmul2_rn(wf, f3);
    const float2 f13 = __fadd2_rn(f1, f3), f23 = __fadd2_rn(f2, f3);
    const float2 yx = make_float2(P0.x, P0.y), yy = make_float2(P0.z, P0.w), yz = make_float2(P1.x, P1.y);
    xt.SE = __fadd2_rn(xt.SE, wE);
    xt.SD = __ffma2_rn(wE, lam_xy, xt.SD);
    xt.SF = __ffma2_rn(wf, f13, xt.SF);
    xt.Wx = __ffma2_rn(wf3, yx, xt.Wx);
    xt.Wy = __ffma2_rn(wf3, yy, xt.Wy);
    xt.Wz = __ffma2_rn(wf3, yz, xt.Wz);
    // minus the y entry's force: wf f3 v_x - wf (f2 + f3) v_y (SIMPLE: -wf = nw)
    const float2 nwf23 = __fmul2_rn(SIMPLE ? nw : __fmul2_rn(wf, M1), f23);
    ys.SE = __fadd2_rn(ys.SE, wE);
    ys.SD = __ffma2_rn(wE, lam_yx, ys.SD);
    ys.NFx = __ffma2_rn(wf3, X.vx, __ffma2_rn(nwf23, yx, ys.NFx));
    ys.NFy = __ffma2_rn(wf3, X.vy, __ffma2_rn(nwf23, yy, ys.NFy));
    ys.NFz = __ffma2_rn(wf3, X.vz, __ffma2_rn(nwf23, yz, ys.NFz));
    if (!SIMPLE) {
        // where the energy / virial weight w of a visit differs from its force weight wf
        // (repeated indices) the apex virial needs (w - wf) times the visit's virial
        // terms: (f_apex-side + f3) v (x) v per entry (coefficients SC, applied once per
        // entry at the end) and the cross terms -f3 (v_x (x) v_y + v_y (x) v_x) (U)
        const float2 dwf = __ffma2_rn(nw, M1, __fmul2_rn(wf, M1)); // -nw - wf = w - wf
        xt.SC = __ffma2_rn(dwf, f13, xt.SC);
        ys.SC = __ffma2_rn(dwf, f23, ys.SC);
        const float2 dwf3 = __fmul2_rn(dwf, f3);
        xt.Ux = __ffma2_rn(dwf3, yx, xt.Ux);
        xt.Uy = __ffma2_rn(dwf3, yy, xt.Uy);
        xt.Uz = __ffma2_rn(dwf3, yz, xt.Uz);
    }
}

// NBUF = 2: the next y block is copied while the current one is visited (up to 8 warps
// per CTA fit the shared memory); NBUF = 1: copy, wait, visit, which leaves room for 12
// warps (three per scheduler) whose visits hide each other's copies
// SIMPLE: this launch takes only the apexes of weight-free structures (no atom twice in a
// list), whose visits skip the repeated-index weights; the other launch takes the rest.
// Each instance then carries only the live values of its own visit form.
// FINE: a packed pair of steps is skipped when no lane has an in-range visit in it (else a
// group of four steps is skipped only when all four are out of range): fewer visit slots,
// less overlap between the two packed pairs of an iteration
template <int NR, int NBUF, bool SIMPLE, bool FINE>
__global__ void __launch_bounds__((NBUF == 2 ? ATMB_MAXW : ATMB_MAXW1) * 32, 1) k_atm32b(KP p, float4 *scratch) {
    extern __shared__ __align__(16) unsigned char smb[];
    const int ne = p.ne;
    const int nw = blockDim.x >> 5;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int mcap = p.atmb_mcap;
    int *sjy = reinterpret_cast<int *>(smb);                             // [mcap] atom of each sorted entry
    float4 *bblo = reinterpret_cast<float4 *>(sjy + mcap);               // [mcap/32]
    float4 *bbhi = bblo + mcap / 32;
    float *r0sq = reinterpret_cast<float *>(bbhi + mcap / 32);           // [ne][ne]
    double *yapex = reinterpret_cast<double *>(r0sq + ((ne * ne + 3) & ~3)); // [ne][NR]
    unsigned char *wbase = smb + atmb_smem_fixed(ne, NR, mcap) + (size_t)warp * atmb_smem_warp(ne, NR, NBUF);
    constexpr int RQ = atmb_row_floats(NR) / 4;                          // float4 quads per row
    // buffer layout: [ne][RQ][32] rows of the y block, [32] vx vy vz d2, [32] ir id2 s g
    float4 *ybuf0 = reinterpret_cast<float4 *>(wbase);
    // the sort's cell counters use the warps' staging area, idle between block-pair phases
    // (every warp region is at least 9 KB and there are at least two warps)
    int *cellpos = reinterpret_cast<int *>(smb + atmb_smem_fixed(ne, NR, mcap)); // [ATMB_CELLS]
    const size_t bufq = atmb_buf_quads(ne, NR);
    __shared__ int s_item, s_row;
    __shared__ double red[NBUF == 2 ? ATMB_MAXW : ATMB_MAXW1][12];
    float4 *sA = scratch + (size_t)blockIdx.x * atmb_scratch_per_cta(mcap); // vx vy vz d2
    float4 *sB = sA + mcap;                                              // ir id2 s g
    float4 *sJ = sB + mcap;                                              // j t lam_ea lam_ae
    float *acc = reinterpret_cast<float *>(sJ + mcap);                   // [6][mcap] (global, L2-resident)
    if (p.atm_off[p.n] > p.atm_cap) return; // list overflowed: the host grows it and re-runs
    for (int k = tid; k < ne * ne; k += blockDim.x) r0sq[k] = (float)(p.r0ab[k] * p.r0ab[k]);
    static_assert(NR == 5 || NR == 7, "reference counts of the parameter tables");
    const float x16c = (float)(4294967296.0 / 43046721.0); // (4/3)^16
    const float third = 1.0f / 3.0f;
    const float ratm2f = (float)p.ratm2;
    const bool force_scaled = p.atm_force_scaled != 0;
    const double rc = sqrt(p.ratm2);
    const double cinv = ATMB_GRID / (2.0 * rc);
    unsigned long long visits = 0;
    while (true) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(p.work, 1);
        __syncthreads();
        // work item = (apex, split): with split count S > 1 (systems with fewer apexes than
        // CTAs can hold) several CTAs share an apex, each taking its rows split, split + S, ...
        const int S = p.atmb_split;
        const int split = s_item % S;
        const int item = (s_item / S) * p.shard_world + p.shard_rank;
        if (item >= p.n) break;
        const int a = p.sorted_of[p.n - 1 - item];
        const long long e0 = p.atm_off[a];
        const int m = (int)(p.atm_off[a + 1] - e0);
        if (m > mcap) continue; // long lists: k_atm32
        const double4 xa = p.xs[a];
        const int ta = (int)xa.w;
        const SG &g = p.sg[p.sid[a]];
        if ((g.atm_simple != 0) != SIMPLE) continue; // the other instance takes this apex
        constexpr bool simple = SIMPLE;
        for (int k = tid; k < ne * NR; k += blockDim.x) yapex[k] = p.Y[(size_t)a * ne * NR + k];
        for (int k = tid; k < ATMB_CELLS; k += blockDim.x) cellpos[k] = 0;
        if (tid == 0) s_row = 0;
        for (int q = 0; q < (SIMPLE ? 5 : 6); ++q)
            for (int e = tid; e < m; e += blockDim.x) __stcg(&acc[q * mcap + e], 0.f);
        double dwa[NR];
#pragma unroll
        for (int b = 0; b < NR; ++b) dwa[b] = p.dw[(size_t)a * NR + b];
        __syncthreads();
        // ---- 1. spatial counting sort of the entries, per-entry set-up in sorted order
        for (int k = tid; k < m; k += blockDim.x) {
            const int2 ent = p.atm_ent[e0 + k];
            const double4 xj = p.xs[ent.x];
            double sx, sy, sz;
            image_vec(g, sext8(ent.y & 0xff), sext8((ent.y >> 8) & 0xff), sext8((ent.y >> 16) & 0xff), sx, sy, sz);
            const int cx = min(ATMB_GRID - 1, max(0, (int)((xj.x + sx - xa.x + rc) * cinv)));
            const int cy = min(ATMB_GRID - 1, max(0, (int)((xj.y + sy - xa.y + rc) * cinv)));
            const int cz = min(ATMB_GRID - 1, max(0, (int)((xj.z + sz - xa.z + rc) * cinv)));
            atomicAdd(&cellpos[atmb_hilbert(cx, cy, cz)], 1);
        }
        __syncthreads();
        if (warp == 0) {
            // exclusive scan of the cell counts, 32 cells per step (conflict-free rows)
            int carry = 0;
            for (int r = 0; r < ATMB_CELLS; r += 32) {
                const int v = cellpos[r + lane];
                int incl = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += u;
                }
                cellpos[r + lane] = carry + incl - v;
                carry += __shfl_sync(0xffffffffu, incl, 31);
            }
        }
        __syncthreads();
        // scatter the entry numbers, then order each cell's entries by entry number: the
        // sorted order (and so the blocks) is then the same in every CTA that sorts this
        // apex, which the apex split relies on (each split walks its own share of block rows)
        for (int k = tid; k < m; k += blockDim.x) {
            const int2 ent = p.atm_ent[e0 + k];
            const double4 xj = p.xs[ent.x];
            double sx, sy, sz;
            image_vec(g, sext8(ent.y & 0xff), sext8((ent.y >> 8) & 0xff), sext8((ent.y >> 16) & 0xff), sx, sy, sz);
            const int cx = min(ATMB_GRID - 1, max(0, (int)((xj.x + sx - xa.x + rc) * cinv)));
            const int cy = min(ATMB_GRID - 1, max(0, (int)((xj.y + sy - xa.y + rc) * cinv)));
            const int cz = min(ATMB_GRID - 1, max(0, (int)((xj.z + sz - xa.z + rc) * cinv)));
            sjy[atomicAdd(&cellpos[atmb_hilbert(cx, cy, cz)], 1)] = k;
        }
        __syncthreads();
        // cell c now spans [end of cell c - 1, cellpos[c]); cells hold a few entries each
        for (int c = tid; c < ATMB_CELLS; c += blockDim.x) {
            const int lo = c ? cellpos[c - 1] : 0, hi = cellpos[c];
            for (int q = lo + 1; q < hi; ++q) {
                const int v = sjy[q];
                int r = q - 1;
                while (r >= lo && sjy[r] > v) {
                    sjy[r + 1] = sjy[r];
                    --r;
                }
                sjy[r + 1] = v;
            }
        }
        __syncthreads();
        for (int pos = tid; pos < m; pos += blockDim.x) {
            const int k = sjy[pos];
            const int2 ent = p.atm_ent[e0 + k];
            const int jp = ent.x;
            const double4 xj = p.xs[jp];
            const int tp = (int)xj.w;
            double sx, sy, sz;
            image_vec(g, sext8(ent.y & 0xff), sext8((ent.y >> 8) & 0xff), sext8((ent.y >> 16) & 0xff), sx, sy, sz);
            const double vx = xj.x + sx - xa.x, vy = xj.y + sy - xa.y, vz = xj.z + sz - xa.z;
            const double d2 = vx * vx + vy * vy + vz * vz;
            const double *ya = yapex + tp * NR;                   // C6_ae = y_{a,tp} . w_e
            const double *yq = p.Y + ((size_t)jp * ne + ta) * NR; // dC6_ae/dCN_a = y_{e,ta} . dw_a
            double c6 = 0, dca = 0, dcq = 0;
#pragma unroll
            for (int b = 0; b < NR; ++b) {
                const double wb = p.w[(size_t)jp * NR + b], dwb = p.dw[(size_t)jp * NR + b];
                c6 += ya[b] * wb;
                dcq += ya[b] * dwb;
                dca += yq[b] * dwa[b];
            }
            sA[pos] = make_float4((float)vx, (float)vy, (float)vz, (float)d2);
            sB[pos] = make_float4((float)(1.0 / sqrt(d2)), (float)(1.0 / d2), (float)sqrt(c6),
                                  (float)pow((double)r0sq[ta * ne + tp] / d2, 8.0 / 3.0));
            sJ[pos] = make_float4(__int_as_float(jp), __int_as_float(tp), (float)(dcq / c6), (float)(dca / c6));
            sjy[pos] = jp; // this thread's own slot: the entry number it replaces was read above
        }
        __syncthreads();
        // ---- block bounding boxes
        const int nb = (m + 31) >> 5;
        for (int b = warp; b < nb; b += nw) {
            const int e = b * 32 + lane;
            const float4 v = sA[e < m ? e : b * 32];
            float lx = v.x, ly = v.y, lz = v.z, hx = v.x, hy = v.y, hz = v.z;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lx = fminf(lx, __shfl_xor_sync(0xffffffffu, lx, o));
                ly = fminf(ly, __shfl_xor_sync(0xffffffffu, ly, o));
                lz = fminf(lz, __shfl_xor_sync(0xffffffffu, lz, o));
                hx = fmaxf(hx, __shfl_xor_sync(0xffffffffu, hx, o));
                hy = fmaxf(hy, __shfl_xor_sync(0xffffffffu, hy, o));
                hz = fmaxf(hz, __shfl_xor_sync(0xffffffffu, hz, o));
            }
            if (lane == 0) {
                bblo[b] = make_float4(lx, ly, lz, 0.f);
                bbhi[b] = make_float4(hx, hy, hz, 0.f);
            }
        }
        __syncthreads();
        // ---- 2./3. block pairs
        // apex force (3) and virial (6) of this lane, and the row sums of its x entry
        // carries: virial cross terms of the weighted form (xx yy zz xy xz yz), and the row
        // sums of this lane's x entry
        const AtmbCarry apx{reinterpret_cast<double *>(wbase + NBUF * bufq * sizeof(float4)) + lane};
        const AtmbCarry xs{apx.p + 6 * 32}; // SE SD SF Wx Wy Wz, weighted form also Ux Uy Uz
        // positions (x, x', y, y'), (z, z', d2, d2') and constants (ir, ir', id2, id2'),
        // (s, s', g, g') of the current y block, entries k and k + 1 at slot k
        float4 *yP0 = reinterpret_cast<float4 *>(wbase + NBUF * bufq * sizeof(float4) + ATMB_NCARRY * 32 * sizeof(double));
        float4 *yP1 = yP0 + 32, *yQ0 = yP1 + 32, *yQ1 = yQ0 + 32;
#pragma unroll
        for (int q = 0; q < 6; ++q) apx[q] = 0.0;
        // rows are handed out in order (row A holds nb - A block pairs, so the dearest go
        // first and the cheapest close the apex, shortening the wait at its barrier)
        for (;;) {
            int A = 0;
            if (lane == 0) A = split + S * atomicAdd(&s_row, 1);
            A = __shfl_sync(0xffffffffu, A, 0);
            if (A >= nb) break;
            const int xe = A * 32 + lane;
            const bool xvalid = xe < m;
            // a lane without entry sits at a far point (distinct from the padding partners)
            // with weights (1, 0, ...), so its visits stay finite
            float vx = 3e4f, vy = 3e4f, vz = 3e4f, d1 = 1.f, ir1 = 1.f, id1 = 1.f, sq = 0.f, gq = 0.f;
            int jx = -1, tx = 0;
            float wx[NR], dwx[NR];
#pragma unroll
            for (int b = 0; b < NR; ++b) {
                wx[b] = b == 0 ? 1.f : 0.f;
                dwx[b] = 0.f;
            }
            if (xvalid) {
                const float4 qa4 = sA[xe], qb4 = sB[xe], qj4 = sJ[xe];
                vx = qa4.x;
                vy = qa4.y;
                vz = qa4.z;
                d1 = qa4.w;
                ir1 = qb4.x;
                id1 = qb4.y;
                sq = qb4.z;
                gq = qb4.w * x16c;
                jx = __float_as_int(qj4.x);
                tx = __float_as_int(qj4.y);
#pragma unroll
                for (int b = 0; b < NR; ++b) {
                    wx[b] = p.w32[(size_t)jx * NR + b];
                    dwx[b] = p.dw32[(size_t)jx * NR + b];
                }
            }
            const bool qa = (jx == a);
            AtmbX2<NR> X;
            X.vx = make_float2(vx, vx);
            X.vy = make_float2(vy, vy);
            X.vz = make_float2(vz, vz);
            X.d1 = make_float2(d1, d1);
            X.ir1 = make_float2(ir1, ir1);
            X.id1 = make_float2(id1, id1);
            X.sq = make_float2(sq, sq);
            X.gq = make_float2(gq, gq);
            X.c1 = make_float2(-0.75f * d1, -0.75f * d1);
            X.d1x3 = make_float2(3.0f * d1, 3.0f * d1);
#pragma unroll
            for (int i = 0; i < (NR - 1) / 2; ++i) {
                X.w.p[i] = make_float2(wx[2 * i], wx[2 * i + 1]);
                X.dw.p[i] = make_float2(dwx[2 * i], dwx[2 * i + 1]);
            }
            X.w.l = wx[NR - 1];
            X.dw.l = dwx[NR - 1];
            X.jx = jx;
            X.qa = qa;
#pragma unroll
            for (int q = 0; q < (simple ? 6 : 9); ++q) xs[q] = 0.0;
            float xsc = 0.f; // weighted form: the x entry's virial coefficient over this row
            // block pairs (A, B) whose boxes are within rc_ATM, visited in order of B; the
            // y block of the next one is copied (cp.async) while the current one is visited
            auto near = [&](int B) {
                const float4 la = bblo[A], ha = bbhi[A], lb = bblo[B], hb = bbhi[B];
                const float dx = fmaxf(0.f, fmaxf(la.x - hb.x, lb.x - ha.x));
                const float dy = fmaxf(0.f, fmaxf(la.y - hb.y, lb.y - ha.y));
                const float dz = fmaxf(0.f, fmaxf(la.z - hb.z, lb.z - ha.z));
                return fmaf(dx, dx, fmaf(dy, dy, dz * dz)) <= ratm2f * 1.0001f;
            };
            auto next_near = [&](int B) {
                while (B < nb && !near(B)) ++B;
                return B;
            };
            auto stage = [&](int B, float4 *buf) {
                float4 *rows = buf, *ya = buf + ne * RQ * 32, *yb = ya + 32;
                const int ye = B * 32 + lane;
                if (ye < m) {
                    atmb_cp16(ya + lane, sA + ye);
                    atmb_cp16(yb + lane, sB + ye);
                    const float4 *src = reinterpret_cast<const float4 *>(p.YD32) + (size_t)sjy[ye] * ne * RQ;
                    for (int t = 0; t < ne; ++t)
#pragma unroll
                        for (int q = 0; q < RQ; ++q) atmb_cp16(rows + (t * RQ + q) * 32 + lane, src + t * RQ + q);
                } else {
                    // padding partner: a far point with zero C6 share that fails every
                    // distance test; unit rows keep C6_xy positive
                    ya[lane] = make_float4(-3e4f, -3e4f, -3e4f, 1.f);
                    yb[lane] = make_float4(1.f, 1.f, 0.f, 0.f);
                    for (int t = 0; t < ne; ++t) AtmbRowFill<NR>::padding(rows + t * RQ * 32 + lane);
                }
            };
            int B = next_near(A);
            int cur = 0;
            __syncwarp(); // the previous row's visits are done with every buffer
            if (NBUF == 2) {
                if (B < nb) stage(B, ybuf0);
                atmb_cp_commit();
            }
            while (B < nb) {
                const int Bn = next_near(B + 1);
                __syncwarp(); // every lane is done with the buffer about to be filled
                if (NBUF == 2) {
                    if (Bn < nb) stage(Bn, ybuf0 + (cur ^ 1) * bufq);
                    atmb_cp_commit();
                    atmb_cp_wait<1>(); // this lane's copies of block B have landed
                } else {
                    stage(B, ybuf0);
                    atmb_cp_commit();
                    atmb_cp_wait<0>();
                }
                __syncwarp(); // ... and every lane's
                const float4 *yrow = ybuf0 + cur * bufq;
                const float4 *yA = yrow + ne * RQ * 32;
                const float4 *yB = yA + 32;
                {
                    // entries k and k + 1 side by side at slot k, for the packed visits
                    const float4 a0 = yA[lane], b0 = yB[lane];
                    const int nx = (lane + 1) & 31;
                    const float a1x = __shfl_sync(0xffffffffu, a0.x, nx), a1y = __shfl_sync(0xffffffffu, a0.y, nx);
                    const float a1z = __shfl_sync(0xffffffffu, a0.z, nx), a1w = __shfl_sync(0xffffffffu, a0.w, nx);
                    const float b1x = __shfl_sync(0xffffffffu, b0.x, nx), b1y = __shfl_sync(0xffffffffu, b0.y, nx);
                    const float b1z = __shfl_sync(0xffffffffu, b0.z, nx), b1w = __shfl_sync(0xffffffffu, b0.w, nx);
                    yP0[lane] = make_float4(a0.x, a1x, a0.y, a1y);
                    yP1[lane] = make_float4(a0.z, a1z, a0.w, a1w);
                    yQ0[lane] = make_float4(b0.x, b1x, b0.y, b1y);
                    yQ1[lane] = make_float4(b0.z, b1z, b0.w, b1w);
                }
                __syncwarp();
                AtmbXSums2<simple> xt{};    // x side of this block pair (two partial sums)
                AtmbYSums2<simple> ys[2]{}; // y sides of steps s + 2p (x) and s + 2p + 1 (y), travelling with their y
                const bool diag = (A == B);
                const int s1 = diag ? 17 : 32;
                const float4 *yrow_x = yrow + tx * RQ * 32; // rows at the x entry's type
                const float2 M1 = make_float2(-1.0f, -1.0f);
                int nv = 0;
                // off-diagonal block pairs take steps 0..31 with one range limit per lane
                // (rc_ATM^2, or -1 for a lane without entry); diagonal ones steps 1..16, where
                // step 16 is taken by lanes 0..15 only (lanes 16..31 would repeat its pairs)
                auto walk = [&](auto diag_c) {
                    constexpr bool DG = decltype(diag_c)::value;
                    const float lim = xvalid ? ratm2f : -1.0f;
                    const float lim16 = DG && lane >= 16 ? -1.0f : lim;
                    for (int s = DG ? 1 : 0; s < (DG ? 17 : 32); s += 4) {
                        // four independent visits per iteration (steps s .. s + 3) as two packed pairs
                        int kp[2];
                        float4 P0q[2], P1q[2];
                        float2 d3p[2];
                        bool a0q[2], a1q[2];
                        bool any = false;
#pragma unroll
                        for (int pq = 0; pq < 2; ++pq) {
                            kp[pq] = (lane + s + 2 * pq) & 31;
                            P0q[pq] = yP0[kp[pq]];
                            P1q[pq] = yP1[kp[pq]];
                            const float2 rx = __ffma2_rn(make_float2(P0q[pq].x, P0q[pq].y), M1, X.vx);
                            const float2 ry = __ffma2_rn(make_float2(P0q[pq].z, P0q[pq].w), M1, X.vy);
                            const float2 rz = __ffma2_rn(make_float2(P1q[pq].x, P1q[pq].y), M1, X.vz);
                            d3p[pq] = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __fmul2_rn(rz, rz)));
                            const int st = s + 2 * pq;
                            const float l0 = DG && st >= 16 ? lim16 : lim, l1 = DG && st + 1 >= 16 ? lim16 : lim;
                            a0q[pq] = d3p[pq].x <= l0 && d3p[pq].x >= 1e-12f;
                            a1q[pq] = d3p[pq].y <= l1 && d3p[pq].y >= 1e-12f;
                            any |= a0q[pq] | a1q[pq];
                            nv += (a0q[pq] ? 2 : 0) + (a1q[pq] ? 2 : 0);
                        }
                        if constexpr (FINE) {
#pragma unroll
                            for (int pq = 0; pq < 2; ++pq)
                                if (__any_sync(0xffffffffu, a0q[pq] | a1q[pq]))
                                    atmb_visit2<NR, simple>(X, kp[pq], d3p[pq], a0q[pq], a1q[pq], P0q[pq], P1q[pq], yQ0,
                                                            yQ1, yrow_x, a, third, force_scaled, xt, ys[pq]);
                        } else if (__any_sync(0xffffffffu, any)) {
#pragma unroll
                            for (int pq = 0; pq < 2; ++pq)
                                atmb_visit2<NR, simple>(X, kp[pq], d3p[pq], a0q[pq], a1q[pq], P0q[pq], P1q[pq], yQ0,
                                                        yQ1, yrow_x, a, third, force_scaled, xt, ys[pq]);
                        }
                        const int src = (lane + 4) & 31;
                        ys[0].shift(src);
                        ys[1].shift(src);
                    }
                };
                if (diag)
                    walk(std::true_type{});
                else
                    walk(std::false_type{});
                visits += (unsigned long long)nv;
                // lane L now holds the complete sums of y entry B[(L + s1 + q) mod 32] from the
                // visits of steps = q (mod 4) (q = 0, 1 in ys[0].x, .y; 2, 3 in ys[1].x, .y):
                // gather the entry B[(L + s1) mod 32]
                AtmbSide<simple> yg = ys[0].part(0);
                yg.add_from(ys[0].part(1), (lane - 1) & 31);
                yg.add_from(ys[1].part(0), (lane - 2) & 31);
                yg.add_from(ys[1].part(1), (lane - 3) & 31);
                yg.flush(acc, mcap, B * 32 + ((lane + s1) & 31), m); // padding partners carry zero sums
                xs[0] += xt.SE.x + xt.SE.y;
                xs[1] += xt.SD.x + xt.SD.y;
                xs[2] += xt.SF.x + xt.SF.y;
                xs[3] += xt.Wx.x + xt.Wx.y;
                xs[4] += xt.Wy.x + xt.Wy.y;
                xs[5] += xt.Wz.x + xt.Wz.y;
                if constexpr (!simple) {
                    xs[6] += xt.Ux.x + xt.Ux.y;
                    xs[7] += xt.Uy.x + xt.Uy.y;
                    xs[8] += xt.Uz.x + xt.Uz.y;
                    xsc += xt.SC.x + xt.SC.y;
                }
                B = Bn;
                if (NBUF == 2) cur ^= 1;
            }
            atmb_cp_wait<0>();
            if (xvalid) {
                // the x entry's force over this row: SF v_x - W
                const double SF = xs[2];
                atomicAdd(&acc[0 * mcap + xe], (float)xs[0]);
                atomicAdd(&acc[1 * mcap + xe], (float)xs[1]);
                atomicAdd(&acc[2 * mcap + xe], (float)(SF * vx - xs[3]));
                atomicAdd(&acc[3 * mcap + xe], (float)(SF * vy - xs[4]));
                atomicAdd(&acc[4 * mcap + xe], (float)(SF * vz - xs[5]));
                if constexpr (!simple) {
                    if (xsc != 0.f) atomicAdd(&acc[5 * mcap + xe], xsc);
                    // the x-y cross terms of the apex virial that the force weights miss
                    apx[0] -= 2.0 * vx * xs[6];
                    apx[1] -= 2.0 * vy * xs[7];
                    apx[2] -= 2.0 * vz * xs[8];
                    apx[3] -= vx * xs[7] + vy * xs[6];
                    apx[4] -= vx * xs[8] + vz * xs[6];
                    apx[5] -= vy * xs[8] + vz * xs[7];
                }
            }
            __syncwarp();
        }
        __syncthreads();
        // ---- 4. per entry: atom shares (FP64 atomics) and the apex's sums
        double ea = 0, ga = 0, af[3] = {0.0, 0.0, 0.0}, av[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) av[k] = apx[k];
        for (int e = tid; e < m; e += blockDim.x) {
            // accumulated at L2 by atomics: read past L1
            const double SE = __ldcg(&acc[e]), SD = __ldcg(&acc[mcap + e]);
            const double Fx = __ldcg(&acc[2 * mcap + e]), Fy = __ldcg(&acc[3 * mcap + e]);
            const double Fz = __ldcg(&acc[4 * mcap + e]);
            const float4 qa4 = sA[e], qj4 = sJ[e];
            const int j = __float_as_int(qj4.x);
            const double lam_ea = qj4.z, lam_ae = qj4.w;
            const double vx = qa4.x, vy = qa4.y, vz = qa4.z;
            atomicAdd(&p.eb[j], SE * (1.0 / 3.0));
            atomicAdd(&p.gb[j], 0.5 * (lam_ea * SE + SD));
            atomicAdd(&p.fb[3 * j], Fx);
            atomicAdd(&p.fb[3 * j + 1], Fy);
            atomicAdd(&p.fb[3 * j + 2], Fz);
            ea += SE * (1.0 / 6.0);
            ga += 0.5 * lam_ae * SE;
            // the apex takes minus the entries' forces (each triplet term depends on relative
            // positions only); the virial is sum v_e (x) F_e (symmetrised), plus in the
            // weighted form SC v_e (x) v_e for the visits whose energy and force weights differ
            af[0] -= Fx;
            af[1] -= Fy;
            af[2] -= Fz;
            const double SC = SIMPLE ? 0.0 : (double)__ldcg(&acc[5 * mcap + e]);
            av[0] += vx * fma(SC, vx, Fx);
            av[1] += vy * fma(SC, vy, Fy);
            av[2] += vz * fma(SC, vz, Fz);
            av[3] += 0.5 * (vx * Fy + vy * Fx) + SC * vx * vy;
            av[4] += 0.5 * (vx * Fz + vz * Fx) + SC * vx * vz;
            av[5] += 0.5 * (vy * Fz + vz * Fy) + SC * vy * vz;
        }
        const double vals[11] = {ea, ga, af[0], af[1], af[2], av[0], av[1], av[2], av[3], av[4], av[5]};
#pragma unroll
        for (int k = 0; k < 11; ++k) {
            const double v = warp_sum(vals[k]);
            if (lane == 0) red[warp][k] = v;
        }
        __syncthreads();
        if (tid == 0) {
            double tot[11];
            for (int k = 0; k < 11; ++k) {
                tot[k] = 0;
                for (int w2 = 0; w2 < nw; ++w2) tot[k] += red[w2][k];
            }
            const double sc = -1.0 / g.vol;
            if (S == 1) {
                p.ea[a] = tot[0];
                p.ga[a] = tot[1];
                p.fa[3 * a] = tot[2];
                p.fa[3 * a + 1] = tot[3];
                p.fa[3 * a + 2] = tot[4];
                for (int k = 0; k < 6; ++k) p.va[6 * (size_t)a + k] = tot[5 + k] * sc;
            } else { // the apex's other splits add theirs (the arrays start at zero)
                atomicAdd(&p.ea[a], tot[0]);
                atomicAdd(&p.ga[a], tot[1]);
                for (int k = 0; k < 3; ++k) atomicAdd(&p.fa[3 * a + k], tot[2 + k]);
                for (int k = 0; k < 6; ++k) atomicAdd(&p.va[6 * (size_t)a + k], tot[5 + k] * sc);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) visits += __shfl_xor_sync(0xffffffffu, visits, o);
    if ((tid & 31) == 0 && p.counters) atomicAdd(p.counters, visits);
}

// ATM three-body kernel, precision form, block-pair schedule: every triplet visited once.
// Included by d3_engine.cu after k_atm32 (same per-entry set-up, weights and outputs).
//
// Per apex a (persistent CTAs take apexes from a work counter, largest lists first):
//  1. The entries of the half list are counting-sorted by a Morton key of an 8^3 grid over
//     [-rc, rc]^3 around the apex, so 32 consecutive entries ("a block") are close in space.
//     Per-entry set-up (FP64 C6 of the apex pair, its CN derivatives, damping ratio) is
//     written once per apex, in sorted order, to this CTA's slot of a global scratch array.
//  2. Block pairs (A, B), B >= A, whose bounding boxes are within rc_ATM of each other are
//     walked by the warps (rows A in a zigzag over the warps). Lane L owns entry x = A[L];
//     at step s it pairs with y = B[(L + s) mod 32], so no two lanes of the warp touch the
//     same y in a step. Diagonal blocks take steps 1..16 (step 16 on lanes 0..15 only), so
//     every unordered pair of entries is visited exactly once.
//  3. x-side sums stay in the lane's registers for the whole row; y-side sums travel with
//     their y: a lane takes two steps per iteration (two independent visits, for ILP) and
//     then passes both sets of y sums two lanes down (six shuffles per step), so after the
//     last step lane L holds the complete sums of two y's and adds them to those entries'
//     accumulators in shared memory (one atomic per quantity per block pair).
//  4. Per entry e at the end: energy share SE/3, dE/dCN 0.5 (lam_ea SE + SD), force
//     SF v_e - W (FP64 atomics to the entry atom, as k_atm32); the apex gets SE/6,
//     0.5 lam_ae SE, the force -sum (wf f_e) v_e and the virial sum SF v_e (x) v_e minus the
//     cross terms (accumulated by the x lanes) plus the w != wf corrections.
// With f1, f2, f3 the force scalars of sides a-x, a-y, x-y of a triplet (mirror symmetry of
// k_atm: f2 of visit (x, y) is f1 of the mirrored visit), the quantities per entry are
//   SE = sum w E, SD = sum w E lam_{e,other}, SF = sum wf (f_e + f3), W = sum wf f3 v_other.
// C6_xy = Y_x[t_y] . w_y, dC6_xy/dCN_x = D_x[t_y] . w_y, dC6_xy/dCN_y = Y_x[t_y] . dw_y with
// the x entry's rows Y, D (all types) staged in shared memory once per row.
// Profile of the one-visit-per-step version on the 2,000-atom box (ncu): issue active 54 %,
// 21 of 32 lanes active per instruction, stalls dominated by fixed-latency dependencies and
// shared-memory/MUFU scoreboards with one 8-warp CTA per SM, and 3.5e9 shared bank conflicts
// from type-dependent row offsets; hence two visits per iteration and the transposed rows.

constexpr int ATMB_MCAP = 4096;   // longest list this kernel takes (longer lists: k_atm32)
constexpr int ATMB_GRID = 8;      // spatial grid per dimension for the entry sort
constexpr int ATMB_MAXW = 8;      // warps per CTA at most
constexpr int ATMB_VPI = 4;       // visits per lane per iteration (independent, for ILP)

// global scratch per CTA (float4 units): per-entry records sA, sB, sJ and the per-entry
// accumulators [6][MCAP] floats
constexpr size_t ATMB_SCRATCH_PER_CTA = 3 * ATMB_MCAP + (6 * ATMB_MCAP + 3) / 4;

// shared memory: fixed part + per-warp staging
__host__ __device__ inline size_t atmb_smem_fixed(int ne, int NR) {
    size_t b = ATMB_MCAP * sizeof(int);                       // atom of each sorted entry
    b += 2 * (ATMB_MCAP / 32) * sizeof(float4);               // block bounding boxes
    b += 512 * sizeof(int);                                   // sort cells
    b += (size_t)((ne * ne + 3) & ~3) * sizeof(float);        // r0^2
    b += (size_t)((ne * NR + 1) & ~1) * sizeof(double);       // apex C6 rows
    return (b + 15) & ~(size_t)15;
}
// per warp: two buffers (the block pair being visited and the next one, filled by
// cp.async meanwhile), each the staged y block: the rows of its entries for every partner
// type as float4 [type][row quad][lane] (lanes read consecutive 16-byte words whatever the
// x type, so the reads are free of bank conflicts) and positions / per-entry constants
__host__ __device__ inline size_t atmb_buf_quads(int ne, int NR) { return 32 * ((size_t)ne * (atmb_row_floats(NR) / 4) + 2); }
__host__ __device__ inline size_t atmb_smem_warp(int ne, int NR) { return 2 * atmb_buf_quads(ne, NR) * sizeof(float4); }

// 16-byte global -> shared copy that bypasses registers (cached in L2 only)
__device__ __forceinline__ void atmb_cp16(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void atmb_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's groups are still in flight
template <int N>
__device__ __forceinline__ void atmb_cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ int atmb_morton(int x, int y, int z) {
    int k = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b) k |= (((x >> b) & 1) << (3 * b)) | (((y >> b) & 1) << (3 * b + 1)) | (((z >> b) & 1) << (3 * b + 2));
    return k;
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

template <int NR>
__device__ __forceinline__ float atmb_dot(const float *r, const float *v) {
    float s = r[0] * v[0];
#pragma unroll
    for (int b = 1; b < NR; ++b) s = fmaf(r[b], v[b], s);
    return s;
}

// per-row constants of the x entry; gq carries the factor (4/3)^16, c1 = -0.75 d1,
// d1x3 = 3 d1; w, dw its own C6 weights and their CN derivatives
template <int NR>
struct AtmbX {
    float vx, vy, vz, d1, ir1, id1, sq, gq, c1, d1x3;
    float w[NR], dw[NR];
    int jx;
    bool qa;
};

// per-side sums of one block pair: SE = sum w E, SD = sum w E lam, SA = sum wf f_apex-side,
// S3 = sum wf f3, W = sum wf f3 v_other; the x side also U = sum w f3 v_y
// (force scalar of the entry SF = SA + S3)
struct AtmbSide {
    float SE, SD, SA, S3, Wx, Wy, Wz, Ux, Uy, Uz;
    __device__ __forceinline__ void shift(int src) {
        SE = __shfl_sync(0xffffffffu, SE, src);
        SD = __shfl_sync(0xffffffffu, SD, src);
        SA = __shfl_sync(0xffffffffu, SA, src);
        S3 = __shfl_sync(0xffffffffu, S3, src);
        Wx = __shfl_sync(0xffffffffu, Wx, src);
        Wy = __shfl_sync(0xffffffffu, Wy, src);
        Wz = __shfl_sync(0xffffffffu, Wz, src);
    }
    // add the y sums that lane src holds
    __device__ __forceinline__ void add_from(const AtmbSide &o, int src) {
        SE += __shfl_sync(0xffffffffu, o.SE, src);
        SD += __shfl_sync(0xffffffffu, o.SD, src);
        SA += __shfl_sync(0xffffffffu, o.SA, src);
        S3 += __shfl_sync(0xffffffffu, o.S3, src);
        Wx += __shfl_sync(0xffffffffu, o.Wx, src);
        Wy += __shfl_sync(0xffffffffu, o.Wy, src);
        Wz += __shfl_sync(0xffffffffu, o.Wz, src);
    }
    __device__ __forceinline__ void flush(float *acc, int e, int m) {
        if (e < m && (SE != 0.f || SA != 0.f || S3 != 0.f || SD != 0.f)) {
            atomicAdd(&acc[0 * ATMB_MCAP + e], SE);
            atomicAdd(&acc[1 * ATMB_MCAP + e], SD);
            atomicAdd(&acc[2 * ATMB_MCAP + e], SA + S3);
            atomicAdd(&acc[3 * ATMB_MCAP + e], Wx);
            atomicAdd(&acc[4 * ATMB_MCAP + e], Wy);
            atomicAdd(&acc[5 * ATMB_MCAP + e], Wz);
        }
    }
};

// One (possible) visit of entry x with staged partner k: triplet term, x-side sums into
// xt, y-side sums into ys, virial corrections where the virial and force weights differ.
// Branch-free: an out-of-range pair (act false) runs on finite stand-in values (lanes
// without entry and padding partners sit at far, distinct points with positive C6 rows)
// with zero weights, so the visits of an iteration can be interleaved by the compiler.
// With P = t1 t2 t3 (t1 = d1 + d2 - d3 ...), the angular term is
// A = (1 + 3/8 P / (d1 d2 d3)) / (r1 r2 r3)^3 and its side derivatives
// dA/dr_k / r_k = q52 G_k, G_k = 15/8 P + 3 d1 d2 d3 - 3/4 d_k (T - 2 t_ij),
// T = t12 + t13 + t23 (t_ij the product of the two t's without t_k).
template <int NR, bool SIMPLE>
__device__ __forceinline__ void atmb_visit(const AtmbX<NR> &X, int k, const float4 ya, float d3in, bool act,
                                           const float4 *yB, const float4 *yrow, int a, float third,
                                           bool force_scaled, AtmbSide &xt, AtmbSide &ys, double *apx) {
    const float d3 = act ? d3in : X.d1;
    const float4 yb = yB[k];
    AtmbRow<NR> R; // the y entry's rows at the x entry's type
    R.load(yrow, k);
    const float ir3 = rsqrtf(d3);
    const float id3 = ir3 * ir3;
    // C6_xy = Y_y[t_x] . w_x, its derivatives dw_x and through D_y[t_x] = dw_y C
    const float c6 = atmb_dot<NR>(R.Y, X.w);
    const float dcx = atmb_dot<NR>(R.Y, X.dw); // dC6_xy/dCN_x
    const float dcy = atmb_dot<NR>(R.D, X.w);  // dC6_xy/dCN_y
    const float is3 = rsqrtf(c6);
    const float s3 = c6 * is3;
    const float is3q = is3 * is3;
    const float lam_xy = dcx * is3q, lam_yx = dcy * is3q;
    const float u = R.r0sq * id3; // r0_xy^2 / d3
    const float g3 = exp2f(__log2f(u) * (8.0f / 3.0f)); // u^(8/3)
    // reference scale factors (src/d3_kernel.cu:1282-1290) as pair weights; SIMPLE: no
    // atom appears twice in the list (cell heights > 2 rc_ATM), every weight is 1
    float w, wf;
    if (SIMPLE) {
        w = wf = act ? 1.0f : 0.0f;
    } else {
        const int jy = R.j;
        const bool same = (X.jx == jy);
        const bool apex_img = X.qa | (jy == a);
        w = act ? (same ? (X.qa ? third : 1.0f) : (apex_img ? 0.5f : 1.0f)) : 0.0f;
        wf = act ? (force_scaled ? w : (same ? 2.0f : 1.0f)) : 0.0f;
    }
    const float d1 = X.d1, d2 = ya.w;
    const float irsq = X.id1 * yb.y * id3;
    const float ir9 = irsq * X.ir1 * yb.x * ir3;
    const float t1 = d1 + d2 - d3, t2 = d1 - d2 + d3, t3 = -d1 + d2 + d3;
    const float t12 = t1 * t2, t13 = t1 * t3, t23 = t2 * t3;
    const float P = t12 * t3;
    const float T = t12 + t13 + t23;
    const float Aang = fmaf(0.375f * P, irsq, 1.0f) * ir9;
    const float q52 = ir9 * irsq;
    const float base = fmaf(1.875f, P, X.d1x3 * d2 * d3);
    const float G1 = fmaf(X.c1, fmaf(-2.0f, t12, T), base);
    const float G2 = fmaf(-0.75f * d2, fmaf(-2.0f, t13, T), base);
    const float G3 = fmaf(-0.75f * d3, fmaf(-2.0f, t23, T), base);
    const float x16 = X.gq * yb.w * g3;
    const float fd = __fdividef(1.0f, fmaf(6.0f, x16, 1.0f));
    const float dfd = 32.0f * x16 * fd * fd;
    const float nC9 = X.sq * yb.z * s3; // -C9
    const float nC9fd = nC9 * fd;
    const float Et = -nC9fd * Aang;
    const float Ap = nC9fd * q52, Bp = nC9 * Aang * dfd;
    const float f1 = fmaf(Ap, G1, -Bp) * X.id1;
    const float f2 = fmaf(Ap, G2, -Bp) * yb.y;
    const float f3 = fmaf(Ap, G3, -Bp) * id3;
    const float wE = w * Et;
    const float wf3 = wf * f3;
    xt.SE += wE;
    xt.SD = fmaf(wE, lam_xy, xt.SD);
    xt.SA = fmaf(wf, f1, xt.SA);
    xt.S3 += wf3;
    xt.Wx = fmaf(wf3, ya.x, xt.Wx);
    xt.Wy = fmaf(wf3, ya.y, xt.Wy);
    xt.Wz = fmaf(wf3, ya.z, xt.Wz);
    if (!SIMPLE) { // SIMPLE: U = W
        const float w3 = w * f3;
        xt.Ux = fmaf(w3, ya.x, xt.Ux);
        xt.Uy = fmaf(w3, ya.y, xt.Uy);
        xt.Uz = fmaf(w3, ya.z, xt.Uz);
    }
    ys.SE += wE;
    ys.SD = fmaf(wE, lam_yx, ys.SD);
    ys.SA = fmaf(wf, f2, ys.SA);
    ys.S3 += wf3;
    ys.Wx = fmaf(wf3, X.vx, ys.Wx);
    ys.Wy = fmaf(wf3, X.vy, ys.Wy);
    ys.Wz = fmaf(wf3, X.vz, ys.Wz);
    if (!SIMPLE && w != wf) {
        // virial weights w where the force weights differ (repeated indices)
        const double c1 = (double)(w - wf) * (double)(f1 + f3), c2 = (double)(w - wf) * (double)(f2 + f3);
        apx[3] += c1 * X.vx * X.vx + c2 * ya.x * ya.x;
        apx[4] += c1 * X.vy * X.vy + c2 * ya.y * ya.y;
        apx[5] += c1 * X.vz * X.vz + c2 * ya.z * ya.z;
        apx[6] += c1 * X.vx * X.vy + c2 * ya.x * ya.y;
        apx[7] += c1 * X.vx * X.vz + c2 * ya.x * ya.z;
        apx[8] += c1 * X.vy * X.vz + c2 * ya.y * ya.z;
    }
}

template <int NR>
__global__ void __launch_bounds__(ATMB_MAXW * 32, 1) k_atm32b(KP p, float4 *scratch) {
    extern __shared__ __align__(16) unsigned char smb[];
    const int ne = p.ne;
    const int nw = blockDim.x >> 5;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int *sjy = reinterpret_cast<int *>(smb);                             // [MCAP] atom of each sorted entry
    float4 *bblo = reinterpret_cast<float4 *>(sjy + ATMB_MCAP);          // [MCAP/32]
    float4 *bbhi = bblo + ATMB_MCAP / 32;
    int *cellpos = reinterpret_cast<int *>(bbhi + ATMB_MCAP / 32);       // [512]
    float *r0sq = reinterpret_cast<float *>(cellpos + 512);              // [ne][ne]
    double *yapex = reinterpret_cast<double *>(r0sq + ((ne * ne + 3) & ~3)); // [ne][NR]
    unsigned char *wbase = smb + atmb_smem_fixed(ne, NR) + (size_t)warp * atmb_smem_warp(ne, NR);
    constexpr int RQ = atmb_row_floats(NR) / 4;                          // float4 quads per row
    // buffer layout: [ne][RQ][32] rows of the y block, [32] vx vy vz d2, [32] ir id2 s g
    float4 *ybuf0 = reinterpret_cast<float4 *>(wbase);
    const size_t bufq = atmb_buf_quads(ne, NR);
    __shared__ int s_item;
    __shared__ double red[ATMB_MAXW][12];
    float4 *sA = scratch + (size_t)blockIdx.x * ATMB_SCRATCH_PER_CTA;    // vx vy vz d2
    float4 *sB = sA + ATMB_MCAP;                                         // ir id2 s g
    float4 *sJ = sB + ATMB_MCAP;                                         // j t lam_ea lam_ae
    float *acc = reinterpret_cast<float *>(sJ + ATMB_MCAP);              // [6][MCAP] (global, L2-resident)
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
        const int item = s_item * p.shard_world + p.shard_rank;
        if (item >= p.n) break;
        const int a = p.sorted_of[p.n - 1 - item];
        const long long e0 = p.atm_off[a];
        const int m = (int)(p.atm_off[a + 1] - e0);
        if (m > ATMB_MCAP) continue; // long lists: k_atm32
        const double4 xa = p.xs[a];
        const int ta = (int)xa.w;
        const SG &g = p.sg[p.sid[a]];
        const bool simple = g.atm_simple != 0;
        for (int k = tid; k < ne * NR; k += blockDim.x) yapex[k] = p.Y[(size_t)a * ne * NR + k];
        for (int k = tid; k < 512; k += blockDim.x) cellpos[k] = 0;
        for (int q = 0; q < 6; ++q)
            for (int e = tid; e < m; e += blockDim.x) __stcg(&acc[q * ATMB_MCAP + e], 0.f);
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
            atomicAdd(&cellpos[atmb_morton(cx, cy, cz)], 1);
        }
        __syncthreads();
        if (warp == 0) {
            int c[16], s = 0;
#pragma unroll
            for (int t = 0; t < 16; ++t) {
                c[t] = cellpos[lane * 16 + t];
                s += c[t];
            }
            int incl = s;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            int run = incl - s;
#pragma unroll
            for (int t = 0; t < 16; ++t) {
                cellpos[lane * 16 + t] = run;
                run += c[t];
            }
        }
        __syncthreads();
        for (int k = tid; k < m; k += blockDim.x) {
            const int2 ent = p.atm_ent[e0 + k];
            const int jp = ent.x;
            const double4 xj = p.xs[jp];
            const int tp = (int)xj.w;
            double sx, sy, sz;
            image_vec(g, sext8(ent.y & 0xff), sext8((ent.y >> 8) & 0xff), sext8((ent.y >> 16) & 0xff), sx, sy, sz);
            const double vx = xj.x + sx - xa.x, vy = xj.y + sy - xa.y, vz = xj.z + sz - xa.z;
            const int cx = min(ATMB_GRID - 1, max(0, (int)((vx + rc) * cinv)));
            const int cy = min(ATMB_GRID - 1, max(0, (int)((vy + rc) * cinv)));
            const int cz = min(ATMB_GRID - 1, max(0, (int)((vz + rc) * cinv)));
            const int pos = atomicAdd(&cellpos[atmb_morton(cx, cy, cz)], 1);
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
            sjy[pos] = jp;
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
        double apx[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}; // apex force (3) and virial (6) of this lane
        for (int r = 0;; ++r) {
            const int A = nw * r + ((r & 1) ? (nw - 1 - warp) : warp);
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
            double xs[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0}; // SE SD SF Wx Wy Wz SA Ux Uy Uz (row carries)
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
            __syncwarp(); // the previous row's visits are done with both buffers
            if (B < nb) stage(B, ybuf0);
            atmb_cp_commit();
            while (B < nb) {
                const int Bn = next_near(B + 1);
                __syncwarp(); // every lane is done with the other buffer
                if (Bn < nb) stage(Bn, ybuf0 + (cur ^ 1) * bufq);
                atmb_cp_commit();
                atmb_cp_wait<1>(); // this lane's copies of block B have landed
                __syncwarp();      // ... and every lane's
                const float4 *yrow = ybuf0 + cur * bufq;
                const float4 *yA = yrow + ne * RQ * 32;
                const float4 *yB = yA + 32;
                AtmbSide xt{}; // x side of this block pair
                AtmbSide ys[ATMB_VPI]; // y sides, travelling with their y (ATMB_VPI steps per iteration)
#pragma unroll
                for (int q = 0; q < ATMB_VPI; ++q) ys[q] = AtmbSide{};
                const bool diag = (A == B);
                const int s0 = diag ? 1 : 0, s1 = diag ? 17 : 32;
                AtmbX<NR> X;
                X.vx = vx;
                X.vy = vy;
                X.vz = vz;
                X.d1 = d1;
                X.ir1 = ir1;
                X.id1 = id1;
                X.sq = sq;
                X.gq = gq;
                X.c1 = -0.75f * d1;
                X.d1x3 = 3.0f * d1;
#pragma unroll
                for (int b = 0; b < NR; ++b) {
                    X.w[b] = wx[b];
                    X.dw[b] = dwx[b];
                }
                X.jx = jx;
                X.qa = qa;
                const float4 *yrow_x = yrow + tx * RQ * 32; // rows at the x entry's type
                int nv = 0;
                for (int s = s0; s < s1; s += ATMB_VPI) {
                    // ATMB_VPI independent visits per iteration (steps s .. s + ATMB_VPI - 1) for ILP
                    int kq[ATMB_VPI];
                    float4 yq[ATMB_VPI];
                    float d3q[ATMB_VPI];
                    bool aq[ATMB_VPI];
                    bool any = false;
#pragma unroll
                    for (int q = 0; q < ATMB_VPI; ++q) {
                        kq[q] = (lane + s + q) & 31;
                        yq[q] = yA[kq[q]];
                        const float rx = vx - yq[q].x, ry = vy - yq[q].y, rz = vz - yq[q].z;
                        d3q[q] = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
                        aq[q] = xvalid && (!diag || s + q < 16 || lane < 16) && d3q[q] <= ratm2f && d3q[q] >= 1e-12f;
                        any |= aq[q];
                        nv += aq[q] ? 2 : 0;
                    }
                    if (__any_sync(0xffffffffu, any)) {
                        if (simple) {
#pragma unroll
                            for (int q = 0; q < ATMB_VPI; ++q)
                                atmb_visit<NR, true>(X, kq[q], yq[q], d3q[q], aq[q], yB, yrow_x, a, third,
                                                     force_scaled, xt, ys[q], apx);
                        } else {
#pragma unroll
                            for (int q = 0; q < ATMB_VPI; ++q)
                                atmb_visit<NR, false>(X, kq[q], yq[q], d3q[q], aq[q], yB, yrow_x, a, third,
                                                      force_scaled, xt, ys[q], apx);
                        }
                    }
                    const int src = (lane + ATMB_VPI) & 31;
#pragma unroll
                    for (int q = 0; q < ATMB_VPI; ++q) ys[q].shift(src);
                }
                visits += (unsigned long long)nv;
                // lane L now holds in ys[q] the complete sums of y entry B[(L + s1 + q) mod 32]
                // from the visits of step parity q: gather the entry B[(L + s1) mod 32] in ys[0]
#pragma unroll
                for (int q = 1; q < ATMB_VPI; ++q) ys[0].add_from(ys[q], (lane - q) & 31);
                {
                    const int ey = (lane + s1) & 31;
                    ys[0].flush(acc, B * 32 + ey, m);
                    // apex force of the a-y sides (padding partners carry zero sums)
                    const float4 vyv = yA[ey];
                    apx[0] -= (double)(ys[0].SA * vyv.x);
                    apx[1] -= (double)(ys[0].SA * vyv.y);
                    apx[2] -= (double)(ys[0].SA * vyv.z);
                }
                const float tSE = xt.SE, tSD = xt.SD, tSF = xt.SA + xt.S3, tWx = xt.Wx, tWy = xt.Wy, tWz = xt.Wz, tSA = xt.SA;
                const float tUx = simple ? xt.Wx : xt.Ux, tUy = simple ? xt.Wy : xt.Uy, tUz = simple ? xt.Wz : xt.Uz;
                xs[0] += tSE;
                xs[1] += tSD;
                xs[2] += tSF;
                xs[3] += tWx;
                xs[4] += tWy;
                xs[5] += tWz;
                xs[6] += tSA;
                xs[7] += tUx;
                xs[8] += tUy;
                xs[9] += tUz;
                B = Bn;
                cur ^= 1;
            }
            atmb_cp_wait<0>();
            if (xvalid) {
                atomicAdd(&acc[0 * ATMB_MCAP + xe], (float)xs[0]);
                atomicAdd(&acc[1 * ATMB_MCAP + xe], (float)xs[1]);
                atomicAdd(&acc[2 * ATMB_MCAP + xe], (float)xs[2]);
                atomicAdd(&acc[3 * ATMB_MCAP + xe], (float)xs[3]);
                atomicAdd(&acc[4 * ATMB_MCAP + xe], (float)xs[4]);
                atomicAdd(&acc[5 * ATMB_MCAP + xe], (float)xs[5]);
                // apex force of the a-x sides and the x-y cross terms of the virial
                apx[0] -= xs[6] * vx;
                apx[1] -= xs[6] * vy;
                apx[2] -= xs[6] * vz;
                apx[3] -= 2.0 * vx * xs[7];
                apx[4] -= 2.0 * vy * xs[8];
                apx[5] -= 2.0 * vz * xs[9];
                apx[6] -= vx * xs[8] + vy * xs[7];
                apx[7] -= vx * xs[9] + vz * xs[7];
                apx[8] -= vy * xs[9] + vz * xs[8];
            }
            __syncwarp();
        }
        __syncthreads();
        // ---- 4. per entry: atom shares (FP64 atomics) and the apex's sums
        double ea = 0, ga = 0;
        for (int e = tid; e < m; e += blockDim.x) {
            // accumulated at L2 by atomics: read past L1
            const double SE = __ldcg(&acc[e]), SD = __ldcg(&acc[ATMB_MCAP + e]), SF = __ldcg(&acc[2 * ATMB_MCAP + e]);
            const double Wx = __ldcg(&acc[3 * ATMB_MCAP + e]), Wy = __ldcg(&acc[4 * ATMB_MCAP + e]);
            const double Wz = __ldcg(&acc[5 * ATMB_MCAP + e]);
            const float4 qa4 = sA[e], qj4 = sJ[e];
            const int j = __float_as_int(qj4.x);
            const double lam_ea = qj4.z, lam_ae = qj4.w;
            const double vx = qa4.x, vy = qa4.y, vz = qa4.z;
            atomicAdd(&p.eb[j], SE * (1.0 / 3.0));
            atomicAdd(&p.gb[j], 0.5 * (lam_ea * SE + SD));
            atomicAdd(&p.fb[3 * j], SF * vx - Wx);
            atomicAdd(&p.fb[3 * j + 1], SF * vy - Wy);
            atomicAdd(&p.fb[3 * j + 2], SF * vz - Wz);
            ea += SE * (1.0 / 6.0);
            ga += 0.5 * lam_ae * SE;
            apx[3] += SF * vx * vx;
            apx[4] += SF * vy * vy;
            apx[5] += SF * vz * vz;
            apx[6] += SF * vx * vy;
            apx[7] += SF * vx * vz;
            apx[8] += SF * vy * vz;
        }
        const double vals[11] = {ea, ga, apx[0], apx[1], apx[2], apx[3], apx[4], apx[5], apx[6], apx[7], apx[8]};
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
            p.ea[a] = tot[0];
            p.ga[a] = tot[1];
            p.fa[3 * a] = tot[2];
            p.fa[3 * a + 1] = tot[3];
            p.fa[3 * a + 2] = tot[4];
            const double sc = -1.0 / g.vol;
            for (int k = 0; k < 6; ++k) p.va[6 * (size_t)a + k] = tot[5 + k] * sc;
        }
    }
    for (int o = 16; o > 0; o >>= 1) visits += __shfl_xor_sync(0xffffffffu, visits, o);
    if ((tid & 31) == 0 && p.counters) atomicAdd(p.counters, visits);
}

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

// shared memory: fixed part + per-warp staging
__host__ __device__ inline size_t atmb_smem_fixed(int ne, int NR) {
    size_t b = 6 * ATMB_MCAP * sizeof(float);                 // per-entry accumulators
    b += 2 * (ATMB_MCAP / 32) * sizeof(float4);               // block bounding boxes
    b += 512 * sizeof(int);                                   // sort cells
    b += (size_t)((ne * ne + 3) & ~3) * sizeof(float);        // r0^2
    b += (size_t)((ne * NR + 1) & ~1) * sizeof(double);       // apex C6 rows
    return (b + 15) & ~(size_t)15;
}
// per warp: the x entries' C6 rows and derivative rows, float2 [type][8][lane] (lanes read
// consecutive 8-byte words whatever the partner type, so the reads are free of bank
// conflicts), and the staged y block as seven float4 arrays [lane]
__host__ __device__ inline size_t atmb_smem_warp(int ne) {
    return 32 * ((size_t)ne * 8 * sizeof(float2) + 7 * sizeof(float4));
}

__device__ __forceinline__ int atmb_morton(int x, int y, int z) {
    int k = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b) k |= (((x >> b) & 1) << (3 * b)) | (((y >> b) & 1) << (3 * b + 1)) | (((z >> b) & 1) << (3 * b + 2));
    return k;
}

// sum_b r[b] v[b] over the NR references: r as four float2 (8 floats), v as two float4
template <int NR>
__device__ __forceinline__ float atmb_dot(const float2 r0, const float2 r1, const float2 r2, const float2 r3,
                                          const float4 v0, const float4 v1) {
    float s = r0.x * v0.x;
    s = fmaf(r0.y, v0.y, s);
    s = fmaf(r1.x, v0.z, s);
    s = fmaf(r1.y, v0.w, s);
    s = fmaf(r2.x, v1.x, s);
    if (NR > 5) {
        s = fmaf(r2.y, v1.y, s);
        s = fmaf(r3.x, v1.z, s);
    }
    return s;
}

struct AtmbX {
    float vx, vy, vz, d1, ir1, id1, sq, gq;
    int jx, tx;
    bool qa, valid;
};

// per-side sums of one block pair: SE = sum w E, SD = sum w E lam, SF = sum wf (f_e + f3),
// W = sum wf f3 v_other; the x side also SA = sum wf f1 and U = sum w f3 v_y
struct AtmbSide {
    float SE, SD, SF, Wx, Wy, Wz, SA, Ux, Uy, Uz;
    __device__ __forceinline__ void shift(int src) {
        SE = __shfl_sync(0xffffffffu, SE, src);
        SD = __shfl_sync(0xffffffffu, SD, src);
        SF = __shfl_sync(0xffffffffu, SF, src);
        Wx = __shfl_sync(0xffffffffu, Wx, src);
        Wy = __shfl_sync(0xffffffffu, Wy, src);
        Wz = __shfl_sync(0xffffffffu, Wz, src);
    }
    __device__ __forceinline__ void flush(float *acc, int e, int m) {
        if (e < m && (SE != 0.f || SF != 0.f || SD != 0.f)) {
            atomicAdd(&acc[0 * ATMB_MCAP + e], SE);
            atomicAdd(&acc[1 * ATMB_MCAP + e], SD);
            atomicAdd(&acc[2 * ATMB_MCAP + e], SF);
            atomicAdd(&acc[3 * ATMB_MCAP + e], Wx);
            atomicAdd(&acc[4 * ATMB_MCAP + e], Wy);
            atomicAdd(&acc[5 * ATMB_MCAP + e], Wz);
        }
    }
};

// One (possible) visit of entry x with staged partner k: range test, triplet term,
// x-side sums into xt, y-side sums into ys, apex force of the a-y side, virial
// corrections where the virial and force weights differ.
// Branch-free: an out-of-range pair (act false) runs on safe stand-in values with zero
// weights, so the two visits of an iteration can be interleaved by the compiler.
template <int NR, bool SIMPLE>
__device__ __forceinline__ void atmb_visit(const AtmbX &X, int k, const float4 ya, float d3in, bool act,
                                           const float4 *yB, const int4 *yJ, const float4 *yW0, const float4 *yW1,
                                           const float4 *yD0, const float4 *yD1, const float2 *xrow, int lane,
                                           const float *r0sq, int ne, int a, float x16c, float third, bool force_scaled,
                                           AtmbSide &xt, AtmbSide &ys, float &aFx, float &aFy, float &aFz,
                                           double *apx) {
    const float d3 = act ? d3in : X.d1;
    const float4 yb = yB[k];
    const int4 yj = yJ[k];
    const int ty = yj.y;
    const float ir3 = rsqrtf(d3);
    const float id3 = ir3 * ir3;
    const float2 *xr = xrow + ty * 8 * 32 + lane;
    const float2 Ya = xr[0], Yb = xr[32], Yc = xr[64], Yd = xr[96];
    const float2 Da = xr[128], Db = xr[160], Dc = xr[192], Dd = xr[224];
    const float4 W0 = yW0[k], W1 = yW1[k], V0 = yD0[k], V1 = yD1[k];
    const float c6 = act ? atmb_dot<NR>(Ya, Yb, Yc, Yd, W0, W1) : 1.0f;
    const float dcx = atmb_dot<NR>(Da, Db, Dc, Dd, W0, W1); // dC6_xy/dCN_x
    const float dcy = atmb_dot<NR>(Ya, Yb, Yc, Yd, V0, V1); // dC6_xy/dCN_y
    const float is3 = rsqrtf(c6);
    const float s3 = c6 * is3;
    const float lam_xy = act ? dcx * is3 * is3 : 0.0f, lam_yx = act ? dcy * is3 * is3 : 0.0f;
    const float u = r0sq[X.tx * ne + ty] * id3;
    const float g3 = exp2f(__log2f(u) * (8.0f / 3.0f)); // u^(8/3)
    // reference scale factors (src/d3_kernel.cu:1282-1290) as pair weights; SIMPLE: no
    // atom appears twice in the list (cell heights > 2 rc_ATM), every weight is 1
    float w, wf;
    if (SIMPLE) {
        w = wf = act ? 1.0f : 0.0f;
    } else {
        const bool same = (X.jx == yj.x);
        const bool apex_img = X.qa | (yj.x == a);
        w = act ? (same ? (X.qa ? third : 1.0f) : (apex_img ? 0.5f : 1.0f)) : 0.0f;
        wf = act ? (force_scaled ? w : (same ? 2.0f : 1.0f)) : 0.0f;
    }
    const float d1 = X.d1, d2 = act ? ya.w : X.d1;
    const float irsq = X.id1 * yb.y * id3;
    const float ir9 = irsq * X.ir1 * yb.x * ir3;
    const float t1 = d1 + d2 - d3, t2 = d1 - d2 + d3, t3 = -d1 + d2 + d3;
    const float t12 = t1 * t2, t13 = t1 * t3, t23 = t2 * t3;
    const float P = t12 * t3;
    const float Aang = fmaf(0.375f * P, irsq, 1.0f) * ir9;
    const float q52 = ir9 * irsq;
    const float base = fmaf(1.875f, P, 3.0f * d1 * d2 * d3);
    const float dang1 = q52 * fmaf(-0.75f * d1, t23 + t13 - t12, base);
    const float dang2 = q52 * fmaf(-0.75f * d2, t23 - t13 + t12, base);
    const float dang3 = q52 * fmaf(-0.75f * d3, t13 + t12 - t23, base);
    const float x16 = act ? x16c * X.gq * yb.w * g3 : 0.0f;
    const float fd = __fdividef(1.0f, fmaf(6.0f, x16, 1.0f));
    const float dfd = 32.0f * x16 * fd * fd;
    const float C9 = -X.sq * yb.z * s3;
    const float Et = C9 * Aang * fd;
    const float Adfd = Aang * dfd;
    const float f1 = -C9 * fmaf(dang1, fd, -Adfd) * X.id1;
    const float f2 = -C9 * fmaf(dang2, fd, -Adfd) * yb.y;
    const float f3 = -C9 * fmaf(dang3, fd, -Adfd) * id3;
    const float wE = w * Et;
    const float wf3 = wf * f3, w3 = w * f3;
    xt.SE += wE;
    xt.SD = fmaf(wE, lam_xy, xt.SD);
    xt.SF = fmaf(wf, f1 + f3, xt.SF);
    xt.Wx = fmaf(wf3, ya.x, xt.Wx);
    xt.Wy = fmaf(wf3, ya.y, xt.Wy);
    xt.Wz = fmaf(wf3, ya.z, xt.Wz);
    xt.SA = fmaf(wf, f1, xt.SA);
    if (!SIMPLE) { // SIMPLE: U = W
        xt.Ux = fmaf(w3, ya.x, xt.Ux);
        xt.Uy = fmaf(w3, ya.y, xt.Uy);
        xt.Uz = fmaf(w3, ya.z, xt.Uz);
    }
    ys.SE += wE;
    ys.SD = fmaf(wE, lam_yx, ys.SD);
    ys.SF = fmaf(wf, f2 + f3, ys.SF);
    ys.Wx = fmaf(wf3, X.vx, ys.Wx);
    ys.Wy = fmaf(wf3, X.vy, ys.Wy);
    ys.Wz = fmaf(wf3, X.vz, ys.Wz);
    const float wf2 = wf * f2;
    aFx = fmaf(wf2, ya.x, aFx);
    aFy = fmaf(wf2, ya.y, aFy);
    aFz = fmaf(wf2, ya.z, aFz);
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
    float *acc = reinterpret_cast<float *>(smb);                         // [6][MCAP]
    float4 *bblo = reinterpret_cast<float4 *>(acc + 6 * ATMB_MCAP);      // [MCAP/32]
    float4 *bbhi = bblo + ATMB_MCAP / 32;
    int *cellpos = reinterpret_cast<int *>(bbhi + ATMB_MCAP / 32);       // [512]
    float *r0sq = reinterpret_cast<float *>(cellpos + 512);              // [ne][ne]
    double *yapex = reinterpret_cast<double *>(r0sq + ((ne * ne + 3) & ~3)); // [ne][NR]
    unsigned char *wbase = smb + atmb_smem_fixed(ne, NR) + (size_t)warp * atmb_smem_warp(ne);
    float2 *xrow = reinterpret_cast<float2 *>(wbase);                    // [ne][8][32]: Y (4 pairs) D (4 pairs)
    float4 *yA = reinterpret_cast<float4 *>(xrow + ne * 8 * 32);         // [32] vx vy vz d2
    float4 *yB = yA + 32;                                                // [32] ir id2 s g
    int4 *yJ = reinterpret_cast<int4 *>(yB + 32);                        // [32] j t
    float4 *yW0 = reinterpret_cast<float4 *>(yJ + 32);                   // [32] w[0..3]
    float4 *yW1 = yW0 + 32;                                              // [32] w[4..7] (zero padded)
    float4 *yD0 = yW1 + 32;                                              // [32] dw[0..3]
    float4 *yD1 = yD0 + 32;                                              // [32] dw[4..7]
    __shared__ int s_item;
    __shared__ double red[ATMB_MAXW][12];
    float4 *sA = scratch + (size_t)blockIdx.x * 3 * ATMB_MCAP;           // vx vy vz d2
    float4 *sB = sA + ATMB_MCAP;                                         // ir id2 s g
    float4 *sJ = sB + ATMB_MCAP;                                         // j t lam_ea lam_ae
    if (p.atm_off[p.n] > p.atm_cap) return; // list overflowed: the host grows it and re-runs
    for (int k = tid; k < ne * ne; k += blockDim.x) r0sq[k] = (float)(p.r0ab[k] * p.r0ab[k]);
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
            for (int e = tid; e < m; e += blockDim.x) acc[q * ATMB_MCAP + e] = 0.f;
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
            float vx = 1e30f, vy = 1e30f, vz = 1e30f, d1 = 1.f, ir1 = 1.f, id1 = 1.f, sq = 0.f, gq = 0.f;
            int jx = -1, tx = 0;
            if (xvalid) {
                const float4 qa4 = sA[xe], qb4 = sB[xe], qj4 = sJ[xe];
                vx = qa4.x;
                vy = qa4.y;
                vz = qa4.z;
                d1 = qa4.w;
                ir1 = qb4.x;
                id1 = qb4.y;
                sq = qb4.z;
                gq = qb4.w;
                jx = __float_as_int(qj4.x);
                tx = __float_as_int(qj4.y);
                // the entry's C6 rows and their CN derivatives for every type
                for (int t = 0; t < ne; ++t) {
                    const float *ys = p.Y32 + ((size_t)jx * ne + t) * NR;
                    const float *ds = p.D32 + ((size_t)jx * ne + t) * NR;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        xrow[(t * 8 + q) * 32 + lane] =
                            make_float2(2 * q < NR ? ys[2 * q] : 0.f, 2 * q + 1 < NR ? ys[2 * q + 1] : 0.f);
                        xrow[(t * 8 + 4 + q) * 32 + lane] =
                            make_float2(2 * q < NR ? ds[2 * q] : 0.f, 2 * q + 1 < NR ? ds[2 * q + 1] : 0.f);
                    }
                }
            } else {
                // rows of a lane without entry stay finite (its visits run with zero weights)
                for (int t = 0; t < ne * 8; ++t) xrow[t * 32 + lane] = make_float2(0.f, 0.f);
            }
            const bool qa = (jx == a);
            double xs[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0}; // SE SD SF Wx Wy Wz SA Ux Uy Uz (row carries)
            for (int B = A; B < nb; ++B) {
                {
                    const float4 la = bblo[A], ha = bbhi[A], lb = bblo[B], hb = bbhi[B];
                    const float dx = fmaxf(0.f, fmaxf(la.x - hb.x, lb.x - ha.x));
                    const float dy = fmaxf(0.f, fmaxf(la.y - hb.y, lb.y - ha.y));
                    const float dz = fmaxf(0.f, fmaxf(la.z - hb.z, lb.z - ha.z));
                    if (fmaf(dx, dx, fmaf(dy, dy, dz * dz)) > ratm2f * 1.0001f) continue;
                }
                __syncwarp();
                {
                    const int ye = B * 32 + lane;
                    if (ye < m) {
                        yA[lane] = sA[ye];
                        yB[lane] = sB[ye];
                        const float4 qj4 = sJ[ye];
                        const int jy = __float_as_int(qj4.x);
                        yJ[lane] = make_int4(jy, __float_as_int(qj4.y), 0, 0);
                        float wv[8], dv[8];
#pragma unroll
                        for (int b = 0; b < 8; ++b) {
                            wv[b] = b < NR ? p.w32[(size_t)jy * NR + b] : 0.f;
                            dv[b] = b < NR ? p.dw32[(size_t)jy * NR + b] : 0.f;
                        }
                        yW0[lane] = make_float4(wv[0], wv[1], wv[2], wv[3]);
                        yW1[lane] = make_float4(wv[4], wv[5], wv[6], wv[7]);
                        yD0[lane] = make_float4(dv[0], dv[1], dv[2], dv[3]);
                        yD1[lane] = make_float4(dv[4], dv[5], dv[6], dv[7]);
                    } else {
                        // far-away dummy: fails every distance test
                        yA[lane] = make_float4(1e30f, 1e30f, 1e30f, 1.f);
                        yB[lane] = make_float4(1.f, 1.f, 0.f, 0.f);
                        yJ[lane] = make_int4(-1, 0, 0, 0);
                        yW0[lane] = yW1[lane] = yD0[lane] = yD1[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                }
                __syncwarp();
                AtmbSide xt{};     // x side of this block pair
                AtmbSide y0{}, y1{}; // y sides, travelling with their y (two steps per iteration)
                float aFx = 0.f, aFy = 0.f, aFz = 0.f; // apex force, a-y sides
                const bool diag = (A == B);
                const int s0 = diag ? 1 : 0, s1 = diag ? 17 : 32;
                const AtmbX X{vx, vy, vz, d1, ir1, id1, sq, gq, jx, tx, qa, xvalid};
                for (int s = s0; s < s1; s += 2) {
                    // two independent visits per iteration (steps s and s + 1) for ILP
                    const int k0 = (lane + s) & 31, k1 = (lane + s + 1) & 31;
                    const float4 ya0 = yA[k0], ya1 = yA[k1];
                    float rx = vx - ya0.x, ry = vy - ya0.y, rz = vz - ya0.z;
                    const float d30 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
                    rx = vx - ya1.x;
                    ry = vy - ya1.y;
                    rz = vz - ya1.z;
                    const float d31 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
                    const bool act0 = xvalid && (!diag || s < 16 || lane < 16) && d30 <= ratm2f && d30 >= 1e-12f;
                    const bool act1 = xvalid && (!diag || s + 1 < 16 || lane < 16) && d31 <= ratm2f && d31 >= 1e-12f;
                    if (__any_sync(0xffffffffu, act0 || act1)) {
                        visits += (act0 ? 2 : 0) + (act1 ? 2 : 0);
                        if (simple) {
                            atmb_visit<NR, true>(X, k0, ya0, d30, act0, yB, yJ, yW0, yW1, yD0, yD1, xrow, lane, r0sq,
                                                 ne, a, x16c, third, force_scaled, xt, y0, aFx, aFy, aFz, apx);
                            atmb_visit<NR, true>(X, k1, ya1, d31, act1, yB, yJ, yW0, yW1, yD0, yD1, xrow, lane, r0sq,
                                                 ne, a, x16c, third, force_scaled, xt, y1, aFx, aFy, aFz, apx);
                        } else {
                            atmb_visit<NR, false>(X, k0, ya0, d30, act0, yB, yJ, yW0, yW1, yD0, yD1, xrow, lane, r0sq,
                                                  ne, a, x16c, third, force_scaled, xt, y0, aFx, aFy, aFz, apx);
                            atmb_visit<NR, false>(X, k1, ya1, d31, act1, yB, yJ, yW0, yW1, yD0, yD1, xrow, lane, r0sq,
                                                  ne, a, x16c, third, force_scaled, xt, y1, aFx, aFy, aFz, apx);
                        }
                    }
                    const int src = (lane + 2) & 31;
                    y0.shift(src);
                    y1.shift(src);
                }
                // lanes now hold the complete sums of y entries B[(lane + s1) mod 32] and
                // B[(lane + s1 + 1) mod 32]
                y0.flush(acc, B * 32 + ((lane + s1) & 31), m);
                y1.flush(acc, B * 32 + ((lane + s1 + 1) & 31), m);
                const float tSE = xt.SE, tSD = xt.SD, tSF = xt.SF, tWx = xt.Wx, tWy = xt.Wy, tWz = xt.Wz, tSA = xt.SA;
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
                apx[0] -= aFx;
                apx[1] -= aFy;
                apx[2] -= aFz;
            }
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
            const double SE = acc[e], SD = acc[ATMB_MCAP + e], SF = acc[2 * ATMB_MCAP + e];
            const double Wx = acc[3 * ATMB_MCAP + e], Wy = acc[4 * ATMB_MCAP + e], Wz = acc[5 * ATMB_MCAP + e];
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

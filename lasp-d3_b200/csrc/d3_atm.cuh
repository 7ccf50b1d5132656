// ATM three-body kernel (replaces the reference's atm_kernel, src/d3_kernel.cu:1199-1509).
// Included by d3_engine.cu after the kernel parameter block and the shared helpers.
//
// Enumeration: for each apex a, the half list L_a = {(j, T): j <= a in caller order,
// 1e-12 <= r^2 <= rc_ATM^2} built by k_atm_list; a triplet is an unordered pair of
// distinct entries {x, y} of L_a with 1e-12 <= r_xy^2 <= rc_ATM^2. This is the
// reference's (b, T_b, c, T_c) loop with c <= b (src/d3_kernel.cu:1235-1327); its
// repeated-index scale factors (:1282-1290) become a weight per unordered pair:
//     distinct atoms, none equal to a     w = 1     (reference force weight 1)
//     distinct atoms, one is a's image    w = 1/2   (force weight 1)
//     same atom, not a                    w = 1     (force weight 2)
//     same atom, equal to a               w = 1/3   (force weight 2)
// (the reference applies the scale to energy, dE/dCN and stress but not to forces;
// the force weight reproduces that, or equals w when atm_force_scaled is set).
//
// Schedule: persistent CTAs pull apexes from a work counter, largest lists first.
// Each thread owns one list entry x and visits every other entry y of the apex; all
// accumulation into x is thread-private and the apex's share is halved per visit.
// Partner entries are staged through shared memory with their C6 rows.
//
// Arithmetic per visit (FP64): one rsqrt (r_xy), one rsqrt (C6_xy), one inverse cube
// root (damping), one reciprocal (damping), each a float seed refined by two Newton
// steps; everything else is multiplication by precomputed reciprocals.

__device__ __forceinline__ double rsqrt_nr(double x) {
    // Newton-Raphson for x^(-1/2): y <- y (3 - x y^2) / 2, from a float seed
    double y = (double)rsqrtf((float)x);
    const double h = 0.5 * x;
    y = y * fma(-h * y, y, 1.5);
    y = y * fma(-h * y, y, 1.5);
    return y;
}

__device__ __forceinline__ double rcp_nr(double x) {
    // Newton-Raphson for 1/x: y <- y + y (1 - x y)
    double y = (double)__frcp_rn((float)x);
    y = fma(fma(-x, y, 1.0), y, y);
    y = fma(fma(-x, y, 1.0), y, y);
    return y;
}

__device__ __forceinline__ double rcbrt_nr(double x) {
    // Newton-Raphson for x^(-1/3): z <- z (4 - x z^3) / 3
    double z = (double)rcbrtf((float)x);
    z = z * fma(-x * z * z, z, 4.0) * (1.0 / 3.0);
    z = z * fma(-x * z * z, z, 4.0) * (1.0 / 3.0);
    return z;
}

struct Partner {
    double vx, vy, vz, d2, ir, id2, s, lam, g;
    int j, t;
};

constexpr int ATM_THREADS = 128;

// derivative polynomial of the angular term along side 1 (src/d3_kernel.cu:1367-1374),
// without the 3/8 / (r^6 r^3 ...) prefactor
__device__ __forceinline__ double dang_poly(double a, double b, double c) {
    // a: the side's own squared length; b, c: the other two
    const double bc = c - b;
    return a * a * a + a * a * (b + c) + a * (3.0 * c * c + 2.0 * c * b + 3.0 * b * b) - 5.0 * bc * bc * (c + b);
}

template <int NR>
__global__ void __launch_bounds__(ATM_THREADS) k_atm(KP p, int tile) {
    extern __shared__ double smem[];
    const int ne = p.ne;
    Partner *ptile = reinterpret_cast<Partner *>(smem);
    double *ytile = reinterpret_cast<double *>(ptile + tile); // [tile][ne][NR]
    double *yapex = ytile + (size_t)tile * ne * NR;           // [ne][NR]
    double *r0sq = yapex + ne * NR;                           // [ne][ne] r0ab^2
    __shared__ int s_item;
    __shared__ double red[ATM_THREADS / 32][12];
    const int tid = threadIdx.x;
    if (p.atm_off[p.n] > p.atm_cap) return; // list overflowed: the host grows it and re-runs
    for (int k = tid; k < ne * ne; k += blockDim.x) r0sq[k] = p.r0ab[k] * p.r0ab[k];
    const double x16c = 4294967296.0 / 43046721.0; // (4/3)^16 = 4^16 / 3^16
    const double third = 1.0 / 3.0;
    unsigned long long visits = 0;
    while (true) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(p.work, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= p.n) break;
        const int a = p.sorted_of[p.n - 1 - item];
        const long long e0 = p.atm_off[a];
        const int m = (int)(p.atm_off[a + 1] - e0);
        const double4 xa = p.xs[a];
        const int ta = (int)xa.w;
        for (int k = tid; k < ne * NR; k += blockDim.x) yapex[k] = p.Y[(size_t)a * ne * NR + k];
        double dwa[NR];
#pragma unroll
        for (int b = 0; b < NR; ++b) dwa[b] = p.dw[(size_t)a * NR + b];
        __syncthreads();
        double ea = 0, ga = 0, fax = 0, fay = 0, faz = 0;
        double vxx = 0, vyy = 0, vzz = 0, vxy = 0, vxz = 0, vyz = 0;
        for (int q0 = 0; q0 < m; q0 += blockDim.x) {
            const int q = q0 + tid;
            const bool active = q < m;
            double vqx = 0, vqy = 0, vqz = 0, d1 = 1, ir1 = 1, id1 = 1, sq = 0, lam_qa = 0, lam_aq = 0, gq = 0;
            double wq[NR], dwq[NR];
            int jq = -1, tq = 0;
            if (active) {
                const int2 ent = p.atm_ent[e0 + q];
                jq = ent.x;
                const int Tx = sext8(ent.y & 0xff), Ty = sext8((ent.y >> 8) & 0xff), Tz = sext8((ent.y >> 16) & 0xff);
                const double4 xj = p.xs[jq];
                tq = (int)xj.w;
                double sx, sy, sz;
                image_vec(p, Tx, Ty, Tz, sx, sy, sz);
                vqx = xj.x + sx - xa.x;
                vqy = xj.y + sy - xa.y;
                vqz = xj.z + sz - xa.z;
                d1 = vqx * vqx + vqy * vqy + vqz * vqz;
                ir1 = rsqrt_nr(d1);
                id1 = ir1 * ir1;
#pragma unroll
                for (int b = 0; b < NR; ++b) {
                    wq[b] = p.w[(size_t)jq * NR + b];
                    dwq[b] = p.dw[(size_t)jq * NR + b];
                }
                const double *ya = yapex + tq * NR;                   // C6_aq = y_{a,tq} . w_q
                const double *yq = p.Y + ((size_t)jq * ne + ta) * NR; // dC6_aq/dCN_a = y_{q,ta} . dw_a
                double c6 = 0, dca = 0, dcq = 0;
#pragma unroll
                for (int b = 0; b < NR; ++b) {
                    c6 += ya[b] * wq[b];
                    dcq += ya[b] * dwq[b];
                    dca += yq[b] * dwa[b];
                }
                const double is = rsqrt_nr(c6);
                sq = c6 * is;
                lam_aq = dca * is * is;
                lam_qa = dcq * is * is;
                const double u = r0sq[ta * ne + tq] * id1;
                gq = u * u * u * rcbrt_nr(u);
            } else {
#pragma unroll
                for (int b = 0; b < NR; ++b) wq[b] = dwq[b] = 0.0;
            }
            double eq = 0, gq_acc = 0, fqx = 0, fqy = 0, fqz = 0;
            for (int p0 = 0; p0 < m; p0 += tile) {
                const int cnt = min(tile, m - p0);
                __syncthreads();
                for (int k = tid; k < cnt; k += blockDim.x) {
                    const int2 ent = p.atm_ent[e0 + p0 + k];
                    const int jp = ent.x;
                    const int Tx = sext8(ent.y & 0xff), Ty = sext8((ent.y >> 8) & 0xff), Tz = sext8((ent.y >> 16) & 0xff);
                    const double4 xj = p.xs[jp];
                    const int tp = (int)xj.w;
                    double sx, sy, sz;
                    image_vec(p, Tx, Ty, Tz, sx, sy, sz);
                    Partner pr;
                    pr.vx = xj.x + sx - xa.x;
                    pr.vy = xj.y + sy - xa.y;
                    pr.vz = xj.z + sz - xa.z;
                    pr.d2 = pr.vx * pr.vx + pr.vy * pr.vy + pr.vz * pr.vz;
                    pr.ir = rsqrt_nr(pr.d2);
                    pr.id2 = pr.ir * pr.ir;
                    const double *ya = yapex + tp * NR;
                    const double *yp = p.Y + ((size_t)jp * ne + ta) * NR;
                    double c6 = 0, dca = 0;
#pragma unroll
                    for (int b = 0; b < NR; ++b) {
                        c6 += ya[b] * p.w[(size_t)jp * NR + b];
                        dca += yp[b] * dwa[b];
                    }
                    const double is = rsqrt_nr(c6);
                    pr.s = c6 * is;
                    pr.lam = dca * is * is; // dlnC6_ap/dCN_a
                    const double u = r0sq[ta * ne + tp] * pr.id2;
                    pr.g = u * u * u * rcbrt_nr(u);
                    pr.j = jp;
                    pr.t = tp;
                    ptile[k] = pr;
                    const double *ysrc = p.Y + (size_t)jp * ne * NR;
                    double *ydst = ytile + (size_t)k * ne * NR;
                    for (int u2 = 0; u2 < ne * NR; ++u2) ydst[u2] = ysrc[u2];
                }
                __syncthreads();
                if (!active) continue;
                for (int k = 0; k < cnt; ++k) {
                    if (p0 + k == q) continue;
                    const Partner &pr = ptile[k];
                    const double rx = vqx - pr.vx, ry = vqy - pr.vy, rz = vqz - pr.vz;
                    const double d3 = rx * rx + ry * ry + rz * rz;
                    if (d3 > p.ratm2 || d3 < 1e-12) continue;
                    ++visits;
                    const double ir3 = rsqrt_nr(d3);
                    const double id3 = ir3 * ir3;
                    const double *yp = ytile + ((size_t)k * ne + tq) * NR; // C6_qp = y_{p,tq} . w_q
                    double c6 = 0, dc6 = 0;
#pragma unroll
                    for (int b = 0; b < NR; ++b) {
                        const double y = yp[b];
                        c6 += y * wq[b];
                        dc6 += y * dwq[b];
                    }
                    const double is3 = rsqrt_nr(c6);
                    const double s3 = c6 * is3;
                    const double lam_qp = dc6 * is3 * is3;
                    const double u = r0sq[tq * ne + pr.t] * id3;
                    const double g3 = u * u * u * rcbrt_nr(u);
                    // weights (reference scale factors, src/d3_kernel.cu:1282-1290)
                    const bool same = (jq == pr.j), qa = (jq == a), pa = (pr.j == a);
                    double w, wf;
                    if (same) {
                        w = qa ? third : 1.0;
                        wf = 2.0;
                    } else if (qa || pa) {
                        w = 0.5;
                        wf = 1.0;
                    } else {
                        w = 1.0;
                        wf = 1.0;
                    }
                    if (p.atm_force_scaled) wf = w;
                    const double d2 = pr.d2;
                    const double irsq = id1 * pr.id2 * id3;
                    const double ir9 = irsq * ir1 * pr.ir * ir3;
                    const double t1 = d1 + d2 - d3, t2 = d1 - d2 + d3, t3 = -d1 + d2 + d3;
                    const double A = fma(0.375 * t1 * t2, t3 * irsq, 1.0) * ir9; // (1 + 3 cos cos cos) / r^9
                    const double dd = 0.375 * ir9 * irsq;
                    const double dang1 = dd * dang_poly(d1, d2, d3);
                    const double dang2 = dd * dang_poly(d2, d3, d1);
                    const double dang3 = dd * dang_poly(d3, d2, d1);
                    const double x16 = x16c * gq * pr.g * g3;
                    const double fd = rcp_nr(fma(6.0, x16, 1.0));
                    const double dfd = 32.0 * x16 * fd * fd;
                    const double C9 = -sq * pr.s * s3;
                    const double Et = C9 * A * fd;
                    const double Adfd = A * dfd;
                    const double f1 = -C9 * (dang1 * fd - Adfd) * id1;
                    const double f2 = -C9 * (dang2 * fd - Adfd) * pr.id2;
                    const double f3 = -C9 * (dang3 * fd - Adfd) * id3;
                    // own entry (atom x): energy share, dE/dCN_x, force on x
                    eq += w * Et * third;
                    gq_acc += w * 0.5 * Et * (lam_qa + lam_qp);
                    fqx += wf * fma(f1, vqx, f3 * rx);
                    fqy += wf * fma(f1, vqy, f3 * ry);
                    fqz += wf * fma(f1, vqz, f3 * rz);
                    // apex share, halved (each unordered pair is visited twice)
                    const double wh = 0.5 * w, wfh = 0.5 * wf;
                    ea += wh * Et * third;
                    ga += wh * 0.5 * Et * (lam_aq + pr.lam);
                    fax -= wfh * fma(f1, vqx, f2 * pr.vx);
                    fay -= wfh * fma(f1, vqy, f2 * pr.vy);
                    faz -= wfh * fma(f1, vqz, f2 * pr.vz);
                    const double a1 = wh * f1, a2 = wh * f2, a3 = wh * f3;
                    vxx += a1 * vqx * vqx + a2 * pr.vx * pr.vx + a3 * rx * rx;
                    vyy += a1 * vqy * vqy + a2 * pr.vy * pr.vy + a3 * ry * ry;
                    vzz += a1 * vqz * vqz + a2 * pr.vz * pr.vz + a3 * rz * rz;
                    vxy += a1 * vqx * vqy + a2 * pr.vx * pr.vy + a3 * rx * ry;
                    vxz += a1 * vqx * vqz + a2 * pr.vx * pr.vz + a3 * rx * rz;
                    vyz += a1 * vqy * vqz + a2 * pr.vy * pr.vz + a3 * ry * rz;
                }
            }
            if (active) {
                atomicAdd(&p.eb[jq], eq);
                atomicAdd(&p.gb[jq], gq_acc);
                atomicAdd(&p.fb[3 * jq], fqx);
                atomicAdd(&p.fb[3 * jq + 1], fqy);
                atomicAdd(&p.fb[3 * jq + 2], fqz);
            }
        }
        // apex reduction over the CTA (fixed order)
        double vals[11] = {ea, ga, fax, fay, faz, vxx, vyy, vzz, vxy, vxz, vyz};
        const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
        for (int k = 0; k < 11; ++k) {
            const double v = warp_sum(vals[k]);
            if (lane == 0) red[wid][k] = v;
        }
        __syncthreads();
        if (tid == 0) {
            double tot[11];
            for (int k = 0; k < 11; ++k) {
                tot[k] = 0;
                for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) tot[k] += red[w2][k];
            }
            p.ea[a] = tot[0];
            p.ga[a] = tot[1];
            p.fa[3 * a] = tot[2];
            p.fa[3 * a + 1] = tot[3];
            p.fa[3 * a + 2] = tot[4];
            const double sc = -1.0 / p.vol;
            for (int k = 0; k < 6; ++k) p.va[6 * (size_t)a + k] = tot[5 + k] * sc;
        }
    }
    // in-range visits (each unordered triplet counted twice)
    for (int o = 16; o > 0; o >>= 1) visits += __shfl_xor_sync(0xffffffffu, visits, o);
    if ((tid & 31) == 0 && p.counters) atomicAdd(p.counters, visits);
}

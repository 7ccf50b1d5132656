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
// Each thread owns one list entry x (entries handed out in order of distance from the
// apex, so the lanes of a warp have similar numbers of partners in range) and visits
// every other entry y of the apex whose distance test passes (a 64-bit mask per tile of
// partners, so only in-range visits execute). Every unordered pair is visited from
// both of its entries; all accumulation into x is thread-private.
//
// Mirror symmetry keeps the per-visit accumulation small: the side a-y force scalar of
// visit (x, y) equals the side a-x scalar of visit (y, x), so the apex force, the apex
// dE/dCN and the a-x/a-y virial terms follow from per-thread scalar sums over the
// thread's own side a-x; the x-y side needs one vector sum (sum f_xy v_y).
//
// Arithmetic per visit (FP64): r_xy^(-1/2), C6_xy^(-1/2), an inverse cube root for the
// damping and one reciprocal, each a float seed refined by one Newton step (relative
// error ~1e-13); everything else is multiplication by precomputed reciprocals.

__device__ __forceinline__ double rsqrt_nr(double x) {
    // Newton-Raphson for x^(-1/2): y <- y (3 - x y^2) / 2, from a float seed
    double y = (double)rsqrtf((float)x);
    const double h = 0.5 * x;
    y = y * fma(-h * y, y, 1.5);
    return y;
}

__device__ __forceinline__ double rsqrt_nr2(double x) {
    double y = rsqrt_nr(x);
    return y * fma(-0.5 * x * y, y, 1.5);
}

__device__ __forceinline__ double rcp_nr(double x) {
    // Newton-Raphson for 1/x: y <- y + y (1 - x y), from the fast float reciprocal
    double y = (double)__fdividef(1.0f, (float)x);
    y = fma(fma(-x, y, 1.0), y, y);
    return y;
}

__device__ __forceinline__ double rcp_nr2(double x) {
    double y = rcp_nr(x);
    return fma(fma(-x, y, 1.0), y, y);
}

__device__ __forceinline__ double rcbrt_nr(double x) {
    // Newton-Raphson for x^(-1/3): z <- z (4 - x z^3) / 3, from a float seed
    // 2^(-log2(x)/3) evaluated with the fast base-2 logarithm and exponential
    double z = (double)exp2f(__log2f((float)x) * (-1.0f / 3.0f));
    z = z * fma(-x * z * z, z, 4.0) * (1.0 / 3.0);
    return z;
}

__device__ __forceinline__ double rcbrt_nr2(double x) {
    double z = rcbrt_nr(x);
    return z * fma(-x * z * z, z, 4.0) * (1.0 / 3.0);
}

struct Partner {
    double vx, vy, vz, d2, ir, id2, s, g;
    float fx, fy, fz;
    int j, t, pad;
};

constexpr int ATM_THREADS = 128;
constexpr int ATM_PERM_CAP = 8192; // longest list whose entries are re-ordered by distance
constexpr int ATM_SHELLS = 32;

// CENTER: centre mode of the surrogate fallback (apexes from p.atm_apex, full lists,
// every triplet weighted 1/3 for energy and forces alike)
template <int NR, bool CENTER>
__global__ void __launch_bounds__(ATM_THREADS) k_atm(KP p, int tile) {
    extern __shared__ double smem[];
    const int ne = p.ne;
    Partner *ptile = reinterpret_cast<Partner *>(smem);
    double *ytile = reinterpret_cast<double *>(ptile + tile); // [tile][ne][NR]
    double *yapex = ytile + (size_t)tile * ne * NR;           // [ne][NR]
    double *r0sq = yapex + ne * NR;                           // [ne][ne] r0ab^2
    unsigned short *perm = reinterpret_cast<unsigned short *>(r0sq + ne * ne); // [ATM_PERM_CAP]
    __shared__ int s_item;
    __shared__ int shell_cnt[ATM_SHELLS], shell_off[ATM_SHELLS];
    __shared__ double red[ATM_THREADS / 32][12];
    const int tid = threadIdx.x;
    if (p.atm_off[p.n] > p.atm_cap) return; // list overflowed: the host grows it and re-runs
    for (int k = tid; k < ne * ne; k += blockDim.x) r0sq[k] = p.r0ab[k] * p.r0ab[k];
    const double x16c = 4294967296.0 / 43046721.0; // (4/3)^16 = 4^16 / 3^16
    const double third = 1.0 / 3.0;
    const float ratm2f = (float)(p.ratm2 * (1.0 + 1e-5)); // conservative single-precision test
    const double inv_rc = 1.0 / sqrt(p.ratm2);
    unsigned long long visits = 0;
    while (true) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(p.work, 1);
        if (tid < ATM_SHELLS) shell_cnt[tid] = 0;
        __syncthreads();
        const int item = CENTER ? s_item : s_item * p.shard_world + p.shard_rank;
        if (item >= (CENTER ? *p.atm_napex : p.n)) break;
        const int a = CENTER ? p.atm_apex[item] : p.sorted_of[p.n - 1 - item];
        const long long e0 = p.atm_off[a];
        const int m = (int)(p.atm_off[a + 1] - e0);
        const double4 xa = p.xs[a];
        const int ta = (int)xa.w;
        const SG &g = p.sg[p.sid[a]];
        for (int k = tid; k < ne * NR; k += blockDim.x) yapex[k] = p.Y[(size_t)a * ne * NR + k];
        double dwa[NR];
#pragma unroll
        for (int b = 0; b < NR; ++b) dwa[b] = p.dw[(size_t)a * NR + b];
        // order the apex's entries by distance shell (counting sort in shared memory)
        const bool sorted = m <= ATM_PERM_CAP;
        if (sorted) {
            for (int k = tid; k < m; k += blockDim.x) {
                const int2 ent = p.atm_ent[e0 + k];
                const int Tx = sext8(ent.y & 0xff), Ty = sext8((ent.y >> 8) & 0xff), Tz = sext8((ent.y >> 16) & 0xff);
                const double4 xj = p.xs[ent.x];
                double sx, sy, sz;
                image_vec(g, Tx, Ty, Tz, sx, sy, sz);
                const double dx = xj.x + sx - xa.x, dy = xj.y + sy - xa.y, dz = xj.z + sz - xa.z;
                const int sh = min(ATM_SHELLS - 1, (int)(sqrt(dx * dx + dy * dy + dz * dz) * inv_rc * ATM_SHELLS));
                atomicAdd(&shell_cnt[sh], 1);
            }
            __syncthreads();
            if (tid == 0) {
                int acc = 0;
                for (int k = 0; k < ATM_SHELLS; ++k) {
                    shell_off[k] = acc;
                    acc += shell_cnt[k];
                }
            }
            __syncthreads();
            for (int k = tid; k < m; k += blockDim.x) {
                const int2 ent = p.atm_ent[e0 + k];
                const int Tx = sext8(ent.y & 0xff), Ty = sext8((ent.y >> 8) & 0xff), Tz = sext8((ent.y >> 16) & 0xff);
                const double4 xj = p.xs[ent.x];
                double sx, sy, sz;
                image_vec(g, Tx, Ty, Tz, sx, sy, sz);
                const double dx = xj.x + sx - xa.x, dy = xj.y + sy - xa.y, dz = xj.z + sz - xa.z;
                const int sh = min(ATM_SHELLS - 1, (int)(sqrt(dx * dx + dy * dy + dz * dz) * inv_rc * ATM_SHELLS));
                perm[atomicAdd(&shell_off[sh], 1)] = (unsigned short)k;
            }
        }
        __syncthreads();
        double ea = 0, ga = 0, fax = 0, fay = 0, faz = 0;
        double vxx = 0, vyy = 0, vzz = 0, vxy = 0, vxz = 0, vyz = 0;
        for (int q0 = 0; q0 < m; q0 += blockDim.x) {
            const int qi = q0 + tid;
            const bool active = qi < m;
            const int q = active ? (sorted ? (int)perm[qi] : qi) : -1;
            double vqx = 0, vqy = 0, vqz = 0, d1 = 1, ir1 = 1, id1 = 1, sq = 0, lam_qa = 0, lam_aq = 0, gq = 0;
            float fqx = 0.f, fqy = 0.f, fqz = 1e30f;
            double wq[NR], dwq[NR];
            int jq = -1, tq = 0;
            if (active) {
                const int2 ent = p.atm_ent[e0 + q];
                jq = ent.x;
                const int Tx = sext8(ent.y & 0xff), Ty = sext8((ent.y >> 8) & 0xff), Tz = sext8((ent.y >> 16) & 0xff);
                const double4 xj = p.xs[jq];
                tq = (int)xj.w;
                double sx, sy, sz;
                image_vec(g, Tx, Ty, Tz, sx, sy, sz);
                vqx = xj.x + sx - xa.x;
                vqy = xj.y + sy - xa.y;
                vqz = xj.z + sz - xa.z;
                fqx = (float)vqx;
                fqy = (float)vqy;
                fqz = (float)vqz;
                d1 = vqx * vqx + vqy * vqy + vqz * vqz;
                ir1 = rsqrt_nr2(d1);
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
                const double is = rsqrt_nr2(c6);
                sq = c6 * is;
                lam_aq = dca * is * is;
                lam_qa = dcq * is * is;
                const double u = r0sq[ta * ne + tq] * id1;
                gq = u * u * u * rcbrt_nr2(u);
            } else {
#pragma unroll
                for (int b = 0; b < NR; ++b) wq[b] = dwq[b] = 0.0;
            }
            // per-thread sums over visits of the own entry x
            double Esum = 0;           // sum w Et
            double Dsum = 0;           // sum w Et lam_xy
            double Ssum = 0;           // sum w (f1 + f3)        (virial, own side + x-y side)
            double Ux = 0, Uy = 0, Uz = 0; // sum w f3 v_y        (virial cross term)
            double Fsum = 0;           // sum wf (f1 + f3)       (force on x along v_x)
            double Wx = 0, Wy = 0, Wz = 0; // sum wf f3 v_y        (force on x)
            double Asum = 0;           // sum wf f1              (apex force)
            for (int p0 = 0; p0 < m; p0 += tile) {
                const int cnt = min(tile, m - p0);
                __syncthreads();
                for (int k = tid; k < cnt; k += blockDim.x) {
                    // partners in the same distance-shell order: a tile is then spread
                    // evenly over directions, so lanes at equal distance from the apex
                    // find similar numbers of partners in range
                    const int pi = p0 + k;
                    const int2 ent = p.atm_ent[e0 + (sorted ? (int)perm[pi] : pi)];
                    const int jp = ent.x;
                    const int Tx = sext8(ent.y & 0xff), Ty = sext8((ent.y >> 8) & 0xff), Tz = sext8((ent.y >> 16) & 0xff);
                    const double4 xj = p.xs[jp];
                    const int tp = (int)xj.w;
                    double sx, sy, sz;
                    image_vec(g, Tx, Ty, Tz, sx, sy, sz);
                    Partner pr;
                    pr.vx = xj.x + sx - xa.x;
                    pr.vy = xj.y + sy - xa.y;
                    pr.vz = xj.z + sz - xa.z;
                    pr.fx = (float)pr.vx;
                    pr.fy = (float)pr.vy;
                    pr.fz = (float)pr.vz;
                    pr.d2 = pr.vx * pr.vx + pr.vy * pr.vy + pr.vz * pr.vz;
                    pr.ir = rsqrt_nr2(pr.d2);
                    pr.id2 = pr.ir * pr.ir;
                    const double *ya = yapex + tp * NR;
                    double c6 = 0;
#pragma unroll
                    for (int b = 0; b < NR; ++b) c6 += ya[b] * p.w[(size_t)jp * NR + b];
                    pr.s = c6 * rsqrt_nr2(c6);
                    const double u = r0sq[ta * ne + tp] * pr.id2;
                    pr.g = u * u * u * rcbrt_nr2(u);
                    pr.j = jp;
                    pr.t = tp;
                    pr.pad = 0;
                    ptile[k] = pr;
                    const double *ysrc = p.Y + (size_t)jp * ne * NR;
                    double *ydst = ytile + (size_t)k * ne * NR;
                    for (int u2 = 0; u2 < ne * NR; ++u2) ydst[u2] = ysrc[u2];
                }
                __syncthreads();
                for (int s0 = 0; s0 < cnt; s0 += 64) {
                    // single-precision distance test builds the mask of in-range partners
                    unsigned long long mask = 0ull;
                    const int sc = min(64, cnt - s0);
                    for (int k = 0; k < sc; ++k) {
                        const Partner &pr = ptile[s0 + k];
                        const float dx = fqx - pr.fx, dy = fqy - pr.fy, dz = fqz - pr.fz;
                        const float d3f = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        if (d3f <= ratm2f) mask |= 1ull << k;
                    }
                    while (__any_sync(0xffffffffu, mask != 0ull)) {
                        if (mask == 0ull) continue;
                        const int k = s0 + __ffsll((long long)mask) - 1;
                        mask &= mask - 1ull;
                        const Partner &pr = ptile[k];
                        const double rx = vqx - pr.vx, ry = vqy - pr.vy, rz = vqz - pr.vz;
                        const double d3 = rx * rx + ry * ry + rz * rz;
                        if (d3 > p.ratm2 || d3 < 1e-12) continue; // exact test (also drops x == y)
                        ++visits;
                        const double ir3 = rsqrt_nr(d3);
                        const double id3 = ir3 * ir3;
                        const double *yp = ytile + ((size_t)k * ne + tq) * NR; // C6_xy = y_{y,tx} . w_x
                        double c6 = 0, dc6 = 0;
#pragma unroll
                        for (int b = 0; b < NR; ++b) {
                            const double y = yp[b];
                            c6 = fma(y, wq[b], c6);
                            dc6 = fma(y, dwq[b], dc6);
                        }
                        const double is3 = rsqrt_nr(c6);
                        const double s3 = c6 * is3;
                        const double lam_xy = dc6 * is3 * is3;
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
                        if (CENTER) w = wf = third;
                        // angular term A = (1 + 3 cos cos cos) / (r1 r2 r3)^3 and its side
                        // derivatives: with t1..t3 the cosine numerators, P = t1 t2 t3 and
                        // Q = d1 d2 d3, -r_k dA/dr_k = Q^(-5/2) (3Q - 3/4 d_k dP/dd_k + 15/8 P)
                        // (the reference's dangle polynomials, src/d3_kernel.cu:1367-1392)
                        const double d2 = pr.d2;
                        const double irsq = id1 * pr.id2 * id3;
                        const double ir9 = irsq * ir1 * pr.ir * ir3;
                        const double t1 = d1 + d2 - d3, t2 = d1 - d2 + d3, t3 = -d1 + d2 + d3;
                        const double t12 = t1 * t2, t13 = t1 * t3, t23 = t2 * t3;
                        const double P = t12 * t3;
                        const double A = fma(0.375 * P, irsq, 1.0) * ir9;
                        const double q52 = ir9 * irsq;
                        const double Q3 = 3.0 * d1 * d2 * d3;
                        const double dang1 = q52 * fma(-0.75 * d1, t23 + t13 - t12, fma(1.875, P, Q3));
                        const double dang3 = q52 * fma(-0.75 * d3, t13 + t12 - t23, fma(1.875, P, Q3));
                        const double x16 = x16c * gq * pr.g * g3;
                        const double fd = rcp_nr(fma(6.0, x16, 1.0));
                        const double dfd = 32.0 * x16 * fd * fd;
                        const double C9 = -sq * pr.s * s3;
                        const double Et = C9 * A * fd;
                        const double Adfd = A * dfd;
                        const double f1 = -C9 * fma(dang1, fd, -Adfd) * id1;
                        const double f3 = -C9 * fma(dang3, fd, -Adfd) * id3;
                        const double wE = w * Et;
                        Esum += wE;
                        Dsum = fma(wE, lam_xy, Dsum);
                        const double wf13 = w * (f1 + f3), w3 = w * f3;
                        Ssum += wf13;
                        Ux = fma(w3, pr.vx, Ux);
                        Uy = fma(w3, pr.vy, Uy);
                        Uz = fma(w3, pr.vz, Uz);
                        const double f13 = wf * (f1 + f3), ff3 = wf * f3;
                        Fsum += f13;
                        Wx = fma(ff3, pr.vx, Wx);
                        Wy = fma(ff3, pr.vy, Wy);
                        Wz = fma(ff3, pr.vz, Wz);
                        Asum = fma(wf, f1, Asum);
                    }
                }
            }
            if (active) {
                // own entry x: energy share Et/3, dE/dCN_x = Et/2 (lam_xa + lam_xy),
                // force F_x = f1 v_x + f3 (v_x - v_y)
                atomicAdd(&p.eb[jq], Esum * third);
                atomicAdd(&p.gb[jq], 0.5 * (lam_qa * Esum + Dsum));
                atomicAdd(&p.fb[3 * jq], Fsum * vqx - Wx);
                atomicAdd(&p.fb[3 * jq + 1], Fsum * vqy - Wy);
                atomicAdd(&p.fb[3 * jq + 2], Fsum * vqz - Wz);
                // apex share (each pair is visited twice): energy Et/3, dE/dCN_a via the own
                // side, force -f1 v_x per visit, virial sum over sides of f r (x) r
                ea += 0.5 * Esum * third;
                ga += 0.5 * lam_aq * Esum;
                fax -= Asum * vqx;
                fay -= Asum * vqy;
                faz -= Asum * vqz;
                // x-y side: f r (x) r with r = v_x - v_y; its v_x (x) v_x part is in Ssum,
                // its v_y (x) v_y part arrives from the mirrored visit, the cross part is
                // split evenly between the two visits
                vxx += Ssum * vqx * vqx - Ux * vqx;
                vyy += Ssum * vqy * vqy - Uy * vqy;
                vzz += Ssum * vqz * vqz - Uz * vqz;
                vxy += Ssum * vqx * vqy - 0.5 * (Ux * vqy + Uy * vqx);
                vxz += Ssum * vqx * vqz - 0.5 * (Ux * vqz + Uz * vqx);
                vyz += Ssum * vqy * vqz - 0.5 * (Uy * vqz + Uz * vqy);
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
            const double sc = -1.0 / g.vol;
            for (int k = 0; k < 6; ++k) p.va[6 * (size_t)a + k] = tot[5 + k] * sc;
        }
    }
    // in-range visits (each unordered triplet counted twice)
    for (int o = 16; o > 0; o >>= 1) visits += __shfl_xor_sync(0xffffffffu, visits, o);
    if ((tid & 31) == 0 && p.counters) atomicAdd(p.counters, visits);
}

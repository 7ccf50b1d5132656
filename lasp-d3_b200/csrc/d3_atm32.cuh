// ATM three-body kernel, precision form: the per-visit triplet arithmetic in FP32.
// Same enumeration, schedule, weights and mirror-symmetric accumulation as k_atm
// (d3_atm.cuh); per-entry set-up (C6 of the apex pairs, damping ratios) is done in FP64
// and rounded once. Per-visit sums are kept in FP32 within one partner tile and carried
// across tiles in FP64 (blocked summation, error ~ sqrt(tile) * eps_32 per block); the
// dE/dCN sum is accumulated in FP64 per visit.

struct Partner32 {
    float vx, vy, vz, d2, ir, id2, s, g;
    int j, t;
};

template <int NR>
__global__ void __launch_bounds__(ATM_THREADS) k_atm32(KP p, int tile) {
    extern __shared__ double smem[];
    const int ne = p.ne;
    Partner32 *ptile = reinterpret_cast<Partner32 *>(smem);
    float *ytile = reinterpret_cast<float *>(ptile + tile);    // [tile][ne][NR]
    double *yapex = reinterpret_cast<double *>(ytile + (((size_t)tile * ne * NR + 1) & ~(size_t)1)); // [ne][NR]
    float *r0sq = reinterpret_cast<float *>(yapex + ne * NR); // [ne][ne]
    unsigned short *perm = reinterpret_cast<unsigned short *>(r0sq + ((ne * ne + 1) & ~1)); // [ATM_PERM_CAP]
    __shared__ int s_item;
    __shared__ int shell_cnt[ATM_SHELLS], shell_off[ATM_SHELLS];
    __shared__ double red[ATM_THREADS / 32][12];
    const int tid = threadIdx.x;
    if (p.atm_off[p.n] > p.atm_cap) return; // list overflowed: the host grows it and re-runs
    for (int k = tid; k < ne * ne; k += blockDim.x) r0sq[k] = (float)(p.r0ab[k] * p.r0ab[k]);
    const double x16c_d = 4294967296.0 / 43046721.0; // (4/3)^16
    const float x16c = (float)x16c_d;
    const float third = 1.0f / 3.0f;
    const float ratm2f = (float)p.ratm2;
    const double inv_rc = 1.0 / sqrt(p.ratm2);
    unsigned long long visits = 0;
    while (true) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(p.work, 1);
        if (tid < ATM_SHELLS) shell_cnt[tid] = 0;
        __syncthreads();
        const int item = s_item;
        if (item >= p.n) break;
        const int a = p.sorted_of[p.n - 1 - item];
        const long long e0 = p.atm_off[a];
        const int m = (int)(p.atm_off[a + 1] - e0);
        const double4 xa = p.xs[a];
        const int ta = (int)xa.w;
        const SG &g = p.sg[p.sid[a]];
        for (int k = tid; k < ne * NR; k += blockDim.x) yapex[k] = p.Y[(size_t)a * ne * NR + k];
        double dwa[NR];
#pragma unroll
        for (int b = 0; b < NR; ++b) dwa[b] = p.dw[(size_t)a * NR + b];
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
            double vqx_d = 0, vqy_d = 0, vqz_d = 0, lam_qa = 0, lam_aq = 0;
            float vqx = 0.f, vqy = 0.f, vqz = 1e30f, d1 = 1.f, ir1 = 1.f, id1 = 1.f, sq = 0.f, gq = 0.f;
            float wq[NR], dwq[NR];
            int jq = -1, tq = 0;
            if (active) {
                const int2 ent = p.atm_ent[e0 + q];
                jq = ent.x;
                const int Tx = sext8(ent.y & 0xff), Ty = sext8((ent.y >> 8) & 0xff), Tz = sext8((ent.y >> 16) & 0xff);
                const double4 xj = p.xs[jq];
                tq = (int)xj.w;
                double sx, sy, sz;
                image_vec(g, Tx, Ty, Tz, sx, sy, sz);
                vqx_d = xj.x + sx - xa.x;
                vqy_d = xj.y + sy - xa.y;
                vqz_d = xj.z + sz - xa.z;
                const double d1d = vqx_d * vqx_d + vqy_d * vqy_d + vqz_d * vqz_d;
                vqx = (float)vqx_d;
                vqy = (float)vqy_d;
                vqz = (float)vqz_d;
                d1 = (float)d1d;
                ir1 = (float)(1.0 / sqrt(d1d));
                id1 = (float)(1.0 / d1d);
                double wd[NR], dwd[NR];
#pragma unroll
                for (int b = 0; b < NR; ++b) {
                    wd[b] = p.w[(size_t)jq * NR + b];
                    dwd[b] = p.dw[(size_t)jq * NR + b];
                    wq[b] = (float)wd[b];
                    dwq[b] = (float)dwd[b];
                }
                const double *ya = yapex + tq * NR;
                const double *yq = p.Y + ((size_t)jq * ne + ta) * NR;
                double c6 = 0, dca = 0, dcq = 0;
#pragma unroll
                for (int b = 0; b < NR; ++b) {
                    c6 += ya[b] * wd[b];
                    dcq += ya[b] * dwd[b];
                    dca += yq[b] * dwa[b];
                }
                sq = (float)sqrt(c6);
                lam_aq = dca / c6;
                lam_qa = dcq / c6;
                gq = (float)pow((double)r0sq[ta * ne + tq] / d1d, 8.0 / 3.0);
            } else {
#pragma unroll
                for (int b = 0; b < NR; ++b) wq[b] = dwq[b] = 0.f;
            }
            double Esum = 0, Dsum = 0, Ssum = 0, Ux = 0, Uy = 0, Uz = 0, Fsum = 0, Wx = 0, Wy = 0, Wz = 0, Asum = 0;
            for (int p0 = 0; p0 < m; p0 += tile) {
                const int cnt = min(tile, m - p0);
                __syncthreads();
                for (int k = tid; k < cnt; k += blockDim.x) {
                    const int pi = p0 + k;
                    const int2 ent = p.atm_ent[e0 + (sorted ? (int)perm[pi] : pi)];
                    const int jp = ent.x;
                    const int Tx = sext8(ent.y & 0xff), Ty = sext8((ent.y >> 8) & 0xff), Tz = sext8((ent.y >> 16) & 0xff);
                    const double4 xj = p.xs[jp];
                    const int tp = (int)xj.w;
                    double sx, sy, sz;
                    image_vec(g, Tx, Ty, Tz, sx, sy, sz);
                    const double vx = xj.x + sx - xa.x, vy = xj.y + sy - xa.y, vz = xj.z + sz - xa.z;
                    const double d2 = vx * vx + vy * vy + vz * vz;
                    const double *ya = yapex + tp * NR;
                    double c6 = 0;
#pragma unroll
                    for (int b = 0; b < NR; ++b) c6 += ya[b] * p.w[(size_t)jp * NR + b];
                    Partner32 pr;
                    pr.vx = (float)vx;
                    pr.vy = (float)vy;
                    pr.vz = (float)vz;
                    pr.d2 = (float)d2;
                    pr.ir = (float)(1.0 / sqrt(d2));
                    pr.id2 = (float)(1.0 / d2);
                    pr.s = (float)sqrt(c6);
                    pr.g = (float)pow((double)r0sq[ta * ne + tp] / d2, 8.0 / 3.0);
                    pr.j = jp;
                    pr.t = tp;
                    ptile[k] = pr;
                    const float *ysrc = p.Y32 + (size_t)jp * ne * NR;
                    float *ydst = ytile + (size_t)k * ne * NR;
                    for (int u2 = 0; u2 < ne * NR; ++u2) ydst[u2] = ysrc[u2];
                }
                __syncthreads();
                float tE = 0.f, tS = 0.f, tUx = 0.f, tUy = 0.f, tUz = 0.f, tF = 0.f, tWx = 0.f, tWy = 0.f, tWz = 0.f,
                      tA = 0.f;
                for (int s0 = 0; s0 < cnt; s0 += 64) {
                    unsigned long long mask = 0ull;
                    const int sc = min(64, cnt - s0);
                    for (int k = 0; k < sc; ++k) {
                        const Partner32 &pr = ptile[s0 + k];
                        const float dx = vqx - pr.vx, dy = vqy - pr.vy, dz = vqz - pr.vz;
                        const float d3 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        if (d3 <= ratm2f && d3 >= 1e-12f) mask |= 1ull << k;
                    }
                    while (__any_sync(0xffffffffu, mask != 0ull)) {
                        if (mask == 0ull) continue;
                        const int k = s0 + __ffsll((long long)mask) - 1;
                        mask &= mask - 1ull;
                        const Partner32 &pr = ptile[k];
                        ++visits;
                        const float rx = vqx - pr.vx, ry = vqy - pr.vy, rz = vqz - pr.vz;
                        const float d3 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
                        const float ir3 = rsqrtf(d3);
                        const float id3 = ir3 * ir3;
                        const float *yp = ytile + ((size_t)k * ne + tq) * NR;
                        float c6 = 0.f, dc6 = 0.f;
#pragma unroll
                        for (int b = 0; b < NR; ++b) {
                            const float y = yp[b];
                            c6 = fmaf(y, wq[b], c6);
                            dc6 = fmaf(y, dwq[b], dc6);
                        }
                        const float is3 = rsqrtf(c6);
                        const float s3 = c6 * is3;
                        const float lam_xy = dc6 * is3 * is3;
                        const float u = r0sq[tq * ne + pr.t] * id3;
                        const float g3 = u * u * u * exp2f(__log2f(u) * (-1.0f / 3.0f));
                        const bool same = (jq == pr.j), qa = (jq == a), pa = (pr.j == a);
                        float w, wf;
                        if (same) {
                            w = qa ? third : 1.0f;
                            wf = 2.0f;
                        } else if (qa || pa) {
                            w = 0.5f;
                            wf = 1.0f;
                        } else {
                            w = 1.0f;
                            wf = 1.0f;
                        }
                        if (p.atm_force_scaled) wf = w;
                        const float d2 = pr.d2;
                        const float irsq = id1 * pr.id2 * id3;
                        const float ir9 = irsq * ir1 * pr.ir * ir3;
                        const float t1 = d1 + d2 - d3, t2 = d1 - d2 + d3, t3 = -d1 + d2 + d3;
                        const float t12 = t1 * t2, t13 = t1 * t3, t23 = t2 * t3;
                        const float P = t12 * t3;
                        const float A = fmaf(0.375f * P, irsq, 1.0f) * ir9;
                        const float q52 = ir9 * irsq;
                        const float Q3 = 3.0f * d1 * d2 * d3;
                        const float dang1 = q52 * fmaf(-0.75f * d1, t23 + t13 - t12, fmaf(1.875f, P, Q3));
                        const float dang3 = q52 * fmaf(-0.75f * d3, t13 + t12 - t23, fmaf(1.875f, P, Q3));
                        const float x16 = x16c * gq * pr.g * g3;
                        const float fd = __fdividef(1.0f, fmaf(6.0f, x16, 1.0f));
                        const float dfd = 32.0f * x16 * fd * fd;
                        const float C9 = -sq * pr.s * s3;
                        const float Et = C9 * A * fd;
                        const float Adfd = A * dfd;
                        const float f1 = -C9 * fmaf(dang1, fd, -Adfd) * id1;
                        const float f3 = -C9 * fmaf(dang3, fd, -Adfd) * id3;
                        const float wE = w * Et;
                        tE += wE;
                        Dsum = fma((double)wE, (double)lam_xy, Dsum);
                        const float w3 = w * f3;
                        tS = fmaf(w, f1 + f3, tS);
                        tUx = fmaf(w3, pr.vx, tUx);
                        tUy = fmaf(w3, pr.vy, tUy);
                        tUz = fmaf(w3, pr.vz, tUz);
                        const float ff3 = wf * f3;
                        tF = fmaf(wf, f1 + f3, tF);
                        tWx = fmaf(ff3, pr.vx, tWx);
                        tWy = fmaf(ff3, pr.vy, tWy);
                        tWz = fmaf(ff3, pr.vz, tWz);
                        tA = fmaf(wf, f1, tA);
                    }
                }
                // carry the tile's FP32 partial sums in FP64
                Esum += tE;
                Ssum += tS;
                Ux += tUx;
                Uy += tUy;
                Uz += tUz;
                Fsum += tF;
                Wx += tWx;
                Wy += tWy;
                Wz += tWz;
                Asum += tA;
            }
            if (active) {
                const double third_d = 1.0 / 3.0;
                atomicAdd(&p.eb[jq], Esum * third_d);
                atomicAdd(&p.gb[jq], 0.5 * (lam_qa * Esum + Dsum));
                atomicAdd(&p.fb[3 * jq], Fsum * vqx_d - Wx);
                atomicAdd(&p.fb[3 * jq + 1], Fsum * vqy_d - Wy);
                atomicAdd(&p.fb[3 * jq + 2], Fsum * vqz_d - Wz);
                ea += 0.5 * Esum * third_d;
                ga += 0.5 * lam_aq * Esum;
                fax -= Asum * vqx_d;
                fay -= Asum * vqy_d;
                faz -= Asum * vqz_d;
                vxx += Ssum * vqx_d * vqx_d - Ux * vqx_d;
                vyy += Ssum * vqy_d * vqy_d - Uy * vqy_d;
                vzz += Ssum * vqz_d * vqz_d - Uz * vqz_d;
                vxy += Ssum * vqx_d * vqy_d - 0.5 * (Ux * vqy_d + Uy * vqx_d);
                vxz += Ssum * vqx_d * vqz_d - 0.5 * (Ux * vqz_d + Uz * vqx_d);
                vyz += Ssum * vqy_d * vqz_d - 0.5 * (Uy * vqz_d + Uz * vqy_d);
            }
        }
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
    for (int o = 16; o > 0; o >>= 1) visits += __shfl_xor_sync(0xffffffffu, visits, o);
    if ((tid & 31) == 0 && p.counters) atomicAdd(p.counters, visits);
}

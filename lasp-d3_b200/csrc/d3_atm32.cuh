// ATM three-body kernel, precision form: the per-visit triplet arithmetic in FP32.
// Same enumeration, schedule, weights and mirror-symmetric accumulation as k_atm
// (d3_atm.cuh); per-entry set-up (C6 of the apex pairs, damping ratios) is done in FP64
// and rounded once. Per-visit sums, dE/dCN included, are kept in FP32 within one
// partner tile and carried across tiles in FP64 (blocked summation, error
// ~ sqrt(tile) * eps_32 per block).
//
// Layout for few instructions per visit: partner records as two float4 and one int2
// (three wide shared-memory loads), C6 rows padded to 8 floats (two 16-byte loads),
// 32-bit in-range masks over tiles padded to a multiple of 32 with far-away dummies.

constexpr int ATM32_NRP = 8; // padded C6 row length (NR <= 7)

template <int NR, bool CENTER>
__global__ void __launch_bounds__(ATM_THREADS) k_atm32(KP p, int tile) {
    extern __shared__ __align__(16) unsigned char smem32[];
    const int ne = p.ne;
    const int tilep = (tile + 31) & ~31;
    float4 *pA = reinterpret_cast<float4 *>(smem32);       // [tilep] vx vy vz d2
    float4 *pB = pA + tilep;                                // [tilep] ir id2 s g
    int2 *pC = reinterpret_cast<int2 *>(pB + tilep);        // [tilep] j t
    float4 *ytile = reinterpret_cast<float4 *>(pC + tilep); // [tilep][ne][2]: C6 row, padded to 8
    double *yapex = reinterpret_cast<double *>(ytile + (size_t)tilep * ne * 2); // [ne][NR]
    float *r0sq = reinterpret_cast<float *>(yapex + ne * NR); // [ne][ne]
    unsigned short *perm = reinterpret_cast<unsigned short *>(r0sq + ((ne * ne + 3) & ~3)); // [ATM_PERM_CAP]
    // per-thread FP64 carries of the entry sums, touched once per partner tile, kept in
    // shared memory to save registers: [11][blockDim]
    double *carry = reinterpret_cast<double *>(perm + ATM_PERM_CAP);
    __shared__ int s_item;
    __shared__ int shell_cnt[ATM_SHELLS], shell_off[ATM_SHELLS];
    __shared__ double red[ATM_THREADS / 32][12];
    const int tid = threadIdx.x;
    if (p.atm_off[p.n] > p.atm_cap) return; // list overflowed: the host grows it and re-runs
    for (int k = tid; k < ne * ne; k += blockDim.x) r0sq[k] = (float)(p.r0ab[k] * p.r0ab[k]);
    const float x16c = (float)(4294967296.0 / 43046721.0); // (4/3)^16
    const float third = 1.0f / 3.0f;
    const float ratm2f = (float)p.ratm2;
    const bool force_scaled = p.atm_force_scaled != 0;
    const bool center = CENTER;
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
        if (!CENTER && m <= p.atm_min_m) continue; // shorter lists: k_atm32b
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
        const int B = blockDim.x;
        double apex[11];
#pragma unroll
        for (int k = 0; k < 11; ++k) apex[k] = 0.0;
        for (int q0 = 0; q0 < m; q0 += blockDim.x) {
            const int qi = q0 + tid;
            const bool active = qi < m;
            const int q = active ? (sorted ? (int)perm[qi] : qi) : -1;
            double vqx_d = 0, vqy_d = 0, vqz_d = 0, lam_qa = 0, lam_aq = 0;
            float vqx = 0.f, vqy = 0.f, vqz = 1e30f, d1 = 1.f, ir1 = 1.f, id1 = 1.f, sq = 0.f, gq = 0.f;
            float wq[ATM32_NRP], dwq[ATM32_NRP];
#pragma unroll
            for (int b = 0; b < ATM32_NRP; ++b) wq[b] = dwq[b] = 0.f;
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
            }
            const bool qa = (jq == a);
#pragma unroll
            for (int k = 0; k < 11; ++k) carry[k * B + tid] = 0.0;
            for (int p0 = 0; p0 < m; p0 += tile) {
                const int cnt = min(tile, m - p0);
                const int cntp = (cnt + 31) & ~31;
                __syncthreads();
                for (int k = tid; k < cntp; k += blockDim.x) {
                    if (k >= cnt) {
                        // padding: far-away dummies fail every distance test
                        pA[k] = make_float4(1e30f, 1e30f, 1e30f, 1.f);
                        continue;
                    }
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
                    pA[k] = make_float4((float)vx, (float)vy, (float)vz, (float)d2);
                    pB[k] = make_float4((float)(1.0 / sqrt(d2)), (float)(1.0 / d2), (float)sqrt(c6),
                                        (float)pow((double)r0sq[ta * ne + tp] / d2, 8.0 / 3.0));
                    pC[k] = make_int2(jp, tp);
                    const float *ysrc = p.Y32 + (size_t)jp * ne * NR;
                    float *ydst = reinterpret_cast<float *>(ytile + (size_t)k * ne * 2);
                    for (int t = 0; t < ne; ++t)
#pragma unroll
                        for (int b = 0; b < ATM32_NRP; ++b) ydst[t * ATM32_NRP + b] = b < NR ? ysrc[t * NR + b] : 0.f;
                }
                __syncthreads();
                float tE = 0.f, tD = 0.f, tS = 0.f, tUx = 0.f, tUy = 0.f, tUz = 0.f, tF = 0.f, tWx = 0.f, tWy = 0.f,
                      tWz = 0.f, tA = 0.f;
                for (int s0 = 0; s0 < cntp; s0 += 32) {
                    // in-range mask over 32 partners (upper bound only; the exact test is below)
                    unsigned mask = 0u;
#pragma unroll 4
                    for (int k = 0; k < 32; ++k) {
                        const float4 pa = pA[s0 + k];
                        const float dx = vqx - pa.x, dy = vqy - pa.y, dz = vqz - pa.z;
                        const float d3 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        mask |= (d3 <= ratm2f) ? (1u << k) : 0u;
                    }
                    while (__any_sync(0xffffffffu, mask != 0u)) {
                        if (mask == 0u) continue;
                        const int k = s0 + __ffs(mask) - 1;
                        mask &= mask - 1u;
                        const float4 pa = pA[k];
                        const float rx = vqx - pa.x, ry = vqy - pa.y, rz = vqz - pa.z;
                        const float d3 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
                        if (d3 < 1e-12f) continue; // the entry itself
                        ++visits;
                        const float4 pb = pB[k];
                        const int2 pc = pC[k];
                        const float ir3 = sfu_rsqrt(d3);
                        const float id3 = ir3 * ir3;
                        const float4 *yr = ytile + ((size_t)k * ne + tq) * 2;
                        const float4 y0 = yr[0], y1 = yr[1];
                        float c6 = y0.x * wq[0];
                        float dc6 = y0.x * dwq[0];
                        c6 = fmaf(y0.y, wq[1], c6);
                        dc6 = fmaf(y0.y, dwq[1], dc6);
                        c6 = fmaf(y0.z, wq[2], c6);
                        dc6 = fmaf(y0.z, dwq[2], dc6);
                        c6 = fmaf(y0.w, wq[3], c6);
                        dc6 = fmaf(y0.w, dwq[3], dc6);
                        c6 = fmaf(y1.x, wq[4], c6);
                        dc6 = fmaf(y1.x, dwq[4], dc6);
                        if (NR > 5) {
                            c6 = fmaf(y1.y, wq[5], c6);
                            dc6 = fmaf(y1.y, dwq[5], dc6);
                            c6 = fmaf(y1.z, wq[6], c6);
                            dc6 = fmaf(y1.z, dwq[6], dc6);
                        }
                        const float is3 = sfu_rsqrt(c6);
                        const float s3 = c6 * is3;
                        const float lam_xy = dc6 * is3 * is3;
                        const float u = r0sq[tq * ne + pc.y] * id3;
                        const float g3 = u * u * u * sfu_exp2(sfu_log2(u) * (-1.0f / 3.0f));
                        // reference scale factors (src/d3_kernel.cu:1282-1290) as pair weights
                        const bool same = (jq == pc.x);
                        const bool apex_img = qa | (pc.x == a);
                        const float w = center ? third : (same ? (qa ? third : 1.0f) : (apex_img ? 0.5f : 1.0f));
                        const float wf = (force_scaled || center) ? w : (same ? 2.0f : 1.0f);
                        const float d2 = pa.w;
                        const float irsq = id1 * pb.y * id3;
                        const float ir9 = irsq * ir1 * pb.x * ir3;
                        const float t1 = d1 + d2 - d3, t2 = d1 - d2 + d3, t3 = -d1 + d2 + d3;
                        const float t12 = t1 * t2, t13 = t1 * t3, t23 = t2 * t3;
                        const float P = t12 * t3;
                        const float A = fmaf(0.375f * P, irsq, 1.0f) * ir9;
                        const float q52 = ir9 * irsq;
                        const float Q3 = 3.0f * d1 * d2 * d3;
                        const float base = fmaf(1.875f, P, Q3);
                        const float dang1 = q52 * fmaf(-0.75f * d1, t23 + t13 - t12, base);
                        const float dang3 = q52 * fmaf(-0.75f * d3, t13 + t12 - t23, base);
                        const float x16 = x16c * gq * pb.w * g3;
                        const float fd = sfu_rcp(fmaf(6.0f, x16, 1.0f));
                        const float dfd = 32.0f * x16 * fd * fd;
                        const float C9 = -sq * pb.z * s3;
                        const float Et = C9 * A * fd;
                        const float Adfd = A * dfd;
                        const float f1 = -C9 * fmaf(dang1, fd, -Adfd) * id1;
                        const float f3 = -C9 * fmaf(dang3, fd, -Adfd) * id3;
                        const float wE = w * Et;
                        tE += wE;
                        tD = fmaf(wE, lam_xy, tD);
                        const float w3 = w * f3;
                        tS = fmaf(w, f1 + f3, tS);
                        tUx = fmaf(w3, pa.x, tUx);
                        tUy = fmaf(w3, pa.y, tUy);
                        tUz = fmaf(w3, pa.z, tUz);
                        const float ff3 = wf * f3;
                        tF = fmaf(wf, f1 + f3, tF);
                        tWx = fmaf(ff3, pa.x, tWx);
                        tWy = fmaf(ff3, pa.y, tWy);
                        tWz = fmaf(ff3, pa.z, tWz);
                        tA = fmaf(wf, f1, tA);
                    }
                }
                // carry the tile's FP32 partial sums in FP64
                const float tv[11] = {tE, tD, tS, tUx, tUy, tUz, tF, tWx, tWy, tWz, tA};
#pragma unroll
                for (int k = 0; k < 11; ++k) carry[k * B + tid] += (double)tv[k];
            }
            if (active) {
                const double Esum = carry[0 * B + tid], Dsum = carry[1 * B + tid], Ssum = carry[2 * B + tid];
                const double Ux = carry[3 * B + tid], Uy = carry[4 * B + tid], Uz = carry[5 * B + tid];
                const double Fsum = carry[6 * B + tid], Wx = carry[7 * B + tid], Wy = carry[8 * B + tid],
                             Wz = carry[9 * B + tid], Asum = carry[10 * B + tid];
                const double third_d = 1.0 / 3.0;
                atomicAdd(&p.eb[jq], Esum * third_d);
                atomicAdd(&p.gb[jq], 0.5 * (lam_qa * Esum + Dsum));
                atomicAdd(&p.fb[3 * jq], Fsum * vqx_d - Wx);
                atomicAdd(&p.fb[3 * jq + 1], Fsum * vqy_d - Wy);
                atomicAdd(&p.fb[3 * jq + 2], Fsum * vqz_d - Wz);
                const double av[11] = {0.5 * Esum * third_d,
                                       0.5 * lam_aq * Esum,
                                       -Asum * vqx_d,
                                       -Asum * vqy_d,
                                       -Asum * vqz_d,
                                       Ssum * vqx_d * vqx_d - Ux * vqx_d,
                                       Ssum * vqy_d * vqy_d - Uy * vqy_d,
                                       Ssum * vqz_d * vqz_d - Uz * vqz_d,
                                       Ssum * vqx_d * vqy_d - 0.5 * (Ux * vqy_d + Uy * vqx_d),
                                       Ssum * vqx_d * vqz_d - 0.5 * (Ux * vqz_d + Uz * vqx_d),
                                       Ssum * vqy_d * vqz_d - 0.5 * (Uy * vqz_d + Uz * vqy_d)};
#pragma unroll
                for (int k = 0; k < 11; ++k) apex[k] += av[k];
            }
        }
        double vals[11];
#pragma unroll
        for (int k = 0; k < 11; ++k) vals[k] = apex[k];
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

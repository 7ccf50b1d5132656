// Two-body pass on spatially compact atom groups (included by d3_engine.cu after the
// per-atom pair kernels; replaces the reference's two_body_kernel, src/d3_kernel.cu:997-1197).
//
// Groups. The bins of a structure are taken in super-rows of gy x gz bin rows (y, z);
// within a super-row the atoms are ordered column by column along x (column = the gy gz
// bins of one x index) and cut into consecutive groups of 32. A group is therefore a
// compact block of about 32 atoms (2 x 2 rows and one or two columns for the benchmark
// box) whose candidate partners are given by one merged stencil: for every row offset
// (dy, dz) relative to the super-row's first row, the union of the x ranges its member
// rows need, widened by the group's own x extent. Every candidate (j, image) appears once
// in that stencil, so a distance test per (i, j) pair is the only filter.
//
// Work. A work item is (group, slice of the stencil rows): one warp, lane L owns the
// group's atom L, partners are staged 32 at a time in the warp's shared memory and visited
// by all lanes together. Items are taken from a counter by persistent warps. Each item
// writes its lanes' sums to its slice's row of a partial array; k_group_reduce adds the
// slices of every atom in a fixed order, so results do not depend on scheduling.
//
// Three passes use the same groups: coordination numbers (k_cn_g, rc_CN stencil, the
// reference's coordination_number_kernel, src/d3_kernel.cu:544-683), the two-body term
// (k_twobody_g, rc stencil; staged partner data: position and the partner's C6 rows at
// every type, where lanes of different types read distinct banks and lanes of one type the
// same word) and the dE/dCN chain rule (k_chain_g, rc_CN stencil, the reference's
// three_body_kernel, src/d3_kernel.cu:1511-1698; staged: position and dE/dCN).

constexpr int PAIRS_MAX_TYPES = 8;    // staged C6 rows per partner: ne * NR values
constexpr int PAIRS_WARPS = 8;        // warps per CTA
constexpr int PAIRS_NSUM = 11;        // e, g, f[3], v[6] per atom and slice (two-body; CN
                                      // uses 1, the chain rule 9 of the 11)

// one super-row: structure, first bin row (y, z) and its row counts (ny | nz << 8)
// one group:     super-row, bx_lo | bx_hi << 16, position of the first atom in column
//                bx_lo's atom sequence, atom count (<= 32)

// Cut the super-rows into groups (one thread per super-row).
__global__ void k_groups(KP p) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= p.nsrow) return;
    const int4 sr = p.srows[r];
    const SG &g = p.sg[sr.x];
    const int ny = sr.w & 0xff, nz = (sr.w >> 8) & 0xff;
    const int *bs = p.bin_start + g.bin_base;
    int lo = 0, skip = 0, cnt = 0, last = 0;
    for (int bx = 0; bx < g.nb[0]; ++bx) {
        int c = 0;
        for (int oz = 0; oz < nz; ++oz)
            for (int oy = 0; oy < ny; ++oy) {
                const int rb = g.nb[0] * ((sr.y + oy) + g.nb[1] * (sr.z + oz));
                c += bs[rb + bx + 1] - bs[rb + bx];
            }
        int used = 0;
        while (used < c) {
            if (cnt == 0) {
                lo = bx;
                skip = used;
            }
            const int take = min(32 - cnt, c - used);
            cnt += take;
            used += take;
            last = bx;
            if (cnt == 32) {
                const int slot = atomicAdd(p.gcount, 1);
                p.groups[slot] = make_int4(r, lo | (bx << 16), skip, 32);
                cnt = 0;
            }
        }
    }
    if (cnt > 0) {
        const int slot = atomicAdd(p.gcount, 1);
        p.groups[slot] = make_int4(r, lo | (last << 16), skip, cnt);
    }
}

// binned index of atom q (0-based, q < group count) of a group
__device__ __forceinline__ int group_atom(const KP &p, const SG &g, int4 sr, int bx_lo, int skip, int q) {
    const int ny = sr.w & 0xff, nz = (sr.w >> 8) & 0xff;
    const int *bs = p.bin_start + g.bin_base;
    q += skip;
    for (int bx = bx_lo; bx < g.nb[0]; ++bx)
        for (int oz = 0; oz < nz; ++oz)
            for (int oy = 0; oy < ny; ++oy) {
                const int b = g.nb[0] * ((sr.y + oy) + g.nb[1] * (sr.z + oz)) + bx;
                const int c = bs[b + 1] - bs[b];
                if (q < c) return bs[b] + q;
                q -= c;
            }
    return -1;
}

template <bool F64>
struct PairReal;
template <>
struct PairReal<false> {
    using R = float;
    using R4 = float4;
};
template <>
struct PairReal<true> {
    using R = double;
    using R4 = double4;
};

// One (i, j) pair of the two-body term: energy (half), dE/dCN_i, force scalar fs with
// F_i += fs r_ij and virial += fs r_ij (x) r_ij. y: partner's C6 row at the type of i.
template <int NR, typename R>
__device__ __forceinline__ void pair_term(const KP &p, R r2, const R *y, const R *wi, const R *dwi, R A6_or_R0,
                                          R A8, R rr, R &e_half, R &G, R &fs) {
    R c6 = 0, dc6 = 0;
#pragma unroll
    for (int b = 0; b < NR; ++b) {
        c6 = fma(y[b], wi[b], c6);
        dc6 = fma(y[b], dwi[b], dc6);
    }
    const R c8 = c6 * rr, dc8 = dc6 * rr;
    const R s6 = (R)p.s6, s8 = (R)p.s8;
    R E6, E8;
    if (p.damping == 1) {
        const R r4 = r2 * r2, r6 = r4 * r2, r8 = r4 * r4;
        R i6, i8;
        if constexpr (sizeof(R) == 4) {
            i6 = sfu_rcp(r6 + A6_or_R0);
            i8 = sfu_rcp(r8 + A8);
        } else {
            i6 = 1.0 / (r6 + A6_or_R0);
            i8 = 1.0 / (r8 + A8);
        }
        E6 = s6 * c6 * i6;
        E8 = s8 * c8 * i8;
        G = s6 * dc6 * i6 + s8 * dc8 * i8;
        fs = (R)-6 * E6 * r4 * i6 - (R)8 * E8 * r6 * i8;
    } else {
        R ir;
        if constexpr (sizeof(R) == 4)
            ir = sfu_rsqrt(r2);
        else
            ir = 1.0 / sqrt(r2);
        const R ir2 = ir * ir, ir6 = ir2 * ir2 * ir2, ir8 = ir6 * ir2;
        const R R0 = A6_or_R0;
        const R x6 = (R)p.p1 * R0 * ir, x8 = (R)p.p2 * R0 * ir;
        const R x6_2 = x6 * x6, x6_4 = x6_2 * x6_2, x6_8 = x6_4 * x6_4, x6_14 = x6_8 * x6_4 * x6_2;
        const R x8_2 = x8 * x8, x8_4 = x8_2 * x8_2, x8_8 = x8_4 * x8_4, x8_16 = x8_8 * x8_8;
        R f6, f8;
        if constexpr (sizeof(R) == 4) {
            f6 = sfu_rcp(fmaf(6.0f, x6_14, 1.0f));
            f8 = sfu_rcp(fmaf(6.0f, x8_16, 1.0f));
        } else {
            f6 = 1.0 / (1.0 + 6.0 * x6_14);
            f8 = 1.0 / (1.0 + 6.0 * x8_16);
        }
        const R df6 = (R)84 * f6 * f6 * x6_14 * ir, df8 = (R)96 * f8 * f8 * x8_16 * ir;
        E6 = s6 * c6 * f6 * ir6;
        E8 = s8 * c8 * f8 * ir8;
        G = s6 * f6 * dc6 * ir6 + s8 * f8 * dc8 * ir8;
        fs = s6 * c6 * ((R)-6 * f6 * ir8 + df6 * ir6 * ir) + s8 * c8 * ((R)-8 * f8 * ir8 * ir2 + df8 * ir8 * ir);
    }
    e_half = (R)0.5 * (E6 + E8);
}

// shared memory of one warp: 32 partner positions, their C6 rows at every type (two-body)
// or their dE/dCN (chain rule)
template <bool F64>
__host__ __device__ constexpr size_t pairs_warp_bytes(int ne, int NR) {
    return 32 * (F64 ? sizeof(double4) : sizeof(float4)) +
           (size_t)32 * (ne * NR > 1 ? ne * NR : 1) * (F64 ? sizeof(double) : sizeof(float)) + 32 * sizeof(double);
}

// One work item of a grouped pass, as the lanes of a warp see it.
struct GroupItem {
    int i;           // this lane's atom (binned), -1 for lanes past the group's count
    int sl;          // stencil-row slice
    int4 sr;         // the group's super-row
    int bx_lo, bx_hi;
    const SG *g;
    bool own;        // sharded evaluation: this rank owns the group's two-body and
                     // chain-rule sums (every rank still covers every group in CN and lists)
};

// Owner rank of a group in a sharded evaluation: a hash of the group's super-row, first
// column and skip count (fields that k_groups writes the same way on every rank, unlike
// the group's slot), so that the ranks partition the groups without talking.
__device__ __forceinline__ int group_owner(int4 grp, int world) {
    const unsigned h = (unsigned)grp.x * 0x9E3779B1u ^ (unsigned)(grp.y & 0xffff) * 0x85EBCA77u ^
                       (unsigned)grp.z * 0xC2B2AE3Du;
    return (int)((h ^ (h >> 15)) % (unsigned)world);
}

__device__ __forceinline__ bool next_item(const KP &p, int *work, GroupItem &it) {
    const int lane = threadIdx.x & 31;
    const int S = p.gslices;
    int k = 0;
    if (lane == 0) k = atomicAdd(work, 1);
    k = __shfl_sync(0xffffffffu, k, 0);
    if (k >= *p.gcount * S) return false;
    const int gi = k / S;
    it.sl = k - gi * S;
    const int4 grp = p.groups[gi];
    it.sr = p.srows[grp.x];
    it.g = &p.sg[it.sr.x];
    it.bx_lo = grp.y & 0xffff;
    it.bx_hi = grp.y >> 16;
    it.i = lane < grp.w ? group_atom(p, *it.g, it.sr, it.bx_lo, grp.z, lane) : -1;
    it.own = p.shard_world <= 1 || group_owner(grp, p.shard_world) == p.shard_rank;
    return true;
}

// Every contiguous candidate range of the item's slice of a block stencil: body(base, m,
// ox, oy, oz, px, Ty, Tz) for each chunk of m <= 32 partners starting at binned index base,
// with this lane's origin o = x_i - T h (rounded once per range). Ranges whose image lies
// outside the reference's image box are skipped whole unless some atom was given outside
// the cell (box_pair: the caller tests each pair).
template <typename R, typename R4, class Body>
__device__ __forceinline__ void group_ranges(const KP &p, const GroupItem &it, const int4 *rows, int nrows,
                                             bool box_pair, const R4 &xi, Body &&body) {
    const SG &g = *it.g;
    const int S = p.gslices;
    const int nb0 = g.nb[0], nb1 = g.nb[1], nb2 = g.nb[2];
    const int *bstart = p.bin_start + g.bin_base;
    for (int r = it.sl; r < nrows; r += S) {
        const int4 row = rows[r];
        const int yy = it.sr.y + row.x, zz = it.sr.z + row.y;
        const int Ty = floordiv(yy, nb1), Tz = floordiv(zz, nb2);
        const int byy = yy - Ty * nb1, bzz = zz - Tz * nb2;
        const int xlo = it.bx_lo + row.z, xhi = it.bx_hi + row.w;
        const int plo = floordiv(xlo, nb0), phi = floordiv(xhi, nb0);
        const int rowbase = nb0 * (byy + nb1 * bzz);
        for (int px = plo; px <= phi; ++px) {
            if (g.box_mode && !box_pair && (abs(px) > g.half[0] || abs(Ty) > g.half[1] || abs(Tz) > g.half[2]))
                continue;
            const int a = max(xlo, px * nb0) - px * nb0;
            const int b = min(xhi, px * nb0 + nb0 - 1) - px * nb0;
            const int jlo = bstart[rowbase + a], jhi = bstart[rowbase + b + 1];
            if (jlo >= jhi) continue;
            const double shx = px * g.h[0] + Ty * g.h[3] + Tz * g.h[6];
            const double shy = px * g.h[1] + Ty * g.h[4] + Tz * g.h[7];
            const double shz = px * g.h[2] + Ty * g.h[5] + Tz * g.h[8];
            const R ox = (R)((double)xi.x - shx), oy = (R)((double)xi.y - shy), oz = (R)((double)xi.z - shz);
            for (int base = jlo; base < jhi; base += 32) body(base, min(32, jhi - base), ox, oy, oz, px, Ty, Tz);
        }
    }
}

// CN term of one pair: value and (d CN / d r) / r; optional tanh^3 smooth cutoff (the
// reference's SMOOTH_CUTOFF_CN)
template <typename R>
__device__ __forceinline__ R cn_pair(const KP &p, R r2, R rsum, R *dcn_over_r) {
    if constexpr (sizeof(R) == 8) {
        return cn_term(p, sqrt(r2), rsum, dcn_over_r);
    } else {
        return cn_term32(p, r2, rsum, dcn_over_r);
    }
}

template <int NR, bool F64>
__global__ void __launch_bounds__(PAIRS_WARPS * 32, F64 ? 1 : 2) k_twobody_g(KP p, int *work) {
    using R = typename PairReal<F64>::R;
    using R4 = typename PairReal<F64>::R4;
    extern __shared__ __align__(16) unsigned char smp[];
    const int ne = p.ne;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // per type pair: BJ A^6, A^8 (zero damping: R0) and 3 r2r4_i r2r4_j
    R *ptab = reinterpret_cast<R *>(smp);
    for (int k = threadIdx.x; k < ne * ne; k += blockDim.x) {
        const double *pa = p.pairA + (size_t)k * 4;
        ptab[3 * k] = (R)pa[0];
        ptab[3 * k + 1] = (R)pa[1];
        ptab[3 * k + 2] = (R)(3.0 * p.r2r4[k / ne] * p.r2r4[k % ne]);
    }
    __syncthreads();
    const size_t tab_bytes = ((size_t)3 * ne * ne * sizeof(R) + 15) & ~(size_t)15;
    unsigned char *wb = smp + tab_bytes + (size_t)warp * pairs_warp_bytes<F64>(ne, NR);
    R4 *sP = reinterpret_cast<R4 *>(wb);
    R *sY = reinterpret_cast<R *>(wb + 32 * sizeof(R4));
    const R4 *xsrc = F64 ? reinterpret_cast<const R4 *>(p.xs) : reinterpret_cast<const R4 *>(p.xs32);
    const R *Ysrc = F64 ? reinterpret_cast<const R *>(p.Y) : reinterpret_cast<const R *>(p.Y32);
    const R *wsrc = F64 ? reinterpret_cast<const R *>(p.w) : reinterpret_cast<const R *>(p.w32);
    const R *dwsrc = F64 ? reinterpret_cast<const R *>(p.dw) : reinterpret_cast<const R *>(p.dw32);
    const int rowlen = ne * NR;
    const R rc2 = (R)p.rc2;
    unsigned long long npair = 0;
    GroupItem it;
    while (next_item(p, work, it)) {
        const int i = it.i;
        const bool iv = i >= 0;
        R4 xi;
        int ti = 0;
        R wi[NR], dwi[NR];
        int4 si = make_int4(0, 0, 0, 0);
        if (iv) {
            xi = xsrc[i];
            ti = (int)xi.w;
            si = p.shift[i];
#pragma unroll
            for (int b = 0; b < NR; ++b) {
                wi[b] = wsrc[(size_t)i * NR + b];
                dwi[b] = dwsrc[(size_t)i * NR + b];
            }
        } else {
            xi.x = xi.y = xi.z = (R)0;
            xi.w = (R)0;
#pragma unroll
            for (int b = 0; b < NR; ++b) wi[b] = dwi[b] = (R)0;
        }
        const SG &g = *it.g;
        const bool box_pair = g.box_mode && p.anyshift[it.sr.x];
        double E = 0, Gd = 0, FX = 0, FY = 0, FZ = 0, V[6] = {0, 0, 0, 0, 0, 0};
        if (it.own)
        group_ranges<R, R4>(p, it, p.stencils + g.st2b_off, g.st2b_n, box_pair, xi,
                            [&](int base, int m, R ox, R oy, R oz, int px, int Ty, int Tz) {
            __syncwarp();
            if (lane < m) sP[lane] = xsrc[base + lane];
            {
                const R *src = Ysrc + (size_t)base * rowlen;
                const int tot = m * rowlen;
                for (int k = lane; k < tot; k += 32) sY[k] = src[k];
            }
            __syncwarp();
            R e = 0, fx = 0, fy = 0, fz = 0, vxx = 0, vyy = 0, vzz = 0, vxy = 0, vxz = 0, vyz = 0;
            // two partners per iteration (independent dependency chains); an inactive one
            // runs on a stand-in distance (rc^2, finite terms) and its sums are dropped
            for (int jj = 0; jj < m; jj += 2) {
                const int j1 = jj + 1 < m ? jj + 1 : jj;
                const R4 x0 = sP[jj], x1 = sP[j1];
                const R dx0 = ox - x0.x, dy0 = oy - x0.y, dz0 = oz - x0.z;
                const R dx1 = ox - x1.x, dy1 = oy - x1.y, dz1 = oz - x1.z;
                const R r20 = fma(dx0, dx0, fma(dy0, dy0, dz0 * dz0));
                const R r21 = fma(dx1, dx1, fma(dy1, dy1, dz1 * dz1));
                bool act0 = iv && r20 < rc2 && r20 > (R)0;
                bool act1 = iv && j1 != jj && r21 < rc2 && r21 > (R)0;
                if (box_pair) {
                    if (act0) act0 = in_box(g, si, p.shift[base + jj], px, Ty, Tz);
                    if (act1) act1 = in_box(g, si, p.shift[base + j1], px, Ty, Tz);
                }
                if (!(act0 || act1)) continue;
                npair += (act0 ? 1 : 0) + (act1 ? 1 : 0);
                const R *tp0 = ptab + 3 * (ti * ne + (int)x0.w), *tp1 = ptab + 3 * (ti * ne + (int)x1.w);
                R eh0, Gt0, fs0, eh1, Gt1, fs1;
                pair_term<NR, R>(p, act0 ? r20 : rc2, sY + jj * rowlen + ti * NR, wi, dwi, tp0[0], tp0[1], tp0[2], eh0,
                                 Gt0, fs0);
                pair_term<NR, R>(p, act1 ? r21 : rc2, sY + j1 * rowlen + ti * NR, wi, dwi, tp1[0], tp1[1], tp1[2], eh1,
                                 Gt1, fs1);
                if (!act0) eh0 = Gt0 = fs0 = (R)0;
                if (!act1) eh1 = Gt1 = fs1 = (R)0;
                e += eh0 + eh1;
                Gd += (double)Gt0 + (double)Gt1;
                fx = fma(fs0, dx0, fma(fs1, dx1, fx));
                fy = fma(fs0, dy0, fma(fs1, dy1, fy));
                fz = fma(fs0, dz0, fma(fs1, dz1, fz));
                const R fdx0 = fs0 * dx0, fdy0 = fs0 * dy0, fdx1 = fs1 * dx1, fdy1 = fs1 * dy1;
                vxx = fma(fdx0, dx0, fma(fdx1, dx1, vxx));
                vyy = fma(fdy0, dy0, fma(fdy1, dy1, vyy));
                vzz = fma(fs0 * dz0, dz0, fma(fs1 * dz1, dz1, vzz));
                vxy = fma(fdx0, dy0, fma(fdx1, dy1, vxy));
                vxz = fma(fdx0, dz0, fma(fdx1, dz1, vxz));
                vyz = fma(fdy0, dz0, fma(fdy1, dz1, vyz));
            }
            // blocked summation: 32-partner sums carried in FP64
            E += e;
            FX += fx;
            FY += fy;
            FZ += fz;
            V[0] += vxx;
            V[1] += vyy;
            V[2] += vzz;
            V[3] += vxy;
            V[4] += vxz;
            V[5] += vyz;
        });
        if (iv) {
            double *o = p.gpart + ((size_t)it.sl * p.n + i) * PAIRS_NSUM;
            o[0] = E;
            o[1] = Gd;
            o[2] = FX;
            o[3] = FY;
            o[4] = FZ;
#pragma unroll
            for (int k = 0; k < 6; ++k) o[5 + k] = V[k];
        }
    }
    for (int o = 16; o > 0; o >>= 1) npair += __shfl_xor_sync(0xffffffffu, npair, o);
    if (lane == 0 && npair) atomicAdd(&p.counters[1], npair);
}

// coordination numbers on atom groups (rc_CN stencil): 0 < r^2 <= rc_CN^2
template <bool F64>
__global__ void __launch_bounds__(PAIRS_WARPS * 32, 2) k_cn_g(KP p, int *work) {
    using R = typename PairReal<F64>::R;
    using R4 = typename PairReal<F64>::R4;
    extern __shared__ __align__(16) unsigned char smp[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    R *rcov = reinterpret_cast<R *>(smp);
    for (int k = threadIdx.x; k < p.ne; k += blockDim.x) rcov[k] = (R)p.rcov[k];
    __syncthreads();
    const size_t tab_bytes = ((size_t)PAIRS_MAX_TYPES * sizeof(double) + 15) & ~(size_t)15;
    R4 *sP = reinterpret_cast<R4 *>(smp + tab_bytes + (size_t)warp * 32 * sizeof(R4));
    const R4 *xsrc = F64 ? reinterpret_cast<const R4 *>(p.xs) : reinterpret_cast<const R4 *>(p.xs32);
    const R rcn2 = (R)p.rcn2;
    unsigned long long npair = 0;
    GroupItem it;
    while (next_item(p, work, it)) {
        const int i = it.i;
        const bool iv = i >= 0;
        R4 xi;
        xi.x = xi.y = xi.z = xi.w = (R)0;
        int4 si = make_int4(0, 0, 0, 0);
        if (iv) {
            xi = xsrc[i];
            si = p.shift[i];
        }
        const R ri = rcov[(int)xi.w];
        const SG &g = *it.g;
        const bool box_pair = g.box_mode && p.anyshift[it.sr.x];
        double CN = 0;
        group_ranges<R, R4>(p, it, p.stencils + g.stcb_off, g.stcb_n, box_pair, xi,
                            [&](int base, int m, R ox, R oy, R oz, int px, int Ty, int Tz) {
            __syncwarp();
            if (lane < m) sP[lane] = xsrc[base + lane];
            __syncwarp();
            R c = 0;
            for (int jj = 0; jj < m; ++jj) {
                const R4 xj = sP[jj];
                const R dx = ox - xj.x, dy = oy - xj.y, dz = oz - xj.z;
                const R r2 = fma(dx, dx, fma(dy, dy, dz * dz));
                bool act = iv && r2 <= rcn2 && r2 > (R)0;
                if (box_pair && act) act = in_box(g, si, p.shift[base + jj], px, Ty, Tz);
                if (!act) continue;
                ++npair;
                R d;
                c += cn_pair<R>(p, r2, ri + rcov[(int)xj.w], &d);
            }
            CN += c;
        });
        if (iv) p.gpart[((size_t)it.sl * p.n + i) * PAIRS_NSUM] = CN;
    }
    for (int o = 16; o > 0; o >>= 1) npair += __shfl_xor_sync(0xffffffffu, npair, o);
    if (lane == 0 && npair) atomicAdd(&p.counters[2], npair);
}

// dE/dCN chain rule on atom groups (rc_CN stencil): F_i += (dE/dCN_i + dE/dCN_j) dCN_ij/dr r_ij / r
template <bool F64>
__global__ void __launch_bounds__(PAIRS_WARPS * 32, 2) k_chain_g(KP p, const double *Gd, int *work) {
    using R = typename PairReal<F64>::R;
    using R4 = typename PairReal<F64>::R4;
    extern __shared__ __align__(16) unsigned char smp[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    R *rcov = reinterpret_cast<R *>(smp);
    for (int k = threadIdx.x; k < p.ne; k += blockDim.x) rcov[k] = (R)p.rcov[k];
    __syncthreads();
    const size_t tab_bytes = ((size_t)PAIRS_MAX_TYPES * sizeof(double) + 15) & ~(size_t)15;
    unsigned char *wb = smp + tab_bytes + (size_t)warp * 32 * (sizeof(R4) + sizeof(double));
    R4 *sP = reinterpret_cast<R4 *>(wb);
    double *sG = reinterpret_cast<double *>(wb + 32 * sizeof(R4));
    const R4 *xsrc = F64 ? reinterpret_cast<const R4 *>(p.xs) : reinterpret_cast<const R4 *>(p.xs32);
    const R rcn2 = (R)p.rcn2;
    GroupItem it;
    while (next_item(p, work, it)) {
        const int i = it.i;
        const bool iv = i >= 0;
        R4 xi;
        xi.x = xi.y = xi.z = xi.w = (R)0;
        int4 si = make_int4(0, 0, 0, 0);
        double gi = 0;
        if (iv) {
            xi = xsrc[i];
            si = p.shift[i];
            gi = Gd[i];
        }
        const R ri = rcov[(int)xi.w];
        const SG &g = *it.g;
        const bool box_pair = g.box_mode && p.anyshift[it.sr.x];
        double F[3] = {0, 0, 0}, V[6] = {0, 0, 0, 0, 0, 0};
        if (it.own)
        group_ranges<R, R4>(p, it, p.stencils + g.stcb_off, g.stcb_n, box_pair, xi,
                            [&](int base, int m, R ox, R oy, R oz, int px, int Ty, int Tz) {
            __syncwarp();
            if (lane < m) {
                sP[lane] = xsrc[base + lane];
                sG[lane] = Gd[base + lane];
            }
            __syncwarp();
            R fx = 0, fy = 0, fz = 0, vxx = 0, vyy = 0, vzz = 0, vxy = 0, vxz = 0, vyz = 0;
            for (int jj = 0; jj < m; ++jj) {
                const R4 xj = sP[jj];
                const R dx = ox - xj.x, dy = oy - xj.y, dz = oz - xj.z;
                const R r2 = fma(dx, dx, fma(dy, dy, dz * dz));
                bool act = iv && r2 <= rcn2 && r2 > (R)0;
                if (box_pair && act) act = in_box(g, si, p.shift[base + jj], px, Ty, Tz);
                if (!act) continue;
                R dcn;
                cn_pair<R>(p, r2, ri + rcov[(int)xj.w], &dcn);
                const R dE = (R)(gi + sG[jj]) * dcn;
                const R fdx = dE * dx, fdy = dE * dy;
                fx += fdx;
                fy += fdy;
                fz = fma(dE, dz, fz);
                vxx = fma(fdx, dx, vxx);
                vyy = fma(fdy, dy, vyy);
                vzz = fma(dE * dz, dz, vzz);
                vxy = fma(fdx, dy, vxy);
                vxz = fma(fdx, dz, vxz);
                vyz = fma(fdy, dz, vyz);
            }
            F[0] += fx;
            F[1] += fy;
            F[2] += fz;
            V[0] += vxx;
            V[1] += vyy;
            V[2] += vzz;
            V[3] += vxy;
            V[4] += vxz;
            V[5] += vyz;
        });
        if (iv) {
            double *o = p.gpart + ((size_t)it.sl * p.n + i) * PAIRS_NSUM;
#pragma unroll
            for (int k = 0; k < 3; ++k) o[k] = F[k];
#pragma unroll
            for (int k = 0; k < 6; ++k) o[3 + k] = V[k];
        }
    }
}

// per atom: the slices' sums in a fixed order. what: 0 two-body (energy, dE/dCN, force,
// virial), 1 CN, 2 chain rule (force, virial)
__global__ void k_group_reduce(KP p, int what) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int nsum = what == 0 ? PAIRS_NSUM : (what == 1 ? 1 : 9);
    double acc[PAIRS_NSUM];
#pragma unroll
    for (int k = 0; k < PAIRS_NSUM; ++k) acc[k] = 0.0;
    for (int s = 0; s < p.gslices; ++s) {
        const double *o = p.gpart + ((size_t)s * p.n + i) * PAIRS_NSUM;
#pragma unroll
        for (int k = 0; k < PAIRS_NSUM; ++k)
            if (k < nsum) acc[k] += o[k];
    }
    const double sc = -1.0 / (2.0 * p.sg[p.sid[i]].vol);
    if (what == 1) {
        p.cn[i] = acc[0];
    } else if (what == 0) {
        p.e2[i] = acc[0];
        p.g2[i] = acc[1];
        p.f2[3 * i] = acc[2];
        p.f2[3 * i + 1] = acc[3];
        p.f2[3 * i + 2] = acc[4];
        double *v = p.v2 + 6 * (size_t)i;
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = acc[5 + k] * sc;
    } else {
        p.fc[3 * i] = acc[0];
        p.fc[3 * i + 1] = acc[1];
        p.fc[3 * i + 2] = acc[2];
        double *v = p.vc + 6 * (size_t)i;
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = acc[3 + k] * sc;
    }
}

// ATM half lists on atom groups (rc_ATM stencil): for apex a the entries (j, T) with j <= a in
// caller order (all of them in centre mode) and 1e-12 <= r^2 <= rc_ATM^2, the distance
// evaluated as the per-apex kernel does (x_a - (x_j + T h)). Count pass: counts per
// (stencil slice, apex) into the partial array; k_atm_list_prefix turns them into offsets
// within the apex and the apex totals; fill pass: every lane writes its apex's entries of
// its slice at atm_off[a] + that offset, so each list is contiguous and its order fixed.
template <bool FILL>
__global__ void __launch_bounds__(PAIRS_WARPS * 32, 2) k_atm_list_g(KP p, int *work) {
    extern __shared__ __align__(16) unsigned char smp[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double4 *sP = reinterpret_cast<double4 *>(smp + (size_t)warp * 32 * (sizeof(double4) + sizeof(int)));
    int *sO = reinterpret_cast<int *>(sP + 32);
    int *gcnt = reinterpret_cast<int *>(p.gpart); // [slice][n]
    const bool full = p.atm_center != 0;
    bool range_err = false, overflow = false;
    GroupItem it;
    while (next_item(p, work, it)) {
        const int a = it.i;
        const SG &g = *it.g;
        double4 xa = make_double4(0, 0, 0, 0);
        int4 sa = make_int4(0, 0, 0, 0);
        int oa = -1;
        bool take = a >= 0;
        if (take) {
            xa = p.xs[a];
            sa = p.shift[a];
            oa = p.orig[a];
            if ((p.atm_center && !p.surr_flag[a]) ||
                (p.shard_world > 1 && (p.n - 1 - oa) % p.shard_world != p.shard_rank))
                take = false;
        }
        const bool box_pair = g.box_mode && p.anyshift[it.sr.x];
        long long pos = 0;
        int count = 0;
        if (FILL && take) pos = p.atm_off[a] + gcnt[(size_t)it.sl * p.n + a];
        group_ranges<double, double4>(p, it, p.stencils + g.stab_off, g.stab_n, box_pair, xa,
                                      [&](int base, int m, double, double, double, int px, int Ty, int Tz) {
            __syncwarp();
            if (lane < m) {
                sP[lane] = p.xs[base + lane];
                sO[lane] = p.orig[base + lane];
            }
            __syncwarp();
            if (!take) return;
            const double shx = px * g.h[0] + Ty * g.h[3] + Tz * g.h[6];
            const double shy = px * g.h[1] + Ty * g.h[4] + Tz * g.h[7];
            const double shz = px * g.h[2] + Ty * g.h[5] + Tz * g.h[8];
            for (int jj = 0; jj < m; ++jj) {
                if (!full && sO[jj] > oa) continue;
                if (box_pair && !in_box(g, sa, p.shift[base + jj], px, Ty, Tz)) continue;
                const double4 xj = sP[jj];
                const double dx = xa.x - (xj.x + shx), dy = xa.y - (xj.y + shy), dz = xa.z - (xj.z + shz);
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 > p.ratm2 || d2 < 1e-12) continue;
                if (FILL) {
                    if (abs(px) > 127 || abs(Ty) > 127 || abs(Tz) > 127) range_err = true;
                    if (pos < p.atm_cap)
                        p.atm_ent[pos] = make_int2(base + jj, (px & 0xff) | ((Ty & 0xff) << 8) | ((Tz & 0xff) << 16));
                    ++pos;
                } else {
                    ++count;
                }
            }
        });
        if (!FILL && a >= 0) gcnt[(size_t)it.sl * p.n + a] = take ? count : 0;
        if (FILL && take && pos > p.atm_cap) overflow = true;
    }
    if (FILL) {
        if (__any_sync(0xffffffffu, range_err) && lane == 0) atomicOr(p.status, ST_SHIFT_RANGE);
        if (__any_sync(0xffffffffu, overflow) && lane == 0) atomicOr(p.status, ST_LIST_OVERFLOW);
    }
}

// per apex: the slices' counts -> offsets within the apex's list, and its length
__global__ void k_atm_list_prefix(KP p) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= p.n) return;
    int *gcnt = reinterpret_cast<int *>(p.gpart);
    int run = 0;
    for (int s = 0; s < p.gslices; ++s) {
        const int c = gcnt[(size_t)s * p.n + a];
        gcnt[(size_t)s * p.n + a] = run;
        run += c;
    }
    p.atm_cnt[a] = run;
}

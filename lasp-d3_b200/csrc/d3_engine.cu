// B200 D3 dispersion engine: device kernels and host orchestration (FP64 plain path).
//
// Replaces the reference's pipeline (LASP-D3 src/d3.cu:130-226):
//   coordination_number_kernel (src/d3_kernel.cu:582-683)
//   atm_kernel                 (src/d3_kernel.cu:1199-1509)
//   two_body_kernel            (src/d3_kernel.cu:997-1197)
//   three_body_kernel          (src/d3_kernel.cu:1571-1698, the dE/dCN chain rule)
// with a GPU cell list instead of per-image all-pairs loops, per-atom factorised C6
// weights instead of per-pair 25-exponential C6, an explicit rc_ATM half neighbour
// list with triplets enumerated from it, and deterministic per-atom accumulation
// except for the ATM scatter to neighbour atoms (FP64 atomics).
//
// Device layout (HBM):
//   xs[n]      double4  wrapped position (bohr) + type in .w, binned order
//   shift[n]   int4     lattice shift removed by wrapping (S, unwrapped = xs + S*h)
//   orig[n] / sorted_of[n]  binned <-> caller order
//   bin_start[nbins+1]      CSR of the bin grid (x fastest)
//   w, dw[n][NR]            normalised Gaussian weights of the C6 reference grid and
//                           their CN derivative
//   Y[n][ne][NR]            y_{i,t}[b] = sum_a w_i[a] C6ref[t_i][t][a][b]
//   per-atom energy / dE/dCN / force / virial partials of each pass
//   atm_off[n+1], atm_ent[] rc_ATM half list (j <= a in caller order), CSR
#include "d3_engine.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <type_traits>

#include "d3_mlp.h"
#include "d3_synth_params.h"

namespace d3 {

#define D3_CUDA(call)                                                                                     \
    do {                                                                                                  \
        cudaError_t err__ = (call);                                                                       \
        if (err__ != cudaSuccess) throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(err__) + \
                                                           " at " + __FILE__ + ":" + std::to_string(__LINE__)); \
    } while (0)

constexpr double K1 = 16.0;
constexpr double K3 = 4.0;
// floats per (atom, partner type) row of the block-pair ATM table (NR 5 or 7: 12 or 16,
// whole float4s)
__host__ __device__ constexpr int atmb_row_floats(int nr) { return 2 * nr + 2; }

// ------------------------------------------------------------------------------------
// kernel parameter block (passed by value)
// ------------------------------------------------------------------------------------
// geometry of one structure (a batch holds many; a plain handle holds one)
struct SG {
    double h[9], inv[9], vol; // rows = lattice vectors (bohr), inverse, signed volume
    int nb[3], nbins;         // bin grid of this structure
    int bin_base;             // first global bin index of this structure
    int box_mode;             // 1: the reference's image box applies (ALL_ITERATE)
    int half[3];              // image box half-widths
    int atom_base, natoms;    // atom range in caller order
    int st2_off, st2_n, stc_off, stc_n, sta_off, sta_n; // stencil rows (two-body, CN, ATM)
    int st2b_off, st2b_n;     // two-body stencil of a block of gy x gz bin rows (atom groups)
    int stcb_off, stcb_n;     // CN / chain-rule stencil of the same blocks
    int stab_off, stab_n;     // rc_ATM stencil of the same blocks (ATM half lists)
    int atm_simple;           // every cell height > 2 rc_ATM: no atom twice in an ATM list
};

struct KP {
    int n;                    // atoms of all structures
    int nstruct;
    int nbins_total;
    int ne, nref;
    const SG *sg;
    const int *sid_in;        // structure of each atom, caller order
    int *sid;                 // structure of each atom, binned order
    const int4 *stencils;     // all stencil rows (x = dy, y = dz, z = dxlo, w = dxhi)
    double rc2, rcn2, ratm2, rc_cn;
    // tables
    const double *cnref; // [ne][MAX_NREF]
    const double *c6;    // [ne][ne][nref][nref]
    const double *r0ab;  // [ne][ne]
    const double *rcov;  // [ne]
    const double *r2r4;  // [ne]
    const double *pairA; // [ne][ne][4]: BJ: A^6, A^8 ; zero: R0
    double s6, s8, p1, p2;
    int damping, smooth_cn, atm_force_scaled;
    // atoms, caller order
    const double *pos_in;
    const int *type_in;
    int *bin_in;
    int4 *shift_in;
    double4 *xw_in;
    // binning
    int *bin_cnt, *bin_start, *bin_fill, *order;
    // atoms, binned order
    double4 *xs;
    int4 *shift;
    int *bin_s, *orig, *sorted_of;
    double *cn, *w, *dw, *Y;
    double *e2, *g2, *f2, *v2; // two-body: energy, dE/dCN, force[3], virial[6]
    double *ea, *ga, *fa, *va; // ATM apex share (direct writes)
    double *eb, *gb, *fb;      // ATM entry share (atomics)
    double *fc, *vc;           // chain rule: force[3], virial[6]
    // ATM list
    int *atm_cnt;
    long long *atm_off;
    int2 *atm_ent;
    long long atm_cap;
    int *work;
    // centre mode (surrogate fallback): full lists of the flagged atoms only, the apexes
    // taken from atm_apex[0 .. *atm_napex), every triplet weighted 1/3
    int atm_center;
    const int *atm_apex;
    const int *atm_napex;
    const unsigned char *surr_flag;
    // outputs: [0, S) energies (eV), [S, S+3n) forces (eV/A, caller order),
    // [S+3n, S+3n+9S) stresses (eV/A^3, row-major per structure)
    double *out;
    unsigned int *status;
    // precision form: FP32 copies of positions, weights and C6 rows
    int precision;
    float4 *xs32;
    float *w32, *dw32, *Y32;
    float *YD32;    // [n][ne][2 NR + 2] (block-pair ATM): per partner type the C6 row, r0^2 of
                    // the type pair, the row of the weight derivatives, the atom index bits
    int atm_min_m;  // k_atm32 takes only apexes with longer lists (the rest: k_atm32b)
    int atmb_mcap;  // longest list k_atm32b takes
    int atmb_split; // CTAs of k_atm32b sharing one apex (each a share of its block rows)
    // sharded evaluation: this process computes the two-body and chain-rule terms of the
    // atom groups it owns (group_owner; without groups: central atoms i = shard_rank +
    // k shard_world, binned order) and the ATM apexes of work items shard_rank +
    // k shard_world; CN and weights for every atom
    int shard_rank, shard_world;
    // work counters: [0] ATM in-range visits (2 per triplet), [1] two-body in-range
    // ordered pairs, [2] CN in-range ordered pairs
    unsigned long long *counters;
    // atom groups of the two-body pass (d3_pairs.cuh): super-rows, groups and their
    // count, stencil-row slices per group, per-slice partial sums, work counter
    int *anyshift;           // per structure: some atom was given outside the cell
    const int4 *srows;
    int nsrow;
    int4 *groups;
    int *gcount;             // groups cut this evaluation (the passes' work counters follow)
    int gslices;
    double *gpart;
};

__device__ __forceinline__ int floordiv(int a, int b) {
    int q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
    return q;
}

__device__ __forceinline__ int shard_atom(const KP &p, int w) { return w * p.shard_world + p.shard_rank; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Traverse every candidate (j, T) of binned atom i through a row-compressed stencil.
// All 32 lanes call f(j, Tx, Ty, Tz, shift, active) together (converged), so f may use
// warp votes; shift = T h (bohr) is computed once per contiguous range of candidates.
// row_end() is called (converged) after each stencil row.
struct NoRowEnd {
    __device__ __forceinline__ void operator()() const {}
};

template <class F, class R = NoRowEnd>
__device__ __forceinline__ void traverse(const KP &p, const SG &g, int bin_global, const int4 *rows, int nrows, F &&f,
                                         R &&row_end = R()) {
    const int lane = threadIdx.x & 31;
    const int nb0 = g.nb[0], nb1 = g.nb[1], nb2 = g.nb[2];
    const int bin = bin_global - g.bin_base;
    const int *bstart = p.bin_start + g.bin_base;
    const int bx = bin % nb0, by = (bin / nb0) % nb1, bz = bin / (nb0 * nb1);
    for (int r = 0; r < nrows; ++r) {
        const int4 row = rows[r];
        const int yy = by + row.x, zz = bz + row.y;
        const int Ty = floordiv(yy, nb1), Tz = floordiv(zz, nb2);
        const int byy = yy - Ty * nb1, bzz = zz - Tz * nb2;
        const int xlo = bx + row.z, xhi = bx + row.w;
        const int plo = floordiv(xlo, nb0), phi = floordiv(xhi, nb0);
        const int rowbase = nb0 * (byy + nb1 * bzz);
        for (int px = plo; px <= phi; ++px) {
            const int a = max(xlo, px * nb0) - px * nb0;
            const int b = min(xhi, px * nb0 + nb0 - 1) - px * nb0;
            const int jlo = bstart[rowbase + a], jhi = bstart[rowbase + b + 1];
            const double3 sh = make_double3(px * g.h[0] + Ty * g.h[3] + Tz * g.h[6], px * g.h[1] + Ty * g.h[4] + Tz * g.h[7],
                                            px * g.h[2] + Ty * g.h[5] + Tz * g.h[8]);
            for (int base = jlo; base < jhi; base += 32) {
                const int j = base + lane;
                f(j, px, Ty, Tz, sh, j < jhi);
            }
        }
        row_end();
    }
}

// FP32 variant for the precision-form pair kernels: instead of the image shift it hands f
// the origin o = x_i - shift (float, rounded once per contiguous range of candidates), so
// that dx = o.x - x_j.x needs no per-candidate conversion.
template <class F, class R = NoRowEnd>
__device__ __forceinline__ void traverse32(const KP &p, const SG &g, int bin_global, const int4 *rows, int nrows,
                                           const float4 xi, F &&f, R &&row_end = R()) {
    const int lane = threadIdx.x & 31;
    const int nb0 = g.nb[0], nb1 = g.nb[1], nb2 = g.nb[2];
    const int bin = bin_global - g.bin_base;
    const int *bstart = p.bin_start + g.bin_base;
    const int bx = bin % nb0, by = (bin / nb0) % nb1, bz = bin / (nb0 * nb1);
    for (int r = 0; r < nrows; ++r) {
        const int4 row = rows[r];
        const int yy = by + row.x, zz = bz + row.y;
        const int Ty = floordiv(yy, nb1), Tz = floordiv(zz, nb2);
        const int byy = yy - Ty * nb1, bzz = zz - Tz * nb2;
        const int xlo = bx + row.z, xhi = bx + row.w;
        const int plo = floordiv(xlo, nb0), phi = floordiv(xhi, nb0);
        const int rowbase = nb0 * (byy + nb1 * bzz);
        for (int px = plo; px <= phi; ++px) {
            const int a = max(xlo, px * nb0) - px * nb0;
            const int b = min(xhi, px * nb0 + nb0 - 1) - px * nb0;
            const int jlo = bstart[rowbase + a], jhi = bstart[rowbase + b + 1];
            const float3 o = make_float3(xi.x - (float)(px * g.h[0] + Ty * g.h[3] + Tz * g.h[6]),
                                         xi.y - (float)(px * g.h[1] + Ty * g.h[4] + Tz * g.h[7]),
                                         xi.z - (float)(px * g.h[2] + Ty * g.h[5] + Tz * g.h[8]));
            for (int base = jlo; base < jhi; base += 32) {
                const int j = base + lane;
                f(j, px, Ty, Tz, o, j < jhi);
            }
        }
        row_end();
    }
}

__device__ __forceinline__ bool in_box(const SG &g, int4 si, int4 sj, int Tx, int Ty, int Tz) {
    if (!g.box_mode) return true;
    // reference lattice shift of this image in unwrapped coordinates
    const int rx = Tx + si.x - sj.x, ry = Ty + si.y - sj.y, rz = Tz + si.z - sj.z;
    return abs(rx) <= g.half[0] && abs(ry) <= g.half[1] && abs(rz) <= g.half[2];
}

__device__ __forceinline__ void image_vec(const SG &g, int Tx, int Ty, int Tz, double &sx, double &sy, double &sz) {
    sx = Tx * g.h[0] + Ty * g.h[3] + Tz * g.h[6];
    sy = Tx * g.h[1] + Ty * g.h[4] + Tz * g.h[7];
    sz = Tx * g.h[2] + Ty * g.h[5] + Tz * g.h[8];
}

// ------------------------------------------------------------------------------------
// binning: wrap into the cell, bin, GPU counting sort (stable in caller order)
// ------------------------------------------------------------------------------------
__global__ void k_bin(KP p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const SG &g = p.sg[p.sid_in[i]];
    const double x = p.pos_in[3 * i], y = p.pos_in[3 * i + 1], z = p.pos_in[3 * i + 2];
    int s[3], b[3];
    bool bad = !(isfinite(x) && isfinite(y) && isfinite(z));
    for (int k = 0; k < 3; ++k) {
        double f = x * g.inv[0 * 3 + k] + y * g.inv[1 * 3 + k] + z * g.inv[2 * 3 + k];
        if (bad || fabs(f) > 1.0e6) {
            bad = true;
            f = 0.0;
        }
        double fl = floor(f);
        s[k] = (int)fl;
        int bk = (int)((f - fl) * g.nb[k]);
        b[k] = min(max(bk, 0), g.nb[k] - 1);
    }
    if (bad) atomicOr(p.status, ST_BAD_INPUT);
    if ((s[0] | s[1] | s[2]) != 0) atomicOr(&p.anyshift[p.sid_in[i]], 1);
    const int bin = g.bin_base + b[0] + g.nb[0] * (b[1] + g.nb[1] * b[2]);
    double xw = x - (s[0] * g.h[0] + s[1] * g.h[3] + s[2] * g.h[6]);
    double yw = y - (s[0] * g.h[1] + s[1] * g.h[4] + s[2] * g.h[7]);
    double zw = z - (s[0] * g.h[2] + s[1] * g.h[5] + s[2] * g.h[8]);
    if (bad) xw = yw = zw = 0.0;
    p.bin_in[i] = bin;
    p.shift_in[i] = make_int4(s[0], s[1], s[2], 0);
    p.xw_in[i] = make_double4(xw, yw, zw, (double)p.type_in[i]);
    atomicAdd(&p.bin_cnt[bin], 1);
}

// exclusive scan of cnt[0..m) into out[0..m] (out[m] = total); one block
template <typename T, typename S>
__global__ void k_scan(const S *cnt, T *out, int m) {
    __shared__ T warp_tot[32];
    __shared__ T carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < m; base += blockDim.x) {
        const int i = base + threadIdx.x;
        T v = (i < m) ? (T)cnt[i] : (T)0;
        T x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[wid] = x;
        __syncthreads();
        if (wid == 0) {
            T t = (lane < nw) ? warp_tot[lane] : (T)0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                T y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            if (lane < nw) warp_tot[lane] = t;
        }
        __syncthreads();
        const T before = carry + (wid > 0 ? warp_tot[wid - 1] : (T)0) + x - v;
        if (i < m) out[i] = before;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = before + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[m] = carry;
}

__global__ void k_scatter(KP p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int b = p.bin_in[i];
    const int slot = p.bin_start[b] + atomicAdd(&p.bin_fill[b], 1);
    p.order[slot] = i;
}

// make the in-bin order deterministic: ascending caller index (bins hold few atoms)
__global__ void k_binsort(KP p) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= p.nbins_total) return;
    const int lo = p.bin_start[b], hi = p.bin_start[b + 1];
    for (int i = lo + 1; i < hi; ++i) {
        int v = p.order[i], k = i - 1;
        while (k >= lo && p.order[k] > v) {
            p.order[k + 1] = p.order[k];
            --k;
        }
        p.order[k + 1] = v;
    }
}

__global__ void k_gather(KP p) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= p.n) return;
    const int i = p.order[s];
    const double4 x = p.xw_in[i];
    p.xs[s] = x;
    if (p.precision) p.xs32[s] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)x.w);
    p.shift[s] = p.shift_in[i];
    p.bin_s[s] = p.bin_in[i];
    p.sid[s] = p.sid_in[i];
    p.orig[s] = i;
    p.sorted_of[i] = s;
}

// ------------------------------------------------------------------------------------
// coordination numbers (src/d3_kernel.cu:544-683): warp per atom
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double cn_term(const KP &p, double r, double rsum, double *dcn_over_r) {
    const double e = exp(-K1 * (rsum / r - 1.0));
    const double ope = 1.0 + e;
    if (p.smooth_cn) {
        const double t = tanh(p.rc_cn - r);
        const double sc = t * t * t;
        const double dsc = -3.0 * t * t * (1.0 - t * t);
        *dcn_over_r = (-K1) * e * rsum / (r * r * r * ope * ope) * sc + dsc / (ope * r);
        return sc / ope;
    }
    *dcn_over_r = (-K1) * e * rsum / (r * r * r * ope * ope);
    return 1.0 / ope;
}

__global__ void k_cn(KP p) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= p.n) return;
    const SG &g = p.sg[p.sid[i]];
    const double4 xi = p.xs[i];
    const int4 si = p.shift[i];
    const double ri = p.rcov[(int)xi.w];
    double acc = 0.0;
    unsigned int npair = 0;
    traverse(p, g, p.bin_s[i], p.stencils + g.stc_off, g.stc_n, [&](int j, int Tx, int Ty, int Tz, const double3 &sh, bool act) {
        if (!act) return;
        if (!in_box(g, si, p.shift[j], Tx, Ty, Tz)) return;
        const double4 xj = p.xs[j];
        const double dx = xi.x - (xj.x + sh.x), dy = xi.y - (xj.y + sh.y), dz = xi.z - (xj.z + sh.z);
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 <= p.rcn2 && d2 > 0.0) {
            double dd;
            acc += cn_term(p, sqrt(d2), ri + p.rcov[(int)xj.w], &dd);
            ++npair;
        }
    });
    acc = warp_sum(acc);
    for (int o = 16; o > 0; o >>= 1) npair += __shfl_xor_sync(0xffffffffu, npair, o);
    if ((threadIdx.x & 31) == 0) {
        p.cn[i] = acc;
        atomicAdd(&p.counters[2], (unsigned long long)npair);
    }
}

// ------------------------------------------------------------------------------------
// per-atom normalised Gaussian weights (src/d3_kernel.cu:709-881, factorised)
//   L_ab = w_i[a] w_j[b] with the max-shift split per atom, so
//   C6_ij = w_i^T C w_j / (sum w_i sum w_j) and dC6/dCN_i = dw_i^T C w_j (normalised)
// ------------------------------------------------------------------------------------
template <int NR>
__global__ void k_weights(KP p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int t = (int)p.xs[i].w;
    const double cn = p.cn[i];
    double w[NR], dw[NR];
    double mx = -INFINITY;
#pragma unroll
    for (int a = 0; a < NR; ++a) {
        const double cr = p.cnref[t * MAX_NREF + a];
        if (cr > -1.0) {
            const double d = cn - cr;
            mx = fmax(mx, -K3 * d * d);
        }
    }
    double sw = 0.0, sdw = 0.0;
#pragma unroll
    for (int a = 0; a < NR; ++a) {
        const double cr = p.cnref[t * MAX_NREF + a];
        if (cr > -1.0) {
            const double d = cn - cr;
            w[a] = exp(-K3 * d * d - mx);
            dw[a] = -2.0 * K3 * d * w[a];
        } else {
            w[a] = 0.0;
            dw[a] = 0.0;
        }
        sw += w[a];
        sdw += dw[a];
    }
    const double isw = sw > 0.0 ? 1.0 / sw : 0.0;
    const double ratio = sdw * isw;
#pragma unroll
    for (int a = 0; a < NR; ++a) {
        const double wn = w[a] * isw;
        const double dwn = dw[a] * isw - wn * ratio;
        p.w[(size_t)i * NR + a] = wn;
        p.dw[(size_t)i * NR + a] = dwn;
        if (p.precision) {
            p.w32[(size_t)i * NR + a] = (float)wn;
            p.dw32[(size_t)i * NR + a] = (float)dwn;
        }
        w[a] = wn;
        dw[a] = dwn;
    }
    for (int tt = 0; tt < p.ne; ++tt) {
        const double *C = p.c6 + ((size_t)t * p.ne + tt) * NR * NR;
        double *Yo = p.Y + ((size_t)i * p.ne + tt) * NR;
#pragma unroll
        for (int b = 0; b < NR; ++b) {
            double acc = 0.0;
#pragma unroll
            for (int a = 0; a < NR; ++a) acc += w[a] * C[a * NR + b];
            Yo[b] = acc;
            if (p.precision) p.Y32[((size_t)i * p.ne + tt) * NR + b] = (float)acc;
            if (p.YD32) {
                double dacc = 0.0;
#pragma unroll
                for (int a = 0; a < NR; ++a) dacc += dw[a] * C[a * NR + b];
                float *r = p.YD32 + ((size_t)i * p.ne + tt) * atmb_row_floats(NR);
                r[b] = (float)acc;
                r[NR + 1 + b] = (float)dacc;
            }
        }
        if (p.YD32) {
            float *r = p.YD32 + ((size_t)i * p.ne + tt) * atmb_row_floats(NR);
            const double r0 = p.r0ab[tt * p.ne + t]; // partner type tt first, as the triplet kernel reads it
            r[NR] = (float)(r0 * r0);
            r[2 * NR + 1] = __int_as_float(i);
        }
    }
}

// ------------------------------------------------------------------------------------
// two-body (src/d3_kernel.cu:902-1197): warp per central atom, every ordered pair
// ------------------------------------------------------------------------------------
template <int NR>
__global__ void k_twobody(KP p) {
    const int i = shard_atom(p, (blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (i >= p.n) return;
    const SG &g = p.sg[p.sid[i]];
    const double4 xi = p.xs[i];
    const int4 si = p.shift[i];
    const int ti = (int)xi.w;
    double wi[NR], dwi[NR];
#pragma unroll
    for (int a = 0; a < NR; ++a) {
        wi[a] = p.w[(size_t)i * NR + a];
        dwi[a] = p.dw[(size_t)i * NR + a];
    }
    const double rri = p.r2r4[ti];
    double e = 0, gacc = 0, fx = 0, fy = 0, fz = 0, vxx = 0, vyy = 0, vzz = 0, vxy = 0, vxz = 0, vyz = 0;
    unsigned int npair = 0;
    traverse(p, g, p.bin_s[i], p.stencils + g.st2_off, g.st2_n, [&](int j, int Tx, int Ty, int Tz, const double3 &sh, bool act) {
        if (!act) return;
        if (!in_box(g, si, p.shift[j], Tx, Ty, Tz)) return;
        const double4 xj = p.xs[j];
        const double dx = xi.x - (xj.x + sh.x), dy = xi.y - (xj.y + sh.y), dz = xi.z - (xj.z + sh.z);
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 < p.rc2 && r2 > 0.0)) return;
        ++npair;
        const int tj = (int)xj.w;
        const double *yj = p.Y + ((size_t)j * p.ne + ti) * NR;
        double c6 = 0.0, dc6 = 0.0;
#pragma unroll
        for (int b = 0; b < NR; ++b) {
            const double y = yj[b];
            c6 += y * wi[b];
            dc6 += y * dwi[b];
        }
        const double rr = 3.0 * rri * p.r2r4[tj];
        const double c8 = c6 * rr, dc8 = dc6 * rr;
        const double *pa = p.pairA + ((size_t)ti * p.ne + tj) * 4;
        double E6, E8, G, fs;
        if (p.damping == 1) {
            const double r4 = r2 * r2, r6 = r4 * r2, r8 = r4 * r4;
            const double i6 = 1.0 / (r6 + pa[0]), i8 = 1.0 / (r8 + pa[1]);
            E6 = p.s6 * c6 * i6;
            E8 = p.s8 * c8 * i8;
            G = p.s6 * dc6 * i6 + p.s8 * dc8 * i8;
            fs = -6.0 * p.s6 * c6 * r4 * i6 * i6 - 8.0 * p.s8 * c8 * r6 * i8 * i8;
        } else {
            const double r = sqrt(r2), ir = 1.0 / r, ir2 = ir * ir;
            const double ir6 = ir2 * ir2 * ir2, ir8 = ir6 * ir2;
            const double R0 = pa[0];
            const double x6 = p.p1 * R0 * ir, x8 = p.p2 * R0 * ir;
            const double x6_2 = x6 * x6, x6_4 = x6_2 * x6_2, x6_8 = x6_4 * x6_4, x6_14 = x6_8 * x6_4 * x6_2;
            const double x8_2 = x8 * x8, x8_4 = x8_2 * x8_2, x8_8 = x8_4 * x8_4, x8_16 = x8_8 * x8_8;
            const double f6 = 1.0 / (1.0 + 6.0 * x6_14), f8 = 1.0 / (1.0 + 6.0 * x8_16);
            const double df6 = 84.0 * f6 * f6 * x6_14 * ir, df8 = 96.0 * f8 * f8 * x8_16 * ir;
            E6 = p.s6 * c6 * f6 * ir6;
            E8 = p.s8 * c8 * f8 * ir8;
            G = p.s6 * f6 * dc6 * ir6 + p.s8 * f8 * dc8 * ir8;
            fs = p.s6 * c6 * (-6.0 * f6 * ir8 + df6 * ir6 * ir) + p.s8 * c8 * (-8.0 * f8 * ir8 * ir2 + df8 * ir8 * ir);
        }
        e += 0.5 * (E6 + E8);
        gacc += G;
        fx += fs * dx;
        fy += fs * dy;
        fz += fs * dz;
        vxx += fs * dx * dx;
        vyy += fs * dy * dy;
        vzz += fs * dz * dz;
        vxy += fs * dx * dy;
        vxz += fs * dx * dz;
        vyz += fs * dy * dz;
    });
    e = warp_sum(e);
    gacc = warp_sum(gacc);
    fx = warp_sum(fx);
    fy = warp_sum(fy);
    fz = warp_sum(fz);
    vxx = warp_sum(vxx);
    vyy = warp_sum(vyy);
    vzz = warp_sum(vzz);
    vxy = warp_sum(vxy);
    vxz = warp_sum(vxz);
    vyz = warp_sum(vyz);
    for (int o = 16; o > 0; o >>= 1) npair += __shfl_xor_sync(0xffffffffu, npair, o);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&p.counters[1], (unsigned long long)npair);
        p.e2[i] = e;
        p.g2[i] = gacc;
        p.f2[3 * i] = fx;
        p.f2[3 * i + 1] = fy;
        p.f2[3 * i + 2] = fz;
        const double sc = -1.0 / (2.0 * g.vol);
        double *v = p.v2 + 6 * (size_t)i;
        v[0] = vxx * sc;
        v[1] = vyy * sc;
        v[2] = vzz * sc;
        v[3] = vxy * sc;
        v[4] = vxz * sc;
        v[5] = vyz * sc;
    }
}

// ------------------------------------------------------------------------------------
// ATM half list: for apex a, entries (j, T) with caller index j <= a, every side in
// [1e-12, rc_ATM^2] (src/d3_kernel.cu:1235-1269). Count pass then fill pass.
// ------------------------------------------------------------------------------------
template <bool FILL>
__global__ void k_atm_list(KP p) {
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (a >= p.n) return;
    const SG &g = p.sg[p.sid[a]];
    const int lane = threadIdx.x & 31;
    const double4 xa = p.xs[a];
    const int4 sa = p.shift[a];
    const int oa = p.orig[a];
    long long pos = 0;
    if (FILL) pos = p.atm_off[a];
    int count = 0;
    bool range_err = false;
    if ((p.atm_center && !p.surr_flag[a]) ||
        (p.shard_world > 1 && (p.n - 1 - oa) % p.shard_world != p.shard_rank)) {
        if (!FILL && lane == 0) p.atm_cnt[a] = 0;
        return;
    }
    const bool full = p.atm_center != 0;
    // the image box needs each partner's wrap shift only when some atom was given outside
    // the cell; otherwise the test is on the image alone
    const bool box_pair = g.box_mode && p.anyshift[p.sid[a]];
    traverse(p, g, p.bin_s[a], p.stencils + g.sta_off, g.sta_n, [&](int j, int Tx, int Ty, int Tz, const double3 &sh, bool act) {
        bool keep = false;
        // (act first: j is a valid index only for active lanes)
        if (act && (full || p.orig[j] <= oa) &&
            (box_pair ? in_box(g, sa, p.shift[j], Tx, Ty, Tz)
                      : !(g.box_mode && (abs(Tx) > g.half[0] || abs(Ty) > g.half[1] || abs(Tz) > g.half[2])))) {
            const double4 xj = p.xs[j];
            const double dx = xa.x - (xj.x + sh.x), dy = xa.y - (xj.y + sh.y), dz = xa.z - (xj.z + sh.z);
            const double d2 = dx * dx + dy * dy + dz * dz;
            keep = !(d2 > p.ratm2 || d2 < 1e-12);
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (FILL) {
            if (keep) {
                const long long slot = pos + __popc(m & ((1u << lane) - 1u));
                if (abs(Tx) > 127 || abs(Ty) > 127 || abs(Tz) > 127) range_err = true;
                if (slot < p.atm_cap) {
                    const int packed = (Tx & 0xff) | ((Ty & 0xff) << 8) | ((Tz & 0xff) << 16);
                    p.atm_ent[slot] = make_int2(j, packed);
                }
            }
            pos += __popc(m);
        } else {
            count += __popc(m);
        }
    });
    if (!FILL && lane == 0) p.atm_cnt[a] = count;
    if (FILL) {
        if (range_err) atomicOr(p.status, ST_SHIFT_RANGE);
        if (lane == 0 && pos > p.atm_cap) atomicOr(p.status, ST_LIST_OVERFLOW);
    }
}

__device__ __forceinline__ int sext8(int v) { return (v << 24) >> 24; }

// Special-function-unit approximations in their subnormal-flushing PTX forms (.ftz): no
// subnormal handling is wrapped around the operation. Relative error about 2^-22 (the
// PTX ISA's bounds for the .approx forms). The FP32 triplet and pair terms stay far from
// the subnormal range (their smallest intermediates are about 1e-25).
__device__ __forceinline__ float sfu_rsqrt(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sfu_rcp(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sfu_log2(float x) {
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sfu_exp2(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// ------------------------------------------------------------------------------------
// precision form: CN, two-body and chain rule with FP32 pair arithmetic. Sums are kept
// in FP32 within one stencil row and carried across rows in FP64 (blocked summation);
// dE/dCN is accumulated in FP64.
// ------------------------------------------------------------------------------------
// FP32 CN term: value and (d CN / d r) / r, with the optional tanh^3 smooth cutoff (the
// reference's SMOOTH_CUTOFF_CN) as in the FP64 term
__device__ __forceinline__ float cn_term32(const KP &p, float r2, float rsum, float *dcn_over_r) {
    const float ir = sfu_rsqrt(r2);
    // exp(-16 (rsum / r - 1)) as a power of two
    const float e = sfu_exp2(-16.0f * 1.44269504f * fmaf(rsum, ir, -1.0f));
    const float inv = sfu_rcp(1.0f + e);
    float d = -16.0f * e * rsum * ir * ir * ir * inv * inv;
    float v = inv;
    if (p.smooth_cn) {
        const float t = tanhf((float)p.rc_cn - r2 * ir);
        const float sc = t * t * t;
        d = d * sc - 3.0f * t * t * (1.0f - t * t) * inv * ir;
        v = inv * sc;
    }
    *dcn_over_r = d;
    return v;
}

__global__ void k_cn32(KP p) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= p.n) return;
    const SG &g = p.sg[p.sid[i]];
    const float4 xi = p.xs32[i];
    const int4 si = p.shift[i];
    const float ri = (float)p.rcov[(int)xi.w];
    const float rcn2 = (float)p.rcn2;
    double acc = 0.0;
    float part = 0.0f;
    unsigned int npair = 0;
    traverse32(
        p, g, p.bin_s[i], p.stencils + g.stc_off, g.stc_n, xi,
        [&](int j, int Tx, int Ty, int Tz, const float3 &o, bool act) {
            if (!act) return;
            if (!in_box(g, si, p.shift[j], Tx, Ty, Tz)) return;
            const float4 xj = p.xs32[j];
            const float dx = o.x - xj.x, dy = o.y - xj.y,
                        dz = o.z - xj.z;
            const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (d2 <= rcn2 && d2 > 0.0f) {
                float dd;
                part += cn_term32(p, d2, ri + (float)p.rcov[(int)xj.w], &dd);
                ++npair;
            }
        },
        [&]() {
            acc += part;
            part = 0.0f;
        });
    acc = warp_sum(acc);
    for (int o = 16; o > 0; o >>= 1) npair += __shfl_xor_sync(0xffffffffu, npair, o);
    if ((threadIdx.x & 31) == 0) {
        p.cn[i] = acc;
        atomicAdd(&p.counters[2], (unsigned long long)npair);
    }
}

template <int NR>
__global__ void k_twobody32(KP p) {
    // per type pair, FP32: BJ A^6, A^8 (zero damping: R0) and 3 sqrt(Q_i Q_j)^2 ratio
    extern __shared__ float4 pair_tab[]; // [ne][ne]
    for (int k = threadIdx.x; k < p.ne * p.ne; k += blockDim.x) {
        const double *pa = p.pairA + (size_t)k * 4;
        pair_tab[k] = make_float4((float)pa[0], (float)pa[1],
                                  3.0f * (float)p.r2r4[k / p.ne] * (float)p.r2r4[k % p.ne], 0.0f);
    }
    __syncthreads();
    const int i = shard_atom(p, (blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (i >= p.n) return;
    const SG &g = p.sg[p.sid[i]];
    const float4 xi = p.xs32[i];
    const int4 si = p.shift[i];
    const int ti = (int)xi.w;
    float wi[NR], dwi[NR];
#pragma unroll
    for (int a = 0; a < NR; ++a) {
        wi[a] = p.w32[(size_t)i * NR + a];
        dwi[a] = p.dw32[(size_t)i * NR + a];
    }
    const float rc2 = (float)p.rc2, s6 = (float)p.s6, s8 = (float)p.s8, p1 = (float)p.p1, p2 = (float)p.p2;
    double E = 0, G = 0, FX = 0, FY = 0, FZ = 0, VXX = 0, VYY = 0, VZZ = 0, VXY = 0, VXZ = 0, VYZ = 0;
    float e = 0, fx = 0, fy = 0, fz = 0, vxx = 0, vyy = 0, vzz = 0, vxy = 0, vxz = 0, vyz = 0;
    unsigned int npair = 0;
    traverse32(
        p, g, p.bin_s[i], p.stencils + g.st2_off, g.st2_n, xi,
        [&](int j, int Tx, int Ty, int Tz, const float3 &o, bool act) {
            if (!act) return;
            if (!in_box(g, si, p.shift[j], Tx, Ty, Tz)) return;
            const float4 xj = p.xs32[j];
            const float dx = o.x - xj.x, dy = o.y - xj.y,
                        dz = o.z - xj.z;
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (!(r2 < rc2 && r2 > 0.0f)) return;
            ++npair;
            const int tj = (int)xj.w;
            const float *yj = p.Y32 + ((size_t)j * p.ne + ti) * NR;
            float c6 = 0.f, dc6 = 0.f;
#pragma unroll
            for (int b = 0; b < NR; ++b) {
                const float y = yj[b];
                c6 = fmaf(y, wi[b], c6);
                dc6 = fmaf(y, dwi[b], dc6);
            }
            const float4 tp = pair_tab[ti * p.ne + tj];
            const float rr = tp.z;
            const float c8 = c6 * rr, dc8 = dc6 * rr;
            float E6, E8, Gt, fs;
            if (p.damping == 1) {
                const float r4 = r2 * r2, r6 = r4 * r2, r8 = r4 * r4;
                const float i6 = sfu_rcp(r6 + tp.x), i8 = sfu_rcp(r8 + tp.y);
                E6 = s6 * c6 * i6;
                E8 = s8 * c8 * i8;
                Gt = s6 * dc6 * i6 + s8 * dc8 * i8;
                fs = -6.0f * E6 * r4 * i6 - 8.0f * E8 * r6 * i8;
            } else {
                const float ir = sfu_rsqrt(r2), ir2 = ir * ir;
                const float ir6 = ir2 * ir2 * ir2, ir8 = ir6 * ir2;
                const float R0 = tp.x;
                const float x6 = p1 * R0 * ir, x8 = p2 * R0 * ir;
                const float x6_2 = x6 * x6, x6_4 = x6_2 * x6_2, x6_8 = x6_4 * x6_4, x6_14 = x6_8 * x6_4 * x6_2;
                const float x8_2 = x8 * x8, x8_4 = x8_2 * x8_2, x8_8 = x8_4 * x8_4, x8_16 = x8_8 * x8_8;
                const float f6 = sfu_rcp(fmaf(6.0f, x6_14, 1.0f)), f8 = sfu_rcp(fmaf(6.0f, x8_16, 1.0f));
                const float df6 = 84.0f * f6 * f6 * x6_14 * ir, df8 = 96.0f * f8 * f8 * x8_16 * ir;
                E6 = s6 * c6 * f6 * ir6;
                E8 = s8 * c8 * f8 * ir8;
                Gt = s6 * f6 * dc6 * ir6 + s8 * f8 * dc8 * ir8;
                fs = s6 * c6 * (-6.0f * f6 * ir8 + df6 * ir6 * ir) + s8 * c8 * (-8.0f * f8 * ir8 * ir2 + df8 * ir8 * ir);
            }
            e += 0.5f * (E6 + E8);
            G += (double)Gt;
            fx = fmaf(fs, dx, fx);
            fy = fmaf(fs, dy, fy);
            fz = fmaf(fs, dz, fz);
            const float fdx = fs * dx, fdy = fs * dy;
            vxx = fmaf(fdx, dx, vxx);
            vyy = fmaf(fdy, dy, vyy);
            vzz = fmaf(fs * dz, dz, vzz);
            vxy = fmaf(fdx, dy, vxy);
            vxz = fmaf(fdx, dz, vxz);
            vyz = fmaf(fdy, dz, vyz);
        },
        [&]() {
            E += e;
            FX += fx;
            FY += fy;
            FZ += fz;
            VXX += vxx;
            VYY += vyy;
            VZZ += vzz;
            VXY += vxy;
            VXZ += vxz;
            VYZ += vyz;
            e = fx = fy = fz = vxx = vyy = vzz = vxy = vxz = vyz = 0.0f;
        });
    E = warp_sum(E);
    G = warp_sum(G);
    FX = warp_sum(FX);
    FY = warp_sum(FY);
    FZ = warp_sum(FZ);
    VXX = warp_sum(VXX);
    VYY = warp_sum(VYY);
    VZZ = warp_sum(VZZ);
    VXY = warp_sum(VXY);
    VXZ = warp_sum(VXZ);
    VYZ = warp_sum(VYZ);
    for (int o = 16; o > 0; o >>= 1) npair += __shfl_xor_sync(0xffffffffu, npair, o);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&p.counters[1], (unsigned long long)npair);
        p.e2[i] = E;
        p.g2[i] = G;
        p.f2[3 * i] = FX;
        p.f2[3 * i + 1] = FY;
        p.f2[3 * i + 2] = FZ;
        const double sc = -1.0 / (2.0 * g.vol);
        double *v = p.v2 + 6 * (size_t)i;
        v[0] = VXX * sc;
        v[1] = VYY * sc;
        v[2] = VZZ * sc;
        v[3] = VXY * sc;
        v[4] = VXZ * sc;
        v[5] = VYZ * sc;
    }
}

__global__ void k_chain32(KP p, const double *Gd) {
    const int i = shard_atom(p, (blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (i >= p.n) return;
    const SG &g = p.sg[p.sid[i]];
    const float4 xi = p.xs32[i];
    const int4 si = p.shift[i];
    const float ri = (float)p.rcov[(int)xi.w];
    const double gi = Gd[i];
    const float rcn2 = (float)p.rcn2;
    double FX = 0, FY = 0, FZ = 0, VXX = 0, VYY = 0, VZZ = 0, VXY = 0, VXZ = 0, VYZ = 0;
    float fx = 0, fy = 0, fz = 0, vxx = 0, vyy = 0, vzz = 0, vxy = 0, vxz = 0, vyz = 0;
    traverse32(
        p, g, p.bin_s[i], p.stencils + g.stc_off, g.stc_n, xi,
        [&](int j, int Tx, int Ty, int Tz, const float3 &o, bool act) {
            if (!act) return;
            if (!in_box(g, si, p.shift[j], Tx, Ty, Tz)) return;
            const float4 xj = p.xs32[j];
            const float dx = o.x - xj.x, dy = o.y - xj.y,
                        dz = o.z - xj.z;
            const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (!(d2 <= rcn2 && d2 > 0.0f)) return;
            float dcn;
            cn_term32(p, d2, ri + (float)p.rcov[(int)xj.w], &dcn);
            const float dE = (float)(gi + Gd[j]) * dcn;
            const float fdx = dE * dx, fdy = dE * dy;
            fx += fdx;
            fy += fdy;
            fz = fmaf(dE, dz, fz);
            vxx = fmaf(fdx, dx, vxx);
            vyy = fmaf(fdy, dy, vyy);
            vzz = fmaf(dE * dz, dz, vzz);
            vxy = fmaf(fdx, dy, vxy);
            vxz = fmaf(fdx, dz, vxz);
            vyz = fmaf(fdy, dz, vyz);
        },
        [&]() {
            FX += fx;
            FY += fy;
            FZ += fz;
            VXX += vxx;
            VYY += vyy;
            VZZ += vzz;
            VXY += vxy;
            VXZ += vxz;
            VYZ += vyz;
            fx = fy = fz = vxx = vyy = vzz = vxy = vxz = vyz = 0.0f;
        });
    FX = warp_sum(FX);
    FY = warp_sum(FY);
    FZ = warp_sum(FZ);
    VXX = warp_sum(VXX);
    VYY = warp_sum(VYY);
    VZZ = warp_sum(VZZ);
    VXY = warp_sum(VXY);
    VXZ = warp_sum(VXZ);
    VYZ = warp_sum(VYZ);
    if ((threadIdx.x & 31) == 0) {
        p.fc[3 * i] = FX;
        p.fc[3 * i + 1] = FY;
        p.fc[3 * i + 2] = FZ;
        const double sc = -1.0 / (2.0 * g.vol);
        double *v = p.vc + 6 * (size_t)i;
        v[0] = VXX * sc;
        v[1] = VYY * sc;
        v[2] = VZZ * sc;
        v[3] = VXY * sc;
        v[4] = VXZ * sc;
        v[5] = VYZ * sc;
    }
}

#include "d3_pairs.cuh"
#include "d3_atm.cuh"
#include "d3_atm32.cuh"
#include "d3_atm32b.cuh"
#include "d3_surrogate.cuh"

// ------------------------------------------------------------------------------------
// learned ATM surrogate: ensemble mean / spread, fallback flags, dE/dG in engine units
// ------------------------------------------------------------------------------------
// Radial basis: 32 Gaussians, centres 0.8 .. 21 A, width 0.7 A (bohr here)
constexpr double SURR_MU0_A = 0.8, SURR_MU1_A = 21.0, SURR_SIGMA_A = 0.7;

struct SurrComb {
    const float *E;        // [members][n] network outputs
    float *dX;             // [n][nfeat]: sum_m dE_m/dG in, dE/dG (engine energy units) out
    const int *center;     // [n]
    const float *e_shift;  // [nch] eV
    float e_scale;         // eV per network unit
    int members, nfeat;
    double thr;            // ensemble standard deviation threshold, eV
    unsigned char *flag;   // [n] 1: exact fallback
    int *apex, *napex;     // flagged atoms (centre-mode ATM apexes)
};

// One warp per atom: ensemble mean and population standard deviation; unflagged atoms
// keep the surrogate energy as their ATM apex share and scale their input gradient to
// the engine's convention (hartree, stored sign); flagged atoms get zero of both and are
// queued for the exact centre-mode pass.
__global__ void k_surr_combine(KP p, SurrComb c) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= p.n) return;
    const int cen = c.center[i];
    double mean = 0.0, var = 0.0;
    for (int m = 0; m < c.members; ++m) mean += (double)c.E[(size_t)m * p.n + i];
    mean /= c.members;
    for (int m = 0; m < c.members; ++m) {
        const double d = (double)c.E[(size_t)m * p.n + i] - mean;
        var += d * d;
    }
    var /= c.members;
    const double sd = sqrt(var) * (double)c.e_scale;
    const bool fl = cen < 0 || !(sd <= c.thr);
    if (lane == 0) {
        c.flag[i] = fl ? 1 : 0;
        const double e_ev = mean * (double)c.e_scale + (cen >= 0 ? (double)c.e_shift[cen] : 0.0);
        p.ea[i] = fl ? 0.0 : -e_ev / HARTREE_EV;
        if (fl) {
            c.apex[atomicAdd(c.napex, 1)] = i;
            if (p.counters) atomicAdd(p.counters + 3, 1ull);
        }
    }
    const float f = fl ? 0.f : (float)(-(double)c.e_scale / ((double)c.members * HARTREE_EV));
    float *row = c.dX + (size_t)i * c.nfeat;
    for (int k = lane; k < c.nfeat; k += 32) row[k] *= f;
}

// descriptors, centre channels and per-atom ATM energies (eV) to caller order
__global__ void k_surr_export(KP p, const float *G, const int *center, int nfeat, float *Go, int *co, double *eo) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= p.n) return;
    const int o = p.orig[i];
    if (Go)
        for (int k = lane; k < nfeat; k += 32) Go[(size_t)o * nfeat + k] = G[(size_t)i * nfeat + k];
    if (lane == 0) {
        if (co) co[o] = center[i];
        if (eo) eo[o] = -(p.ea[i] + p.eb[i]) * HARTREE_EV;
    }
}

// ------------------------------------------------------------------------------------
// chain rule (src/d3_kernel.cu:1511-1698): F_i += (dE/dCN_i + dE/dCN_j) dCN_ij/dr r_hat
// ------------------------------------------------------------------------------------
__global__ void k_chain(KP p, const double *G) {
    const int i = shard_atom(p, (blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (i >= p.n) return;
    const SG &g = p.sg[p.sid[i]];
    const double4 xi = p.xs[i];
    const int4 si = p.shift[i];
    const double ri = p.rcov[(int)xi.w];
    const double gi = G[i];
    double fx = 0, fy = 0, fz = 0, vxx = 0, vyy = 0, vzz = 0, vxy = 0, vxz = 0, vyz = 0;
    traverse(p, g, p.bin_s[i], p.stencils + g.stc_off, g.stc_n, [&](int j, int Tx, int Ty, int Tz, const double3 &sh, bool act) {
        if (!act) return;
        if (!in_box(g, si, p.shift[j], Tx, Ty, Tz)) return;
        const double4 xj = p.xs[j];
        const double dx = xi.x - (xj.x + sh.x), dy = xi.y - (xj.y + sh.y), dz = xi.z - (xj.z + sh.z);
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 <= p.rcn2 && d2 > 0.0)) return;
        double dcn;
        cn_term(p, sqrt(d2), ri + p.rcov[(int)xj.w], &dcn);
        const double dE = (gi + G[j]) * dcn;
        fx += dE * dx;
        fy += dE * dy;
        fz += dE * dz;
        vxx += dE * dx * dx;
        vyy += dE * dy * dy;
        vzz += dE * dz * dz;
        vxy += dE * dx * dy;
        vxz += dE * dx * dz;
        vyz += dE * dy * dz;
    });
    fx = warp_sum(fx);
    fy = warp_sum(fy);
    fz = warp_sum(fz);
    vxx = warp_sum(vxx);
    vyy = warp_sum(vyy);
    vzz = warp_sum(vzz);
    vxy = warp_sum(vxy);
    vxz = warp_sum(vxz);
    vyz = warp_sum(vyz);
    if ((threadIdx.x & 31) == 0) {
        p.fc[3 * i] = fx;
        p.fc[3 * i + 1] = fy;
        p.fc[3 * i + 2] = fz;
        const double sc = -1.0 / (2.0 * g.vol);
        double *v = p.vc + 6 * (size_t)i;
        v[0] = vxx * sc;
        v[1] = vyy * sc;
        v[2] = vzz * sc;
        v[3] = vxy * sc;
        v[4] = vxz * sc;
        v[5] = vyz * sc;
    }
}

__global__ void k_sum_g(KP p, double *G) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    G[i] = p.g2[i] + p.ga[i] + p.gb[i];
}

// forces in caller order, unit conversion (src/d3.cu:203-219)
__global__ void k_forces_out(KP p) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= p.n) return;
    const int i = p.orig[s];
    const double cf = HARTREE_EV * ANG2BOHR;
    double *F = p.out + p.nstruct;
    for (int k = 0; k < 3; ++k)
        F[3 * i + k] = (p.f2[3 * s + k] + p.fa[3 * s + k] + p.fb[3 * s + k] + p.fc[3 * s + k]) * cf;
}

// deterministic total energy and virial of each structure: one block per structure over
// its atoms (contiguous in binned order), fixed order
__global__ void k_reduce(KP p) {
    __shared__ double red[32][7];
    const SG &g = p.sg[blockIdx.x];
    const int lo = p.bin_start[g.bin_base], hi = p.bin_start[g.bin_base + g.nbins];
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int s = lo + threadIdx.x; s < hi; s += blockDim.x) {
        acc[0] += p.e2[s] + p.ea[s] + p.eb[s];
        for (int k = 0; k < 6; ++k) acc[1 + k] += p.v2[6 * (size_t)s + k] + p.va[6 * (size_t)s + k] + p.vc[6 * (size_t)s + k];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < 7; ++k) {
        const double v = warp_sum(acc[k]);
        if (lane == 0) red[wid][k] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            for (int k = 0; k < 7; ++k) t[k] += red[w][k];
        p.out[blockIdx.x] = -t[0] * HARTREE_EV;
        const double cs = HARTREE_EV * ANG2BOHR * ANG2BOHR * ANG2BOHR;
        double *st = p.out + p.nstruct + 3 * (size_t)p.n + 9 * (size_t)blockIdx.x;
        // symmetric virial: xx yy zz xy xz yz
        st[0] = t[1] * cs;
        st[4] = t[2] * cs;
        st[8] = t[3] * cs;
        st[1] = st[3] = t[4] * cs;
        st[2] = st[6] = t[5] * cs;
        st[5] = st[7] = t[6] * cs;
    }
}

// ------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------
template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    void ensure(size_t m) {
        if (m <= n && p) return;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        size_t want = std::max<size_t>(m, 1);
        D3_CUDA(cudaMalloc(&p, want * sizeof(T)));
        n = want;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// learned ATM surrogate: model on the device and its per-evaluation work arrays
struct SurrState {
    bool loaded = false;
    d3mlp::Layout L;
    int members = 0;
    float e_scale = 1.0f;
    double thr_ev = 2e-4;
    DBuf<int> chan, center, apex, napex, xchan, xcenter;
    DBuf<float> master, mean, inv_std, e_shift, G, E, dX, xG;
    DBuf<uint16_t> packed;
    DBuf<unsigned char> flag;
    void release() {
        DBuf<int> *is[] = {&chan, &center, &apex, &napex, &xchan, &xcenter};
        for (auto *d : is) d->release();
        DBuf<float> *fs[] = {&master, &mean, &inv_std, &e_shift, &G, &E, &dX, &xG};
        for (auto *d : fs) d->release();
        packed.release();
        flag.release();
    }
};

struct Engine {
    // configuration
    int nref = 5;
    bool extended = false;
    std::vector<int> elements; // sorted unique atomic numbers (handle slots)
    int ne = 0;
    uint64_t max_atoms = 0;
    uint64_t max_structs = 1;
    double rc = 0, rc_cn = 0, rc_atm = 0;
    float rc_f = 0, rc_cn_f = 0;
    bool use_atm = false;
    int damping = 1, functional = 0;
    FuncParams fp{};
    Options opt{};
    // state
    uint64_t n = 0;
    bool atoms_set = false, cell_set = false;
    unsigned int cell_status = 0; // status of the last set_cell that failed (bad input / cell)
    int nstruct = 0;
    int nbins_total = 0;
    std::vector<SG> sg;          // per-structure geometry
    std::vector<CellGeom> geoms; // per-structure cell (host)
    std::vector<int4> stencil_rows;
    std::vector<uint64_t> counts; // atoms per structure, cells (bohr, float copy) of the geometry
    std::vector<double> cells;
    std::vector<float> cells_f;
    double first_cell[9] = {0};  // single-structure API: cell kept until atoms are set
    float first_cell_f[9] = {0};
    int dev_sms = 148;
    cudaStream_t stream = nullptr;
    // tables
    DBuf<double> t_cnref, t_c6, t_r0, t_rcov, t_r2r4, t_pairA;
    // atoms
    DBuf<double> pos_in;
    DBuf<int> type_in, bin_in;
    DBuf<int4> shift_in, shift;
    DBuf<double4> xw_in, xs;
    DBuf<int> bin_cnt, bin_start, bin_fill, order, bin_s, orig, sorted_of;
    DBuf<double> cn, w, dw, Y, e2, g2, f2, v2, ea, ga, fa, va, eb, gb, fb, fc, vc, G;
    DBuf<int> atm_cnt, work, sid_in, sid;
    DBuf<SG> sg_dev;
    DBuf<float4> xs32;
    DBuf<float> w32, dw32, Y32, YD32;
    DBuf<float4> atmb_scratch;
    DBuf<long long> atm_off;
    DBuf<int2> atm_ent;
    long long atm_cap = 0;
    DBuf<int4> st_dev;
    // two-body atom groups: super-row table (host-built per geometry), groups, counters
    // ([0] group count, [1] work items taken), per-slice partial sums, per-structure flags
    std::vector<int4> srow_host;
    DBuf<int4> srows, groups;
    DBuf<int> gctl, anyshift;
    DBuf<double> gpart;
    size_t group_bound = 0;
    DBuf<double> out;
    DBuf<unsigned int> status;
    DBuf<unsigned long long> counters;
    std::vector<double> host_out;
    // pass boundaries of the last evaluation: bin | cn+weights | two-body | atm list |
    // atm | chain | finalize
    static constexpr int NEV = 8;
    cudaEvent_t ev[NEV] = {};
    bool have_events = false;
    struct OccCache {
        const void *fn = nullptr;
        size_t sm = 0;
        int blocks = 1;
    } atm_occ_cache[12]; // 0-3 mirror / FP64 ATM, 5 grouped two-body, 8-11 block-pair ATM
    SurrState surr;
    int shard_rank = 0, shard_world = 0; // set by engine_shard_begin

    ~Engine() {
        DBuf<double> *ds[] = {&t_cnref, &t_c6, &t_r0, &t_rcov, &t_r2r4, &t_pairA, &pos_in, &cn, &w, &dw, &Y, &e2,
                              &g2, &f2, &v2, &ea, &ga, &fa, &va, &eb, &gb, &fb, &fc, &vc, &G, &out};
        for (auto *d : ds) d->release();
        DBuf<int> *is[] = {&type_in, &bin_in, &bin_cnt, &bin_start, &bin_fill, &order, &bin_s, &orig, &sorted_of,
                           &atm_cnt, &work, &sid_in, &sid};
        for (auto *d : is) d->release();
        shift_in.release();
        shift.release();
        xs32.release();
        w32.release();
        dw32.release();
        Y32.release();
        YD32.release();
        atmb_scratch.release();
        xw_in.release();
        xs.release();
        atm_off.release();
        atm_ent.release();
        st_dev.release();
        srows.release();
        groups.release();
        gctl.release();
        anyshift.release();
        gpart.release();
        sg_dev.release();
        status.release();
        counters.release();
        surr.release();
        for (auto &x : ev)
            if (x) cudaEventDestroy(x);
        if (stream) cudaStreamDestroy(stream);
    }
};

static void build_structures(Engine *e, int nstruct, const uint64_t *counts, const double *cells,
                             const float *cells_f);

static const double FUNC_TABLE[7][7] = {
    // s6, s8_zero, s8_bj, sr6, sr8, a1, a2 (src/d3_types.h:46-54)
    {1.0, 0.722, 0.7875, 1.217, 1.0, 0.4289, 4.4407}, {1.0, 0.928, 1.2177, 1.287, 1.0, 0.4145, 4.8593},
    {1.0, 1.703, 1.9889, 1.261, 1.0, 0.3981, 4.4211}, {1.0, 1.682, 2.6996, 1.094, 1.0, 0.4298, 4.2359},
    {1.0, 1.683, 3.2822, 1.139, 1.0, 0.3946, 4.8516}, {1.0, 1.010, 2.3550, 0.923, 1.0, 0.5238, 3.5016},
    {1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0}};

static FuncParams func_params(int functional, int damping) {
    int idx = (functional >= 0 && functional <= 5) ? functional : 6;
    // the reference stores these as float (real_t); keep the float-rounded values
    auto f = [](double v) { return (double)(float)v; };
    const double *t = FUNC_TABLE[idx];
    FuncParams p;
    p.s6 = f(t[0]);
    if (damping == 1) {
        p.s8 = f(t[2]);
        p.p1 = f(t[5]);
        p.p2 = f(t[6]);
    } else {
        p.s8 = f(t[1]);
        p.p1 = f(t[3]);
        p.p2 = f(t[4]);
    }
    return p;
}

static void upload_pair_table(Engine *e) {
    std::vector<double> r2r4(e->ne), r0(e->ne * e->ne);
    // recompute host copies from the device tables
    D3_CUDA(cudaMemcpy(r2r4.data(), e->t_r2r4.p, sizeof(double) * e->ne, cudaMemcpyDeviceToHost));
    D3_CUDA(cudaMemcpy(r0.data(), e->t_r0.p, sizeof(double) * e->ne * e->ne, cudaMemcpyDeviceToHost));
    std::vector<double> pa((size_t)e->ne * e->ne * 4, 0.0);
    for (int i = 0; i < e->ne; ++i)
        for (int j = 0; j < e->ne; ++j) {
            double *q = &pa[((size_t)i * e->ne + j) * 4];
            if (e->damping == 1) {
                const double R0 = std::sqrt(3.0 * r2r4[i] * r2r4[j]);
                const double A = e->fp.p1 * R0 + e->fp.p2;
                const double A2 = A * A, A4 = A2 * A2;
                q[0] = A4 * A2;
                q[1] = A4 * A4;
                q[2] = R0;
            } else {
                q[0] = r0[(size_t)i * e->ne + j];
            }
        }
    e->t_pairA.ensure(pa.size());
    D3_CUDA(cudaMemcpy(e->t_pairA.p, pa.data(), sizeof(double) * pa.size(), cudaMemcpyHostToDevice));
}

struct FullTable {
    std::vector<float> c6, r0, rcov, r2r4;
};

static const FullTable &full_table(bool extended) {
    static FullTable tabs[2];
    static std::once_flag once[2];
    const int t = extended ? 1 : 0;
    std::call_once(once[t], [t]() {
        const int NE = t ? D3_NE_EXTENDED : D3_NE_ORIGINAL, NR = t ? D3_NREF_EXTENDED : D3_NREF_ORIGINAL;
        FullTable &f = tabs[t];
        f.c6.resize((size_t)NE * NE * NR * NR * 3);
        f.r0.resize((size_t)NE * NE);
        f.rcov.resize(NE);
        f.r2r4.resize(NE);
        d3_synth_fill(D3_SYNTH_SEED, NE, NR, t, f.c6.data(), f.r0.data(), f.rcov.data(), f.r2r4.data());
    });
    return tabs[t];
}

Engine *engine_create(const uint16_t *elements, uint64_t n_elements, uint64_t max_atoms, double rc, double rc_cn,
                      double rc_atm, bool use_atm, int damping, int functional, bool extended, std::string &err,
                      uint64_t max_structs) {
    Engine *e = nullptr;
    try {
        if (!elements && n_elements) throw std::runtime_error("elements is NULL");
        if (max_atoms == 0) throw std::runtime_error("max_length must be positive");
        if (max_atoms > (uint64_t)INT32_MAX / 2) throw std::runtime_error("max_length too large");
        if (damping != 0 && damping != 1) throw std::runtime_error("unknown damping type");
        const int NE = extended ? D3_NE_EXTENDED : D3_NE_ORIGINAL;
        const int NR = extended ? D3_NREF_EXTENDED : D3_NREF_ORIGINAL;
        bool present[128] = {false};
        for (uint64_t i = 0; i < n_elements; ++i) {
            int z = elements[i];
            int slot = extended ? z - 1 : z;
            if (z >= 118 || slot < 0 || slot >= NE)
                throw std::runtime_error("element " + std::to_string(z) + " is outside the parameter table");
            present[z] = true;
        }
        e = new Engine();
        e->extended = extended;
        e->nref = NR;
        for (int z = 0; z < 118; ++z)
            if (present[z]) e->elements.push_back(z);
        e->ne = (int)e->elements.size();
        if (e->ne == 0) throw std::runtime_error("no elements given");
        if (e->ne > MAX_TYPES) throw std::runtime_error("too many distinct elements for one handle");
        e->max_atoms = max_atoms;
        if (max_structs == 0 || max_structs > max_atoms) throw std::runtime_error("bad structure capacity");
        e->max_structs = max_structs;
        e->rc = rc;
        e->rc_cn = rc_cn;
        e->rc_atm = rc_atm;
        e->rc_f = (float)rc;
        e->rc_cn_f = (float)rc_cn;
        e->use_atm = use_atm;
        e->damping = damping;
        e->functional = functional;
        e->fp = func_params(functional, damping);
        int dev = 0;
        D3_CUDA(cudaGetDevice(&dev));
        D3_CUDA(cudaDeviceGetAttribute(&e->dev_sms, cudaDevAttrMultiProcessorCount, dev));
        D3_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        // parameter tables: full synthetic table (generated once per process and layout),
        // gathered for this handle's elements
        const FullTable &tab = full_table(extended);
        const std::vector<float> &c6 = tab.c6, &r0 = tab.r0, &rcv = tab.rcov, &rr = tab.r2r4;
        const int ne = e->ne;
        std::vector<double> cnref((size_t)ne * MAX_NREF, -1.0), c6m((size_t)ne * ne * NR * NR, 0.0),
            r0m((size_t)ne * ne), rcovm(ne), r2r4m(ne);
        std::vector<int> slot(ne);
        for (int i = 0; i < ne; ++i) slot[i] = extended ? e->elements[i] - 1 : e->elements[i];
        auto C = [&](int si, int sj, int a, int b, int k) {
            return c6[((((size_t)si * NE + sj) * NR + a) * NR + b) * 3 + k];
        };
        for (int i = 0; i < ne; ++i) {
            rcovm[i] = rcv[slot[i]];
            r2r4m[i] = rr[slot[i]];
            for (int a = 0; a < NR; ++a) cnref[(size_t)i * MAX_NREF + a] = C(slot[i], slot[i], a, 0, 1) > -1.0f
                                                                                  ? (double)C(slot[i], slot[i], a, 0, 1)
                                                                                  : -1.0;
        }
        // the factorised weights need CNref to depend on (element, reference) only and
        // validity to be per element; check that for every element pair of this handle
        for (int i = 0; i < ne; ++i)
            for (int j = 0; j < ne; ++j) {
                r0m[(size_t)i * ne + j] = r0[(size_t)slot[i] * NE + slot[j]];
                for (int a = 0; a < NR; ++a)
                    for (int b = 0; b < NR; ++b) {
                        float c1 = C(slot[i], slot[j], a, b, 1), c2 = C(slot[i], slot[j], a, b, 2);
                        bool valid = c1 > -1.0f && c2 > -1.0f;
                        bool vi = cnref[(size_t)i * MAX_NREF + a] > -1.0, vj = cnref[(size_t)j * MAX_NREF + b] > -1.0;
                        if (valid != (vi && vj) ||
                            (valid && ((double)c1 != cnref[(size_t)i * MAX_NREF + a] ||
                                       (double)c2 != cnref[(size_t)j * MAX_NREF + b])))
                            throw std::runtime_error("parameter table is not separable per element; "
                                                     "the factorised C6 form cannot be used");
                        c6m[(((size_t)i * ne + j) * NR + a) * NR + b] = valid ? (double)C(slot[i], slot[j], a, b, 0) : 0.0;
                    }
            }
        e->t_cnref.ensure(cnref.size());
        e->t_c6.ensure(c6m.size());
        e->t_r0.ensure(r0m.size());
        e->t_rcov.ensure(ne);
        e->t_r2r4.ensure(ne);
        D3_CUDA(cudaMemcpy(e->t_cnref.p, cnref.data(), sizeof(double) * cnref.size(), cudaMemcpyHostToDevice));
        D3_CUDA(cudaMemcpy(e->t_c6.p, c6m.data(), sizeof(double) * c6m.size(), cudaMemcpyHostToDevice));
        D3_CUDA(cudaMemcpy(e->t_r0.p, r0m.data(), sizeof(double) * r0m.size(), cudaMemcpyHostToDevice));
        D3_CUDA(cudaMemcpy(e->t_rcov.p, rcovm.data(), sizeof(double) * ne, cudaMemcpyHostToDevice));
        D3_CUDA(cudaMemcpy(e->t_r2r4.p, r2r4m.data(), sizeof(double) * ne, cudaMemcpyHostToDevice));
        upload_pair_table(e);
        // per-atom buffers at capacity
        const size_t N = max_atoms;
        e->pos_in.ensure(3 * N);
        e->type_in.ensure(N);
        e->bin_in.ensure(N);
        e->shift_in.ensure(N);
        e->shift.ensure(N);
        e->xw_in.ensure(N);
        e->xs.ensure(N);
        e->order.ensure(N);
        e->bin_s.ensure(N);
        e->orig.ensure(N);
        e->sorted_of.ensure(N);
        e->cn.ensure(N);
        e->w.ensure(N * NR);
        e->dw.ensure(N * NR);
        e->Y.ensure(N * ne * NR);
        e->e2.ensure(N);
        e->g2.ensure(N);
        e->f2.ensure(3 * N);
        e->v2.ensure(6 * N);
        e->ea.ensure(N);
        e->ga.ensure(N);
        e->fa.ensure(3 * N);
        e->va.ensure(6 * N);
        e->eb.ensure(N);
        e->gb.ensure(N);
        e->fb.ensure(3 * N);
        e->fc.ensure(3 * N);
        e->vc.ensure(6 * N);
        e->G.ensure(N);
        e->atm_cnt.ensure(N);
        e->atm_off.ensure(N + 1);
        e->work.ensure(1);
        e->sid_in.ensure(N);
        e->sid.ensure(N);
        e->sg_dev.ensure(max_structs);
        e->out.ensure(10 * max_structs + 3 * N);
        e->status.ensure(1);
        e->counters.ensure(4);
        for (auto &x : e->ev) D3_CUDA(cudaEventCreate(&x));
        e->host_out.resize(10 * max_structs + 3 * N);
        return e;
    } catch (const std::exception &ex) {
        err = ex.what();
        delete e;
        return nullptr;
    }
}

void engine_destroy(Engine *e) {
    if (!e) return;
    if (e->stream) cudaStreamSynchronize(e->stream);
    delete e;
}

void engine_set_options(Engine *e, const Options &o) {
    const bool regrid = o.bin_divisor != e->opt.bin_divisor;
    const bool recap = o.atm_list_capacity != e->opt.atm_list_capacity;
    e->opt = o;
    if (recap && e->use_atm) {
        // a given capacity replaces the estimate (0: estimate again at the next evaluation)
        e->atm_cap = o.atm_list_capacity;
        if (e->atm_cap > 0) e->atm_ent.ensure((size_t)e->atm_cap);
    }
    if (regrid && e->cell_set && e->nstruct > 0) {
        const std::vector<uint64_t> c = e->counts;
        const std::vector<double> cl = e->cells;
        const std::vector<float> cf = e->cells_f;
        build_structures(e, e->nstruct, c.data(), cl.data(), cf.data());
    }
}
Options engine_get_options(const Engine *e) { return e->opt; }
void engine_set_functional_params(Engine *e, const FuncParams &p) {
    e->fp = p;
    upload_pair_table(e);
}
uint64_t engine_num_atoms(const Engine *e) { return e->n; }
const double *engine_device_results(const Engine *e) { return e->out.p; }

static std::vector<int> map_types(const Engine *e, const uint16_t *Z, uint64_t n) {
    std::vector<int> types(n);
    for (uint64_t i = 0; i < n; ++i) {
        auto it = std::lower_bound(e->elements.begin(), e->elements.end(), (int)Z[i]);
        if (it == e->elements.end() || *it != (int)Z[i])
            throw std::runtime_error("element " + std::to_string(Z[i]) + " was not given when the handle was created");
        types[i] = (int)(it - e->elements.begin());
    }
    return types;
}

// Geometry of every structure: reference image box and workload decision, bin grid,
// stencils; uploads the records, the stencil rows and the per-atom structure index.
static void build_structures(Engine *e, int nstruct, const uint64_t *counts, const double *cells,
                             const float *cells_f) {
    std::vector<SG> sg(nstruct);
    std::vector<CellGeom> geoms(nstruct);
    std::vector<int4> rows, srow;
    std::vector<int> sid;
    int bin_base = 0, atom_base = 0;
    const double rmin = std::min(e->rc_cn, e->use_atm ? std::min(e->rc, e->rc_atm) : e->rc);
    const double target = std::max(rmin / e->opt.bin_divisor, 1.0);
    for (int k = 0; k < nstruct; ++k) {
        for (int i = 0; i < 9; ++i)
            if (!std::isfinite(cells[9 * k + i])) throw std::runtime_error("cell has a non-finite entry");
        CellGeom g = make_geom(cells + 9 * k);
        if (!(std::fabs(g.volume) > 1e-12) || !std::isfinite(g.volume)) throw std::runtime_error("degenerate cell");
        geoms[k] = g;
        SG &r = sg[k];
        memset(&r, 0, sizeof(SG));
        for (int i = 0; i < 9; ++i) {
            r.h[i] = g.h[i];
            r.inv[i] = g.inv[i];
        }
        r.vol = g.volume;
        // a nonzero lattice vector is at least as long as the smallest height, so with every
        // height above 2 rc_ATM two images of one atom never lie within rc_ATM of an apex
        r.atm_simple = std::min(g.height[0], std::min(g.height[1], g.height[2])) > 2.0 * e->rc_atm * (1.0 + 1e-9);
        int64_t mcb[3];
        r.box_mode = reference_box(cells_f + 9 * k, e->rc_f, e->rc_cn_f, mcb) ? 1 : 0;
        for (int i = 0; i < 3; ++i) r.half[i] = (int)(mcb[i] / 2);
        const int64_t max_bins = std::max<int64_t>(64, (int64_t)std::max<uint64_t>(counts[k], 1) * 2);
        choose_bins(g, target, max_bins, r.nb);
        r.nbins = r.nb[0] * r.nb[1] * r.nb[2];
        r.bin_base = bin_base;
        bin_base += r.nbins;
        r.atom_base = atom_base;
        r.natoms = (int)counts[k];
        atom_base += (int)counts[k];
        auto add = [&](double rc, int &off, int &cnt) {
            auto st = build_stencil(g, r.nb, rc);
            off = (int)rows.size();
            cnt = (int)st.size();
            for (auto &x : st) rows.push_back(make_int4(x.dy, x.dz, x.dxlo, x.dxhi));
        };
        add(e->rc, r.st2_off, r.st2_n);
        add(e->rc_cn, r.stc_off, r.stc_n);
        if (e->use_atm) add(e->rc_atm, r.sta_off, r.sta_n);
        // two-body atom groups: blocks of gy x gz bin rows holding about 16 atoms per
        // column, so that a group of 32 spans one or two columns
        {
            const double per_bin = (double)counts[k] / std::max(1, r.nbins);
            const int gb = std::max(1, std::min(4, (int)std::lround(std::sqrt(16.0 / std::max(per_bin, 1e-3)))));
            const int gy = std::min(gb, r.nb[1]), gz = std::min(gb, r.nb[2]);
            std::vector<StencilRow> s2;
            for (int q = r.st2_off; q < r.st2_off + r.st2_n; ++q)
                s2.push_back({rows[q].x, rows[q].y, rows[q].z, rows[q].w});
            const auto blk = merge_block_stencil(s2, gy, gz);
            r.st2b_off = (int)rows.size();
            r.st2b_n = (int)blk.size();
            for (auto &x : blk) rows.push_back(make_int4(x.dy, x.dz, x.dxlo, x.dxhi));
            std::vector<StencilRow> sc;
            for (int q = r.stc_off; q < r.stc_off + r.stc_n; ++q)
                sc.push_back({rows[q].x, rows[q].y, rows[q].z, rows[q].w});
            const auto blkc = merge_block_stencil(sc, gy, gz);
            r.stcb_off = (int)rows.size();
            r.stcb_n = (int)blkc.size();
            for (auto &x : blkc) rows.push_back(make_int4(x.dy, x.dz, x.dxlo, x.dxhi));
            if (e->use_atm) {
                std::vector<StencilRow> sa;
                for (int q = r.sta_off; q < r.sta_off + r.sta_n; ++q)
                    sa.push_back({rows[q].x, rows[q].y, rows[q].z, rows[q].w});
                const auto blka = merge_block_stencil(sa, gy, gz);
                r.stab_off = (int)rows.size();
                r.stab_n = (int)blka.size();
                for (auto &x : blka) rows.push_back(make_int4(x.dy, x.dz, x.dxlo, x.dxhi));
            }
            for (int bz = 0; bz < r.nb[2]; bz += gz)
                for (int by = 0; by < r.nb[1]; by += gy)
                    srow.push_back(make_int4(k, by, bz, std::min(gy, r.nb[1] - by) | (std::min(gz, r.nb[2] - bz) << 8)));
        }
        sid.insert(sid.end(), counts[k], k);
    }
    e->sg = sg;
    e->geoms = geoms;
    e->counts.assign(counts, counts + nstruct);
    e->cells.assign(cells, cells + 9 * (size_t)nstruct);
    e->cells_f.assign(cells_f, cells_f + 9 * (size_t)nstruct);
    e->stencil_rows = rows;
    e->srow_host = srow;
    // groups: at most ceil(atoms of a super-row / 32) per super-row
    e->group_bound = 0;
    for (int k = 0; k < nstruct; ++k) e->group_bound += counts[k] / 32;
    e->group_bound += srow.size() + 1;
    e->srows.ensure(std::max<size_t>(1, srow.size()));
    if (!srow.empty())
        D3_CUDA(cudaMemcpy(e->srows.p, srow.data(), sizeof(int4) * srow.size(), cudaMemcpyHostToDevice));
    e->groups.ensure(e->group_bound);
    e->gctl.ensure(6); // [0] groups, [1..5] work counters: CN, two-body, chain, ATM list count, fill
    e->anyshift.ensure(std::max(1, nstruct));
    e->nstruct = nstruct;
    e->nbins_total = bin_base;
    e->sg_dev.ensure(nstruct);
    D3_CUDA(cudaMemcpy(e->sg_dev.p, sg.data(), sizeof(SG) * nstruct, cudaMemcpyHostToDevice));
    e->st_dev.ensure(rows.size());
    if (!rows.empty())
        D3_CUDA(cudaMemcpy(e->st_dev.p, rows.data(), sizeof(int4) * rows.size(), cudaMemcpyHostToDevice));
    e->bin_cnt.ensure(bin_base);
    e->bin_fill.ensure(bin_base);
    e->bin_start.ensure(bin_base + 1);
    if (!sid.empty()) D3_CUDA(cudaMemcpy(e->sid_in.p, sid.data(), sizeof(int) * sid.size(), cudaMemcpyHostToDevice));
}

int engine_set_atoms(Engine *e, const double *pos_bohr, const uint16_t *Z, uint64_t n, std::string &err) {
    try {
        if (n > e->max_atoms)
            throw std::runtime_error("length " + std::to_string(n) + " exceeds the handle capacity " +
                                     std::to_string(e->max_atoms));
        if (n == 0) throw std::runtime_error("no atoms given");
        std::vector<int> types = map_types(e, Z, n);
        D3_CUDA(cudaMemcpyAsync(e->pos_in.p, pos_bohr, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, e->stream));
        D3_CUDA(cudaMemcpyAsync(e->type_in.p, types.data(), sizeof(int) * n, cudaMemcpyHostToDevice, e->stream));
        D3_CUDA(cudaStreamSynchronize(e->stream));
        const bool recount = e->n != n;
        e->n = n;
        e->atoms_set = true;
        if (e->cell_set && (recount || e->nstruct != 1)) {
            const uint64_t c = n;
            build_structures(e, 1, &c, e->first_cell, e->first_cell_f);
        }
        return 0;
    } catch (const std::exception &ex) {
        err = ex.what();
        return 1;
    }
}

int engine_set_cell(Engine *e, const double cell[9], const float cell_f[9], std::string &err) {
    try {
        for (int i = 0; i < 9; ++i) {
            e->first_cell[i] = cell[i];
            e->first_cell_f[i] = cell_f[i];
        }
        const uint64_t c = e->n;
        build_structures(e, 1, &c, cell, cell_f);
        e->cell_set = true;
        e->cell_status = 0;
        return 0;
    } catch (const std::exception &ex) {
        // an evaluation without a valid cell returns this status (not the generic "not set")
        e->cell_set = false;
        err = ex.what();
        e->cell_status = err.find("non-finite") != std::string::npos ? ST_BAD_INPUT : ST_BAD_CELL;
        return 1;
    }
}

int engine_set_batch(Engine *e, uint64_t nstruct, const uint64_t *counts, const double *pos_bohr, const uint16_t *Z,
                     const double *cells_bohr, const float *cells_f, std::string &err) {
    try {
        if (nstruct == 0 || nstruct > e->max_structs)
            throw std::runtime_error("structure count " + std::to_string(nstruct) + " outside 1.." +
                                     std::to_string(e->max_structs));
        uint64_t n = 0;
        for (uint64_t k = 0; k < nstruct; ++k) {
            if (counts[k] == 0) throw std::runtime_error("structure without atoms");
            n += counts[k];
        }
        if (n > e->max_atoms)
            throw std::runtime_error(std::to_string(n) + " atoms exceed the handle capacity " + std::to_string(e->max_atoms));
        std::vector<int> types = map_types(e, Z, n);
        build_structures(e, (int)nstruct, counts, cells_bohr, cells_f);
        D3_CUDA(cudaMemcpyAsync(e->pos_in.p, pos_bohr, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, e->stream));
        D3_CUDA(cudaMemcpyAsync(e->type_in.p, types.data(), sizeof(int) * n, cudaMemcpyHostToDevice, e->stream));
        D3_CUDA(cudaStreamSynchronize(e->stream));
        e->n = n;
        e->atoms_set = true;
        e->cell_set = true;
        return 0;
    } catch (const std::exception &ex) {
        err = ex.what();
        return 1;
    }
}

__global__ void k_set_positions(double *pos_in, const double *coords_ang, int n3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n3) pos_in[i] = coords_ang[i] * ANG2BOHR;
}

int engine_set_positions_device(Engine *e, const double *coords_ang_dev, cudaStream_t stream) {
    if (!e->atoms_set) return 1;
    const int n3 = (int)(3 * e->n);
    k_set_positions<<<(n3 + 255) / 256, 256, 0, stream ? stream : e->stream>>>(e->pos_in.p, coords_ang_dev, n3);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int engine_num_structures(const Engine *e) { return e->nstruct; }

void engine_fetch_results(Engine *e, double *energies, double *forces, double *stresses) {
    const size_t S = e->nstruct, n = e->n;
    std::vector<double> h(10 * S + 3 * n);
    D3_CUDA(cudaMemcpy(h.data(), e->out.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
    if (energies) memcpy(energies, h.data(), sizeof(double) * S);
    if (forces) memcpy(forces, h.data() + S, sizeof(double) * 3 * n);
    if (stresses) memcpy(stresses, h.data() + S + 3 * n, sizeof(double) * 9 * S);
}

// warps per CTA of the block-pair ATM kernel for this handle, 0 when it is not used
// (plain form, surrogate, mirror schedule chosen, or the type count leaves too little
// shared memory)
struct AtmbShape {
    int warps, ctas, mcap, nbuf; // warps per CTA (0: kernel not used), CTAs per SM, longest
                                 // list, y buffers per warp
};
static AtmbShape blockpair_shape(const Engine *e) {
    if (!e->use_atm || !e->opt.precision || e->opt.atm_schedule != 0) return {0, 0, 0, 0};
    if (e->opt.atm_surrogate && e->surr.loaded) return {0, 0, 0, 0};
    const size_t limit = 227 * 1024 - 2048; // opt-in maximum minus the static arrays
    // a requested shape (autotuner): warps per CTA (more than 8 with one y buffer per
    // warp), CTAs per SM (2 when both fit), list capacity; kept only if it fits
    if (e->opt.atmb_warps > 0) {
        const int w = std::min(e->opt.atmb_warps, ATMB_MAXW1);
        const int nbuf = w > ATMB_MAXW ? 1 : 2;
        const size_t per = atmb_smem_warp(e->ne, e->nref, nbuf);
        const int ctas = e->opt.atm_ctas_per_sm == 2 ? 2 : 1;
        const size_t cap_sm = ctas == 2 ? (228 * 1024) / 2 - 2048 : limit;
        int mcap = e->opt.atmb_mcap > 0 ? std::max(ATMB_MCAP_MIN, std::min(ATMB_MCAP_MAX, e->opt.atmb_mcap & ~511))
                                        : ATMB_MCAP_MAX;
        while (mcap >= ATMB_MCAP_MIN && atmb_smem_fixed(e->ne, e->nref, mcap) + w * per > cap_sm) mcap -= 512;
        // the entry sort's cell counters live in the warps' staging area
        if (w >= 2 && mcap >= ATMB_MCAP_MIN && w * per >= ATMB_CELLS * sizeof(int)) return {w, ctas, mcap, nbuf};
    }
    // default: up to 12 warps with one y buffer each (three warps per scheduler hide each
    // other's copies; measured 266 ms against 288 ms with 8 double-buffered warps on the
    // 20,000-atom box), as long as the shared memory leaves a list capacity of 4,096
    for (int w = ATMB_MAXW1; w > ATMB_MAXW; --w) {
        const size_t per1 = atmb_smem_warp(e->ne, e->nref, 1);
        int mcap = ATMB_MCAP_MAX;
        while (mcap >= ATMB_MCAP_MIN && atmb_smem_fixed(e->ne, e->nref, mcap) + w * per1 > limit) mcap -= 512;
        if (mcap >= ATMB_MCAP_MIN && w * per1 >= ATMB_CELLS * sizeof(int)) return {w, 1, mcap, 1};
    }
    const size_t per = atmb_smem_warp(e->ne, e->nref);
    // two CTAs of four warps per SM, so that one CTA's per-apex sort and set-up overlap the
    // other's block pairs, when both fit the SM's 228 KB (each with 2 KB for the static
    // arrays and the system's share)
    if (ATMB_CTAS_PER_SM == 2 && 2 * (atmb_smem_fixed(e->ne, e->nref, ATMB_MCAP_MIN) + 4 * per + 2048) <= 228 * 1024)
        return {4, 2, ATMB_MCAP_MIN, 2};
    // else one CTA of up to ATMB_MAXW warps; the shared memory they leave sets the list
    // capacity (longer lists go to the mirror kernel)
    for (int w = ATMB_MAXW; w >= 2; --w) {
        int mcap = ATMB_MCAP_MAX;
        while (mcap >= ATMB_MCAP_MIN && atmb_smem_fixed(e->ne, e->nref, mcap) + w * per > limit) mcap -= 512;
        if (mcap >= ATMB_MCAP_MIN) return {w, 1, mcap, 2};
    }
    return {0, 0, 0, 0};
}
static int blockpair_warps(const Engine *e) { return blockpair_shape(e).warps; }

// the two-body pass on atom groups (d3_pairs.cuh), unless chosen off or the handle has more
// element types than the staged rows hold; sharded evaluations (which split by central
// atom) take the per-atom kernels whatever this says
static bool pairs_grouped(const Engine *e) { return e->opt.pair_kernel == 0 && e->ne <= PAIRS_MAX_TYPES; }

static size_t pairs_smem(const Engine *e) {
    const bool f64 = e->opt.precision == 0;
    const size_t rsz = f64 ? sizeof(double) : sizeof(float);
    const size_t tab = ((size_t)3 * e->ne * e->ne * rsz + 15) & ~(size_t)15;
    return tab + PAIRS_WARPS * (f64 ? pairs_warp_bytes<true>(e->ne, e->nref) : pairs_warp_bytes<false>(e->ne, e->nref));
}

static const void *pairs_kernel(const Engine *e) {
    const bool f64 = e->opt.precision == 0;
    if (e->nref == 5) return f64 ? (const void *)k_twobody_g<5, true> : (const void *)k_twobody_g<5, false>;
    return f64 ? (const void *)k_twobody_g<7, true> : (const void *)k_twobody_g<7, false>;
}

// CTAs per SM of the grouped two-body kernel (attribute and query cached, so that an
// evaluation inside a graph capture makes no such call)
static int pairs_occupancy(Engine *e) {
    auto &c = e->atm_occ_cache[5];
    const void *fn = pairs_kernel(e);
    const size_t sm = pairs_smem(e);
    if (c.fn == fn && c.sm == sm) return c.blocks;
    D3_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int blocks = 0;
    D3_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, PAIRS_WARPS * 32, sm));
    c.fn = fn;
    c.sm = sm;
    c.blocks = std::max(1, blocks);
    return c.blocks;
}

static KP make_kp(Engine *e) {
    KP p;
    memset(&p, 0, sizeof(p));
    p.shard_rank = 0;
    p.shard_world = 1;
    p.n = (int)e->n;
    p.nstruct = e->nstruct;
    p.nbins_total = e->nbins_total;
    p.ne = e->ne;
    p.nref = e->nref;
    p.sg = e->sg_dev.p;
    p.sid_in = e->sid_in.p;
    p.sid = e->sid.p;
    p.stencils = e->st_dev.p;
    // cutoffs: the reference compares squared distances against rc*rc of its float cutoff
    p.rc2 = e->rc * e->rc;
    p.rcn2 = e->rc_cn * e->rc_cn;
    p.ratm2 = e->rc_atm * e->rc_atm;
    p.rc_cn = e->rc_cn;
    p.cnref = e->t_cnref.p;
    p.c6 = e->t_c6.p;
    p.r0ab = e->t_r0.p;
    p.rcov = e->t_rcov.p;
    p.r2r4 = e->t_r2r4.p;
    p.pairA = e->t_pairA.p;
    p.s6 = e->fp.s6;
    p.s8 = e->fp.s8;
    p.p1 = e->fp.p1;
    p.p2 = e->fp.p2;
    p.damping = e->damping;
    p.smooth_cn = e->opt.smooth_cn ? 1 : 0;
    p.precision = e->opt.precision;
    if (p.precision) {
        const size_t N = e->max_atoms;
        e->xs32.ensure(N);
        e->w32.ensure(N * e->nref);
        e->dw32.ensure(N * e->nref);
        e->Y32.ensure(N * e->ne * e->nref);
    }
    p.xs32 = e->xs32.p;
    p.w32 = e->w32.p;
    p.dw32 = e->dw32.p;
    p.Y32 = e->Y32.p;
    p.YD32 = nullptr;
    p.atm_min_m = 0;
    p.atmb_split = 1;
    if (blockpair_warps(e) > 0) {
        e->YD32.ensure((size_t)e->max_atoms * e->ne * atmb_row_floats(e->nref));
        const AtmbShape sh = blockpair_shape(e);
        e->atmb_scratch.ensure((size_t)e->dev_sms * sh.ctas * atmb_scratch_per_cta(sh.mcap));
        p.atmb_mcap = sh.mcap;
        p.YD32 = e->YD32.p;
        // few apexes (small structures): split each apex's block rows over several CTAs so
        // that about three work items per CTA exist (every split repeats the apex's entry
        // sort and set-up: on the 96-atom water box splits 3 / 5 / 7 / 10 / 16 took
        // 1.60 / 1.48 / 1.78 / 2.13 / 2.77 ms)
        const int ctas = e->dev_sms * sh.ctas;
        p.atmb_split = e->opt.atmb_split > 0 ? std::min(e->opt.atmb_split, 64)
                                             : std::max(1, std::min(16, (3 * ctas + p.n - 1) / std::max(1, p.n)));
    }
    p.atm_force_scaled = e->opt.atm_force_scaled ? 1 : 0;
    p.anyshift = e->anyshift.p;
    p.srows = e->srows.p;
    p.nsrow = (int)e->srow_host.size();
    p.groups = e->groups.p;
    p.gcount = e->gctl.p;
    p.gslices = 0;
    p.gpart = nullptr;
    if (pairs_grouped(e)) {
        // slices per group: about six work items per resident warp, so that the items
        // taken last are short against the pass
        const int warps = e->dev_sms * pairs_occupancy(e) * PAIRS_WARPS;
        const long long want = (6LL * warps + (long long)e->group_bound - 1) / std::max<long long>(1, e->group_bound);
        p.gslices = (int)std::max<long long>(1, std::min<long long>(64, want));
        e->gpart.ensure((size_t)p.gslices * e->max_atoms * PAIRS_NSUM);
        p.gpart = e->gpart.p;
    }
    p.pos_in = e->pos_in.p;
    p.type_in = e->type_in.p;
    p.bin_in = e->bin_in.p;
    p.shift_in = e->shift_in.p;
    p.xw_in = e->xw_in.p;
    p.bin_cnt = e->bin_cnt.p;
    p.bin_start = e->bin_start.p;
    p.bin_fill = e->bin_fill.p;
    p.order = e->order.p;
    p.xs = e->xs.p;
    p.shift = e->shift.p;
    p.bin_s = e->bin_s.p;
    p.orig = e->orig.p;
    p.sorted_of = e->sorted_of.p;
    p.cn = e->cn.p;
    p.w = e->w.p;
    p.dw = e->dw.p;
    p.Y = e->Y.p;
    p.e2 = e->e2.p;
    p.g2 = e->g2.p;
    p.f2 = e->f2.p;
    p.v2 = e->v2.p;
    p.ea = e->ea.p;
    p.ga = e->ga.p;
    p.fa = e->fa.p;
    p.va = e->va.p;
    p.eb = e->eb.p;
    p.gb = e->gb.p;
    p.fb = e->fb.p;
    p.fc = e->fc.p;
    p.vc = e->vc.p;
    p.atm_cnt = e->atm_cnt.p;
    p.atm_off = e->atm_off.p;
    p.atm_ent = e->atm_ent.p;
    p.atm_cap = e->atm_cap;
    p.work = e->work.p;
    p.out = e->out.p;
    p.status = e->status.p;
    p.counters = e->counters.p;
    return p;
}

// the block-pair ATM kernel instance of a buffering, apex kind and skip granularity
template <int NR, int NBUF, bool SIMPLE>
static const void *blockpair_fn(bool fine) {
    return fine ? (const void *)k_atm32b<NR, NBUF, SIMPLE, true> : (const void *)k_atm32b<NR, NBUF, SIMPLE, false>;
}

// dynamic shared memory attribute and occupancy of an ATM kernel, cached per kernel and
// size so that evaluations inside a CUDA-graph capture make no such host calls
static int atm_occupancy(Engine *e, int which, size_t sm, const void *fn) {
    auto &c = e->atm_occ_cache[which];
    if (c.fn == fn && c.sm == sm) return c.blocks;
    D3_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int blocks = 0;
    D3_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, ATM_THREADS, sm));
    c.fn = fn;
    c.sm = sm;
    c.blocks = std::max(1, blocks);
    return c.blocks;
}

// one launch of the block-pair ATM kernel for the apexes of one kind (weight-free or not)
template <int NR>
static void launch_blockpair(Engine *e, const KP &p, cudaStream_t s, const AtmbShape &shb, bool simple, int grid,
                             size_t smb) {
    const bool fine = e->opt.atmb_fine_skip != 0;
    const void *fn = shb.nbuf == 2 ? (simple ? blockpair_fn<NR, 2, true>(fine) : blockpair_fn<NR, 2, false>(fine))
                                   : (simple ? blockpair_fn<NR, 1, true>(fine) : blockpair_fn<NR, 1, false>(fine));
    atm_occupancy(e, 8 + (shb.nbuf == 2 ? 0 : 2) + (simple ? 1 : 0), smb, fn);
    void *args[] = {(void *)&p, (void *)&e->atmb_scratch.p};
    D3_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(32 * shb.warps), args, smb, s));
}

static SurrDesc surr_desc(const int *chan, int nch, float *G, const float *dEdG, int *center) {
    SurrDesc sd{};
    sd.chan = chan;
    sd.nch = nch;
    sd.mu0 = (float)(SURR_MU0_A * ANG2BOHR);
    sd.dmu = (float)((SURR_MU1_A - SURR_MU0_A) / (SURR_NRBF - 1) * ANG2BOHR);
    const double sig = SURR_SIGMA_A * ANG2BOHR;
    sd.inv2s2 = (float)(1.0 / (2.0 * sig * sig));
    sd.G = G;
    sd.dEdG = dEdG;
    sd.center = center;
    return sd;
}

static d3mlp::Net surr_net(const SurrState &S) {
    d3mlp::Net net;
    net.L = S.L;
    net.members = S.members;
    net.master = S.master.p;
    net.packed = S.packed.p;
    net.mean = S.mean.p;
    net.inv_std = S.inv_std.p;
    return net;
}

// stage 0: the whole evaluation; stage 1: everything up to the summed dE/dCN (written to
// G_ext when given); stage 2: chain rule (dE/dCN read from G_ext), forces and reductions.
// Stages 1 and 2 with an all-reduce of dE/dCN between them make a sharded evaluation.
template <int NR>
static void launch_all(Engine *e, const KP &p0, cudaStream_t s, int stage = 0, double *G_ext = nullptr) {
    KP p = p0;
    const int n = p.n;
    const int T = 256;
    const int gb = (n + T - 1) / T;
    const int gw = (int)(((long long)n * 32 + T - 1) / T);
    cudaEvent_t *ev = e->ev;
    double *Gsum = G_ext ? G_ext : e->G.p;
    if (stage != 2) {
        D3_CUDA(cudaEventRecord(ev[0], s));
        D3_CUDA(cudaMemsetAsync(p.counters, 0, sizeof(unsigned long long) * 4, s));
        D3_CUDA(cudaMemsetAsync(p.anyshift, 0, sizeof(int) * p.nstruct, s));
        D3_CUDA(cudaMemsetAsync(p.bin_cnt, 0, sizeof(int) * p.nbins_total, s));
        D3_CUDA(cudaMemsetAsync(p.bin_fill, 0, sizeof(int) * p.nbins_total, s));
        k_bin<<<gb, T, 0, s>>>(p);
        k_scan<int, int><<<1, 1024, 0, s>>>(p.bin_cnt, p.bin_start, p.nbins_total);
        k_scatter<<<gb, T, 0, s>>>(p);
        k_binsort<<<(p.nbins_total + T - 1) / T, T, 0, s>>>(p);
        k_gather<<<gb, T, 0, s>>>(p);
        if (p.gslices > 0) {
            D3_CUDA(cudaMemsetAsync(e->gctl.p, 0, 6 * sizeof(int), s));
            k_groups<<<(p.nsrow + 127) / 128, 128, 0, s>>>(p);
        }
        D3_CUDA(cudaEventRecord(ev[1], s));
        if (p.gslices > 0) {
            const size_t sm = 64 + PAIRS_WARPS * 32 * (p.precision ? sizeof(float4) : sizeof(double4));
            if (p.precision)
                k_cn_g<false><<<e->dev_sms * 2, PAIRS_WARPS * 32, sm, s>>>(p, e->gctl.p + 1);
            else
                k_cn_g<true><<<e->dev_sms * 2, PAIRS_WARPS * 32, sm, s>>>(p, e->gctl.p + 1);
            k_group_reduce<<<gb, T, 0, s>>>(p, 1);
        } else if (p.precision)
            k_cn32<<<gw, T, 0, s>>>(p);
        else
            k_cn<<<gw, T, 0, s>>>(p);
        k_weights<NR><<<gb, T, 0, s>>>(p);
        D3_CUDA(cudaEventRecord(ev[2], s));
        if (p.shard_world > 1) {
            // only this shard's central atoms are written
            D3_CUDA(cudaMemsetAsync(p.e2, 0, sizeof(double) * n, s));
            D3_CUDA(cudaMemsetAsync(p.g2, 0, sizeof(double) * n, s));
            D3_CUDA(cudaMemsetAsync(p.f2, 0, sizeof(double) * 3 * n, s));
            D3_CUDA(cudaMemsetAsync(p.v2, 0, sizeof(double) * 6 * n, s));
        }
        if (p.gslices > 0) {
            const int grid = e->dev_sms * pairs_occupancy(e);
            if (p.precision)
                k_twobody_g<NR, false><<<grid, PAIRS_WARPS * 32, pairs_smem(e), s>>>(p, e->gctl.p + 2);
            else
                k_twobody_g<NR, true><<<grid, PAIRS_WARPS * 32, pairs_smem(e), s>>>(p, e->gctl.p + 2);
            k_group_reduce<<<gb, T, 0, s>>>(p, 0);
        } else if (p.precision)
            k_twobody32<NR><<<gw, T, (size_t)p.ne * p.ne * sizeof(float4), s>>>(p);
        else
            k_twobody<NR><<<gw, T, 0, s>>>(p);
        D3_CUDA(cudaEventRecord(ev[3], s));
        D3_CUDA(cudaMemsetAsync(p.ea, 0, sizeof(double) * n, s));
        D3_CUDA(cudaMemsetAsync(p.ga, 0, sizeof(double) * n, s));
        D3_CUDA(cudaMemsetAsync(p.fa, 0, sizeof(double) * 3 * n, s));
        D3_CUDA(cudaMemsetAsync(p.va, 0, sizeof(double) * 6 * n, s));
        D3_CUDA(cudaMemsetAsync(p.eb, 0, sizeof(double) * n, s));
        D3_CUDA(cudaMemsetAsync(p.gb, 0, sizeof(double) * n, s));
        D3_CUDA(cudaMemsetAsync(p.fb, 0, sizeof(double) * 3 * n, s));
        // learned surrogate: descriptors -> ensemble -> fallback flags; the exact ATM pass
        // below then runs in centre mode over the flagged atoms only
        const bool surr = e->use_atm && e->opt.atm_surrogate && e->surr.loaded;
        KP pc = p;
        SurrDesc sd{};
        if (surr) {
            SurrState &S = e->surr;
            sd = surr_desc(S.chan.p, S.L.nch, S.G.p, S.dX.p, S.center.p);
            k_desc_fwd<NR><<<gw, T, 0, s>>>(p, sd);
            d3mlp::infer(surr_net(S), S.G.p, S.center.p, n, S.E.p, S.dX.p, e->dev_sms, s);
            D3_CUDA(cudaMemsetAsync(S.napex.p, 0, sizeof(int), s));
            SurrComb c{};
            c.E = S.E.p;
            c.dX = S.dX.p;
            c.center = S.center.p;
            c.e_shift = S.e_shift.p;
            c.e_scale = S.e_scale;
            c.members = S.members;
            c.nfeat = S.L.nch * SURR_NRBF;
            c.thr = S.thr_ev;
            c.flag = S.flag.p;
            c.apex = S.apex.p;
            c.napex = S.napex.p;
            k_surr_combine<<<gw, T, 0, s>>>(p, c);
            pc.atm_center = 1;
            pc.atm_apex = S.apex.p;
            pc.atm_napex = S.napex.p;
            pc.surr_flag = S.flag.p;
        }
        if (e->use_atm && p.gslices > 0) {
            const size_t sm = PAIRS_WARPS * 32 * (sizeof(double4) + sizeof(int));
            k_atm_list_g<false><<<e->dev_sms * 2, PAIRS_WARPS * 32, sm, s>>>(pc, e->gctl.p + 4);
            k_atm_list_prefix<<<gb, T, 0, s>>>(pc);
            k_scan<long long, int><<<1, 1024, 0, s>>>(p.atm_cnt, p.atm_off, n);
            k_atm_list_g<true><<<e->dev_sms * 2, PAIRS_WARPS * 32, sm, s>>>(pc, e->gctl.p + 5);
        } else if (e->use_atm) {
            k_atm_list<false><<<gw, T, 0, s>>>(pc);
            k_scan<long long, int><<<1, 1024, 0, s>>>(p.atm_cnt, p.atm_off, n);
            k_atm_list<true><<<gw, T, 0, s>>>(pc);
        }
        D3_CUDA(cudaEventRecord(ev[4], s));
        if (e->use_atm) {
            D3_CUDA(cudaMemsetAsync(p.work, 0, sizeof(int), s));
            if (p.precision) {
                const size_t fixed = (size_t)p.ne * NR * sizeof(double) + ((p.ne * p.ne + 3) & ~3) * sizeof(float) +
                                     ATM_PERM_CAP * sizeof(unsigned short) + 11 * ATM_THREADS * sizeof(double);
                const size_t per = 2 * sizeof(float4) + sizeof(int2) + (size_t)p.ne * 2 * sizeof(float4);
                const int tmax = (int)std::max<size_t>(32, std::min<size_t>(256, (100 * 1024 - fixed) / per)) & ~31;
                const int tile = e->opt.atm_tile > 0 ? std::min(tmax, std::max(32, e->opt.atm_tile & ~31)) : std::min(tmax, 128);
                const size_t sm = (size_t)tile * per + fixed;
                const AtmbShape shb = blockpair_shape(e);
                const int nwb = shb.warps;
                if (nwb > 0 && !surr) {
                    // lists up to shb.mcap entries: block-pair schedule; longer ones below
                    const size_t smb =
                        atmb_smem_fixed(p.ne, NR, shb.mcap) + (size_t)nwb * atmb_smem_warp(p.ne, NR, shb.nbuf);
                    // one launch per apex kind present: weight-free structures (every cell
                    // height above 2 rc_ATM) and the others
                    bool kind[2] = {false, false};
                    for (const SG &q : e->sg) kind[q.atm_simple ? 1 : 0] = true;
                    const int grid = e->dev_sms * shb.ctas;
                    for (int k = 1; k >= 0; --k) {
                        if (!kind[k]) continue;
                        if (k == 0 && kind[1]) D3_CUDA(cudaMemsetAsync(p.work, 0, sizeof(int), s));
                        launch_blockpair<NR>(e, p, s, shb, k == 1, grid, smb);
                    }
                    D3_CUDA(cudaMemsetAsync(p.work, 0, sizeof(int), s));
                    pc.atm_min_m = shb.mcap;
                }
                const void *fn = surr ? (const void *)k_atm32<NR, true> : (const void *)k_atm32<NR, false>;
                const int blocks_per_sm = atm_occupancy(e, surr ? 3 : 1, sm, fn);
                const int per_sm = e->opt.atm_ctas_per_sm > 0 ? std::min(e->opt.atm_ctas_per_sm, blocks_per_sm) : blocks_per_sm;
                const int grid = std::max(1, std::min(n, e->dev_sms * std::max(1, per_sm)));
                if (surr)
                    k_atm32<NR, true><<<grid, ATM_THREADS, sm, s>>>(pc, tile);
                else
                    k_atm32<NR, false><<<grid, ATM_THREADS, sm, s>>>(pc, tile);
            } else {
                // partner tile: as many entries as fit in ~160 KB next to the apex tables
                const size_t fixed = (size_t)p.ne * NR * sizeof(double) + (size_t)p.ne * p.ne * sizeof(double) +
                                     ATM_PERM_CAP * sizeof(unsigned short);
                const size_t per = sizeof(Partner) + (size_t)p.ne * NR * sizeof(double);
                const int tmax = (int)std::max<size_t>(8, std::min<size_t>(256, (160 * 1024 - fixed) / per));
                const int tile = e->opt.atm_tile > 0 ? std::min(tmax, std::max(8, e->opt.atm_tile)) : std::min(tmax, 128);
                const size_t sm = (size_t)tile * per + fixed;
                const void *fn = surr ? (const void *)k_atm<NR, true> : (const void *)k_atm<NR, false>;
                const int blocks_per_sm = atm_occupancy(e, surr ? 2 : 0, sm, fn);
                const int per_sm = e->opt.atm_ctas_per_sm > 0 ? std::min(e->opt.atm_ctas_per_sm, blocks_per_sm) : blocks_per_sm;
                const int grid = std::max(1, std::min(n, e->dev_sms * std::max(1, per_sm)));
                if (surr)
                    k_atm<NR, true><<<grid, ATM_THREADS, sm, s>>>(pc, tile);
                else
                    k_atm<NR, false><<<grid, ATM_THREADS, sm, s>>>(pc, tile);
            }
            if (surr) k_desc_bwd<NR><<<gw, T, 0, s>>>(p, sd);
        }
        D3_CUDA(cudaEventRecord(ev[5], s));
        k_sum_g<<<gb, T, 0, s>>>(p, Gsum);
        if (stage == 1) {
            D3_CUDA(cudaGetLastError());
            return;
        }
    } // stage != 2
    if (p.shard_world > 1) {
        D3_CUDA(cudaMemsetAsync(p.fc, 0, sizeof(double) * 3 * n, s));
        D3_CUDA(cudaMemsetAsync(p.vc, 0, sizeof(double) * 6 * n, s));
    }
    if (p.gslices > 0) {
        const size_t sm = 64 + PAIRS_WARPS * 32 * ((p.precision ? sizeof(float4) : sizeof(double4)) + sizeof(double));
        if (p.precision)
            k_chain_g<false><<<e->dev_sms * 2, PAIRS_WARPS * 32, sm, s>>>(p, Gsum, e->gctl.p + 3);
        else
            k_chain_g<true><<<e->dev_sms * 2, PAIRS_WARPS * 32, sm, s>>>(p, Gsum, e->gctl.p + 3);
        k_group_reduce<<<gb, T, 0, s>>>(p, 2);
    } else if (p.precision)
        k_chain32<<<gw, T, 0, s>>>(p, Gsum);
    else
        k_chain<<<gw, T, 0, s>>>(p, Gsum);
    D3_CUDA(cudaEventRecord(ev[6], s));
    k_forces_out<<<gb, T, 0, s>>>(p);
    k_reduce<<<p.nstruct, 256, 0, s>>>(p);
    D3_CUDA(cudaEventRecord(ev[7], s));
    e->have_events = true;
    D3_CUDA(cudaGetLastError());
}

int engine_pass_times(Engine *e, float *ms, int cap, unsigned long long *counters) {
    if (!e->have_events) return 0;
    D3_CUDA(cudaEventSynchronize(e->ev[Engine::NEV - 1]));
    int k = 0;
    for (; k < Engine::NEV - 1 && k < cap; ++k) D3_CUDA(cudaEventElapsedTime(&ms[k], e->ev[k], e->ev[k + 1]));
    if (counters) D3_CUDA(cudaMemcpy(counters, e->counters.p, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost));
    return k;
}

int engine_launches_per_eval(const Engine *e) {
    // grouped passes: group cut, three slice reductions and the ATM lists' prefix pass
    const int pairs = pairs_grouped(e) ? (e->use_atm ? 5 : 4) : 0;
    if (!e->use_atm) return 12 + pairs;
    if (e->opt.atm_surrogate && e->surr.loaded) return 20 + pairs;
    return (blockpair_warps(e) > 0 ? 17 : 16) + pairs;
}

// Accuracy check of the Newton-refined helpers used by the ATM kernel against CUDA's
// double-precision 1/sqrt, 1/x and cbrt over log-spaced inputs in [1e-12, 1e14].
__global__ void k_selftest_math(double *err, int m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const double x = exp(log(1e-12) + (log(1e14) - log(1e-12)) * (double)i / (double)(m - 1));
    const double sq = sqrt(x), c = cbrt(x);
    err[6 * i + 0] = fabs(rsqrt_nr(x) * sq - 1.0);
    err[6 * i + 1] = fabs(rcp_nr(x) * x - 1.0);
    err[6 * i + 2] = fabs(rcbrt_nr(x) * c - 1.0);
    err[6 * i + 3] = fabs(rsqrt_nr2(x) * sq - 1.0);
    err[6 * i + 4] = fabs(rcp_nr2(x) * x - 1.0);
    err[6 * i + 5] = fabs(rcbrt_nr2(x) * c - 1.0);
}

// FMA throughput probe: 8 independent FMA chains per thread, enough blocks to fill the
// GPU; the result is written so the chains are not removed. Used to measure the FP64 and
// FP32 pipe peaks the roofline is reported against.
template <typename T>
__global__ void k_fma_probe(T *out, int iters, T a, T b) {
    T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = fma(x0, a, b);
            x1 = fma(x1, a, b);
            x2 = fma(x2, a, b);
            x3 = fma(x3, a, b);
            x4 = fma(x4, a, b);
            x5 = fma(x5, a, b);
            x6 = fma(x6, a, b);
            x7 = fma(x7, a, b);
        }
    }
    const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)-1.2345) out[blockIdx.x] = s;
}

double engine_peak_probe(int fp64) {
    int dev = 0, sms = 148;
    D3_CUDA(cudaGetDevice(&dev));
    D3_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    void *out = nullptr;
    D3_CUDA(cudaMalloc(&out, 8 * 65536));
    cudaEvent_t a, b;
    D3_CUDA(cudaEventCreate(&a));
    D3_CUDA(cudaEventCreate(&b));
    const int blocks = sms * 8, threads = 256, iters = fp64 ? 2048 : 4096;
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        D3_CUDA(cudaEventRecord(a));
        if (fp64)
            k_fma_probe<double><<<blocks, threads>>>((double *)out, iters, 0.999999, 1e-7);
        else
            k_fma_probe<float><<<blocks, threads>>>((float *)out, iters, 0.999999f, 1e-7f);
        D3_CUDA(cudaEventRecord(b));
        D3_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        D3_CUDA(cudaEventElapsedTime(&ms, a, b));
        if (rep > 0) best = std::min(best, ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    const double flops = 2.0 * 8.0 * 16.0 * iters * (double)blocks * threads;
    return flops / (best * 1e-3) / 1e12; // TFLOP/s
}

int engine_selftest_math(double max_rel[6]) {
    const int m = 1 << 16;
    double *d = nullptr;
    D3_CUDA(cudaMalloc(&d, sizeof(double) * 6 * m));
    k_selftest_math<<<(m + 255) / 256, 256>>>(d, m);
    std::vector<double> h(6 * (size_t)m);
    cudaError_t err = cudaMemcpy(h.data(), d, sizeof(double) * 6 * m, cudaMemcpyDeviceToHost);
    cudaFree(d);
    D3_CUDA(err);
    for (int k = 0; k < 6; ++k) max_rel[k] = 0;
    for (int i = 0; i < m; ++i)
        for (int k = 0; k < 6; ++k) max_rel[k] = std::max(max_rel[k], h[6 * (size_t)i + k]);
    return 0;
}

// initial ATM list capacity from each structure's density over the half sphere
static void ensure_atm_capacity(Engine *e) {
    if (!e->use_atm || e->atm_cap != 0) return;
    double cap = 0.0;
    for (int k = 0; k < e->nstruct; ++k) {
        const double nk = (double)e->sg[k].natoms;
        const double rho = nk / std::fabs(e->geoms[k].volume);
        const double k_half = 0.5 * rho * 4.18879020478639 * e->rc_atm * e->rc_atm * e->rc_atm;
        cap += nk * (k_half * 1.25 + 64.0);
    }
    e->atm_cap = (long long)cap + 1024;
    e->atm_ent.ensure((size_t)e->atm_cap);
}

long long engine_atm_capacity(const Engine *e) { return e->use_atm ? e->atm_cap : 0; }

uint16_t engine_fetch_status(Engine *e) {
    unsigned int st = 0;
    D3_CUDA(cudaMemcpy(&st, e->status.p, sizeof(unsigned int), cudaMemcpyDeviceToHost));
    return (uint16_t)st;
}

uint16_t engine_compute(Engine *e, double *energy, double *forces, double *stress, cudaStream_t stream, bool sync) {
    if (!e->cell_set && e->cell_status) return (uint16_t)e->cell_status;
    if (!e->atoms_set || !e->cell_set) return ST_NOT_READY;
    cudaStream_t s = stream ? stream : e->stream;
    try {
        const uint64_t n = e->n;
        ensure_atm_capacity(e);
        for (int attempt = 0; attempt < 4; ++attempt) {
            D3_CUDA(cudaMemsetAsync(e->status.p, 0, sizeof(unsigned int), s));
            KP p = make_kp(e);
            if (e->nref == 5)
                launch_all<5>(e, p, s);
            else
                launch_all<7>(e, p, s);
            if (!sync) return ST_OK;
            unsigned int st = 0;
            D3_CUDA(cudaMemcpyAsync(&st, e->status.p, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
            D3_CUDA(cudaStreamSynchronize(s));
            if ((st & ST_LIST_OVERFLOW) && e->use_atm) {
                long long need = 0;
                D3_CUDA(cudaMemcpy(&need, e->atm_off.p + n, sizeof(long long), cudaMemcpyDeviceToHost));
                e->atm_cap = (long long)(need * 1.1) + 1024;
                e->atm_ent.ensure((size_t)e->atm_cap);
                continue;
            }
            const size_t S = e->nstruct;
            const size_t nout = 10 * S + 3 * n;
            D3_CUDA(cudaMemcpyAsync(e->host_out.data(), e->out.p, sizeof(double) * nout, cudaMemcpyDeviceToHost, s));
            D3_CUDA(cudaStreamSynchronize(s));
            // energies [S], forces [3n], stresses [9S]
            if (energy) memcpy(energy, e->host_out.data(), sizeof(double) * S);
            if (forces) memcpy(forces, e->host_out.data() + S, sizeof(double) * 3 * n);
            if (stress) memcpy(stress, e->host_out.data() + S + 3 * n, sizeof(double) * 9 * S);
            return (uint16_t)st;
        }
        return ST_LIST_OVERFLOW;
    } catch (const std::exception &ex) {
        fprintf(stderr, "d3: %s\n", ex.what());
        return ST_CUDA_ERROR;
    }
}

int engine_debug_atom_arrays(Engine *e, double *cn, double *dedcn, double *energy_atoms) {
    const uint64_t n = e->n;
    std::vector<int> orig(n);
    std::vector<double> a(n), b(n), c(n), d(n), g(n);
    D3_CUDA(cudaStreamSynchronize(e->stream));
    D3_CUDA(cudaMemcpy(orig.data(), e->orig.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    D3_CUDA(cudaMemcpy(a.data(), e->cn.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    D3_CUDA(cudaMemcpy(g.data(), e->G.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    D3_CUDA(cudaMemcpy(b.data(), e->e2.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    D3_CUDA(cudaMemcpy(c.data(), e->ea.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    D3_CUDA(cudaMemcpy(d.data(), e->eb.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    for (uint64_t s = 0; s < n; ++s) {
        const int i = orig[s];
        if (cn) cn[i] = a[s];
        if (dedcn) dedcn[i] = g[s];
        if (energy_atoms) energy_atoms[i] = b[s] + (e->use_atm ? c[s] + d[s] : 0.0);
    }
    return 0;
}

int engine_debug_pass_terms(Engine *e, double *out) {
    // per atom (caller order), D3_DEBUG_TERM_COLUMNS doubles, internal units (hartree,
    // bohr): two-body e, dE/dCN, force[3], virial[6]; ATM apex share e, dE/dCN, force[3],
    // virial[6]; chain-rule force[3], virial[6]; virials as xx yy zz xy xz yz, already
    // scaled by the pass's volume factor
    const uint64_t n = e->n;
    std::vector<int> orig(n);
    D3_CUDA(cudaStreamSynchronize(e->stream));
    D3_CUDA(cudaMemcpy(orig.data(), e->orig.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    struct Col {
        const double *src;
        int width, col;
    };
    const bool atm = e->use_atm;
    const Col cols[] = {{e->e2.p, 1, 0}, {e->g2.p, 1, 1}, {e->f2.p, 3, 2}, {e->v2.p, 6, 5},
                        {atm ? e->ea.p : nullptr, 1, 11}, {atm ? e->ga.p : nullptr, 1, 12},
                        {atm ? e->fa.p : nullptr, 3, 13}, {atm ? e->va.p : nullptr, 6, 16},
                        {e->fc.p, 3, 22}, {e->vc.p, 6, 25}};
    constexpr int W = 31;
    std::vector<double> buf(6 * n);
    for (const Col &c : cols) {
        if (c.src)
            D3_CUDA(cudaMemcpy(buf.data(), c.src, sizeof(double) * c.width * n, cudaMemcpyDeviceToHost));
        for (uint64_t s = 0; s < n; ++s)
            for (int k = 0; k < c.width; ++k) out[(size_t)orig[s] * W + c.col + k] = c.src ? buf[s * c.width + k] : 0.0;
    }
    return 0;
}

int64_t engine_debug_atm_pairs(Engine *e, int64_t *outp, int64_t cap) {
    // returns (apex, j, Tref_x, Tref_y, Tref_z) rows in caller indices and reference shifts
    if (!e->use_atm) return 0;
    const uint64_t n = e->n;
    std::vector<long long> off(n + 1);
    std::vector<int> orig(n);
    std::vector<int4> sh(n);
    D3_CUDA(cudaStreamSynchronize(e->stream));
    D3_CUDA(cudaMemcpy(off.data(), e->atm_off.p, sizeof(long long) * (n + 1), cudaMemcpyDeviceToHost));
    D3_CUDA(cudaMemcpy(orig.data(), e->orig.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    D3_CUDA(cudaMemcpy(sh.data(), e->shift.p, sizeof(int4) * n, cudaMemcpyDeviceToHost));
    const long long tot = off[n];
    std::vector<int2> ent((size_t)tot);
    if (tot) D3_CUDA(cudaMemcpy(ent.data(), e->atm_ent.p, sizeof(int2) * tot, cudaMemcpyDeviceToHost));
    if (!outp) return tot;
    int64_t k = 0;
    for (uint64_t a = 0; a < n && k < cap; ++a)
        for (long long q = off[a]; q < off[a + 1] && k < cap; ++q, ++k) {
            const int j = ent[q].x;
            const int T[3] = {(int)(int8_t)(ent[q].y & 0xff), (int)(int8_t)((ent[q].y >> 8) & 0xff),
                              (int)(int8_t)((ent[q].y >> 16) & 0xff)};
            const int sa[3] = {sh[a].x, sh[a].y, sh[a].z}, sj[3] = {sh[j].x, sh[j].y, sh[j].z};
            int64_t *r = outp + 5 * k;
            r[0] = orig[a];
            r[1] = orig[j];
            // unwrapped: x_a - (x_j + Tref h) equals the wrapped pair vector
            for (int c = 0; c < 3; ++c) r[2 + c] = T[c] + sa[c] - sj[c];
        }
    return k;
}

int engine_debug_bins(Engine *e, int64_t *wrap_shift, int64_t *bin_index, int nb_out[3]) {
    const uint64_t n = e->n;
    std::vector<int4> sh(n);
    std::vector<int> b(n);
    D3_CUDA(cudaStreamSynchronize(e->stream));
    D3_CUDA(cudaMemcpy(sh.data(), e->shift_in.p, sizeof(int4) * n, cudaMemcpyDeviceToHost));
    D3_CUDA(cudaMemcpy(b.data(), e->bin_in.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i < n; ++i) {
        if (wrap_shift) {
            wrap_shift[3 * i] = sh[i].x;
            wrap_shift[3 * i + 1] = sh[i].y;
            wrap_shift[3 * i + 2] = sh[i].z;
        }
        if (bin_index) bin_index[i] = b[i];
    }
    if (nb_out)
        for (int k = 0; k < 3; ++k) nb_out[k] = e->sg.empty() ? 0 : e->sg[0].nb[k];
    return 0;
}

// ------------------------------------------------------------------------------------
// learned ATM surrogate: host side
// ------------------------------------------------------------------------------------
static std::vector<int> channel_map(const Engine *e, const int *channel_z, int nch) {
    std::vector<int> chan(e->ne, -1);
    for (int t = 0; t < e->ne; ++t)
        for (int c = 0; c < nch; ++c)
            if (channel_z[c] == e->elements[t]) chan[t] = c;
    return chan;
}

int engine_set_surrogate(Engine *e, const SurrogateModel &m, std::string &err) {
    try {
        const int nch = (int)m.channel_z.size();
        if (nch < 1 || nch > SURR_MAXCH) {
            err = "surrogate: 1 to " + std::to_string(SURR_MAXCH) + " channels supported";
            return -1;
        }
        const d3mlp::Layout L = d3mlp::make_layout(nch);
        const size_t nfeat = (size_t)nch * SURR_NRBF;
        if (m.members < 1 || m.master.size() != (size_t)m.members * L.nparam || m.mean.size() != nfeat ||
            m.inv_std.size() != nfeat || m.e_shift.size() != (size_t)nch) {
            err = "surrogate: model arrays do not match its channel and member counts";
            return -1;
        }
        const std::vector<int> chan = channel_map(e, m.channel_z.data(), nch);
        for (int t = 0; t < e->ne; ++t)
            if (chan[t] < 0) {
                err = "surrogate: element Z=" + std::to_string(e->elements[t]) + " of the handle is not a model channel";
                return -1;
            }
        SurrState &S = e->surr;
        S.loaded = false;
        S.L = L;
        S.members = m.members;
        S.e_scale = m.e_scale;
        S.chan.ensure(e->ne);
        S.master.ensure(m.master.size());
        S.mean.ensure(nfeat);
        S.inv_std.ensure(nfeat);
        S.e_shift.ensure(nch);
        S.packed.ensure((size_t)m.members * L.packed);
        D3_CUDA(cudaMemcpy(S.chan.p, chan.data(), sizeof(int) * e->ne, cudaMemcpyHostToDevice));
        D3_CUDA(cudaMemcpy(S.master.p, m.master.data(), sizeof(float) * m.master.size(), cudaMemcpyHostToDevice));
        D3_CUDA(cudaMemcpy(S.mean.p, m.mean.data(), sizeof(float) * nfeat, cudaMemcpyHostToDevice));
        D3_CUDA(cudaMemcpy(S.inv_std.p, m.inv_std.data(), sizeof(float) * nfeat, cudaMemcpyHostToDevice));
        D3_CUDA(cudaMemcpy(S.e_shift.p, m.e_shift.data(), sizeof(float) * nch, cudaMemcpyHostToDevice));
        d3mlp::pack(L, m.members, S.master.p, S.packed.p, e->stream);
        const size_t na = std::max<uint64_t>(e->max_atoms, 1);
        S.G.ensure(na * nfeat);
        S.dX.ensure(na * nfeat);
        S.E.ensure(na * m.members);
        S.center.ensure(na);
        S.apex.ensure(na);
        S.flag.ensure(na);
        S.napex.ensure(1);
        D3_CUDA(cudaStreamSynchronize(e->stream));
        S.loaded = true;
        return 0;
    } catch (const std::exception &ex) {
        err = ex.what();
        return -1;
    }
}

void engine_set_surrogate_threshold(Engine *e, double ev) { e->surr.thr_ev = ev; }

int engine_surrogate_flagged(Engine *e) {
    if (!e->surr.loaded) return 0;
    int k = 0;
    D3_CUDA(cudaStreamSynchronize(e->stream));
    D3_CUDA(cudaDeviceSynchronize());
    D3_CUDA(cudaMemcpy(&k, e->surr.napex.p, sizeof(int), cudaMemcpyDeviceToHost));
    return k;
}

int engine_surrogate_descriptors(Engine *e, const int *channel_z, int nch, float *G_dev, int *center_dev,
                                 double *e_atm_dev, cudaStream_t stream, std::string &err) {
    try {
        if (!e->have_events || !e->atoms_set) {
            err = "surrogate descriptors: no evaluation yet";
            return -1;
        }
        if (nch < 1 || nch > SURR_MAXCH) {
            err = "surrogate descriptors: 1 to " + std::to_string(SURR_MAXCH) + " channels supported";
            return -1;
        }
        cudaStream_t s = stream ? stream : e->stream;
        const std::vector<int> chan = channel_map(e, channel_z, nch);
        SurrState &S = e->surr;
        const size_t n = e->n, nfeat = (size_t)nch * SURR_NRBF;
        S.xchan.ensure(e->ne);
        S.xG.ensure(std::max<size_t>(n, 1) * nfeat);
        S.xcenter.ensure(std::max<size_t>(n, 1));
        D3_CUDA(cudaMemcpy(S.xchan.p, chan.data(), sizeof(int) * e->ne, cudaMemcpyHostToDevice));
        if (n == 0) return 0;
        KP p = make_kp(e);
        const SurrDesc sd = surr_desc(S.xchan.p, nch, S.xG.p, nullptr, S.xcenter.p);
        const int T = 256;
        const int gw = (int)(((long long)n * 32 + T - 1) / T);
        if (e->nref == 5)
            k_desc_fwd<5><<<gw, T, 0, s>>>(p, sd);
        else
            k_desc_fwd<7><<<gw, T, 0, s>>>(p, sd);
        k_surr_export<<<gw, T, 0, s>>>(p, S.xG.p, S.xcenter.p, (int)nfeat, G_dev, center_dev, e_atm_dev);
        D3_CUDA(cudaGetLastError());
        D3_CUDA(cudaStreamSynchronize(s));
        return 0;
    } catch (const std::exception &ex) {
        err = ex.what();
        return -1;
    }
}

// ------------------------------------------------------------------------------------
// sharded evaluation of one structure over several processes
// ------------------------------------------------------------------------------------
uint16_t engine_shard_begin(Engine *e, int rank, int world, double *G_out, cudaStream_t stream, std::string &err) {
    if (!e->atoms_set || !e->cell_set) return ST_NOT_READY;
    if (world < 1 || rank < 0 || rank >= world || !G_out) {
        err = "shard: rank must be in [0, world) and the dE/dCN buffer given";
        return ST_BAD_INPUT;
    }
    if (e->opt.atm_surrogate && e->surr.loaded) {
        err = "shard: the learned surrogate is not available in a sharded evaluation";
        return ST_BAD_INPUT;
    }
    cudaStream_t s = stream ? stream : e->stream;
    try {
        ensure_atm_capacity(e);
        for (int attempt = 0; attempt < 4; ++attempt) {
            D3_CUDA(cudaMemsetAsync(e->status.p, 0, sizeof(unsigned int), s));
            KP p = make_kp(e);
            p.shard_rank = rank;
            p.shard_world = world;
            if (e->nref == 5)
                launch_all<5>(e, p, s, 1, G_out);
            else
                launch_all<7>(e, p, s, 1, G_out);
            unsigned int st = 0;
            D3_CUDA(cudaMemcpyAsync(&st, e->status.p, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
            D3_CUDA(cudaStreamSynchronize(s));
            if ((st & ST_LIST_OVERFLOW) && e->use_atm) {
                long long need = 0;
                D3_CUDA(cudaMemcpy(&need, e->atm_off.p + e->n, sizeof(long long), cudaMemcpyDeviceToHost));
                e->atm_cap = (long long)(need * 1.1) + 1024;
                e->atm_ent.ensure((size_t)e->atm_cap);
                continue;
            }
            e->shard_rank = rank;
            e->shard_world = world;
            return (uint16_t)st;
        }
        return ST_LIST_OVERFLOW;
    } catch (const std::exception &ex) {
        err = ex.what();
        return ST_CUDA_ERROR;
    }
}

uint16_t engine_shard_end(Engine *e, const double *G_in, double *out_dev, cudaStream_t stream, std::string &err) {
    if (e->shard_world < 1 || !G_in || !out_dev) {
        err = "shard: d3_shard_begin first, and give the dE/dCN and result buffers";
        return ST_NOT_READY;
    }
    cudaStream_t s = stream ? stream : e->stream;
    try {
        KP p = make_kp(e);
        p.shard_rank = e->shard_rank;
        p.shard_world = e->shard_world;
        if (e->nref == 5)
            launch_all<5>(e, p, s, 2, const_cast<double *>(G_in));
        else
            launch_all<7>(e, p, s, 2, const_cast<double *>(G_in));
        const size_t nout = 10 * (size_t)e->nstruct + 3 * (size_t)e->n;
        D3_CUDA(cudaMemcpyAsync(out_dev, e->out.p, sizeof(double) * nout, cudaMemcpyDeviceToDevice, s));
        return ST_OK;
    } catch (const std::exception &ex) {
        err = ex.what();
        return ST_CUDA_ERROR;
    }
}

} // namespace d3

// Descriptors of the learned ATM surrogate and their backward pass.
// Included by d3_engine.cu after the kernel parameter block and the traversal helper.
//
// For atom i, neighbour-element channel c and radial function k (32 per channel):
//     G_i[c][k] = sum_{j,T: 0 < r_ij <= rc_ATM, chan(j) = c} C6_ij psi_k(r_ij)
//     psi_k(r) = exp(-(r - mu_k)^2 / (2 sigma^2)) fc(r),  fc(r) = (1 + cos(pi r / rc)) / 2
// with mu_k uniform in [0.8, 21] A and sigma = 0.7 A (in bohr here), C6_ij the exact
// CN-dependent coefficient of the pair. The smooth cutoff keeps energies continuous.
//
// Backward, given dE/dG for every atom (E = sum_i E_i(G_i), E in the engine's stored sign):
//     a_ij = C6_ij sum_k dE_i/dG_i[c_j][k] psi_k'(r),   b_ij = sum_k dE_i/dG_i[c_j][k] psi_k(r)
//     force (gradient) on i:  sum_j (a_ij + a_ji) (x_i - x_j) / r_ij
//     dE/dCN_i:               sum_j (b_ij + b_ji) dC6_ij/dCN_i
//     virial:                 -(x_i - x_j) (x) (x_i - x_j) (a_ij + a_ji) / (2 V r) per ordered pair
// Forward: one warp per atom, one lane per radial function; backward: one lane per
// neighbour. Neighbours come from the rc_ATM stencil. The cutoff function is evaluated in
// FP32 (sincospif) in both passes.

constexpr int SURR_NRBF = 32;
constexpr int SURR_MAXCH = 8;

struct SurrDesc {
    const int *chan;   // channel of each handle type (-1: not covered)
    int nch;
    float mu0, dmu;    // bohr
    float inv2s2;      // 1 / (2 sigma^2), bohr^-2
    float *G;          // [n][nch][32], binned order
    const float *dEdG; // [n][nch][32], binned order (backward input)
    int *center;       // [n] channel of each atom (binned order), -1: not a channel
};

// smooth cutoff fc(r) = (1 + cos(pi r / rc)) / 2 and its derivative, FP32 (the same
// values in the forward and the backward pass)
__device__ __forceinline__ void surr_cutoff(float r, float inv_rc, float &fc, float &dfc) {
    float sn, cs;
    sincospif(r * inv_rc, &sn, &cs);
    fc = 0.5f * (1.0f + cs);
    dfc = -0.5f * 3.14159265358979f * inv_rc * sn;
}

// Forward: lane k of the atom's warp owns radial function k of every channel, in
// registers. Each stencil chunk's in-range neighbours are broadcast channel by channel
// (one ballot per channel), so each channel's sum is a register of a compile-time index.
template <int NR>
__global__ void k_desc_fwd(KP p, SurrDesc sd) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= p.n) return;
    const SG &g = p.sg[p.sid[i]];
    const double4 xi = p.xs[i];
    const int4 si = p.shift[i];
    const int ti = (int)xi.w;
    if (lane == 0) sd.center[i] = sd.chan[ti];
    double wi[NR];
#pragma unroll
    for (int a = 0; a < NR; ++a) wi[a] = p.w[(size_t)i * NR + a];
    const float mu_k = sd.mu0 + sd.dmu * lane;
    const float inv_rc = (float)(1.0 / sqrt(p.ratm2));
    const int nch = sd.nch;
    float acc[SURR_MAXCH];
#pragma unroll
    for (int c = 0; c < SURR_MAXCH; ++c) acc[c] = 0.0f;
    traverse(p, g, p.bin_s[i], p.stencils + g.sta_off, g.sta_n,
             [&](int j, int Tx, int Ty, int Tz, const double3 &sh, bool act) {
                 float r = 0.f, wgt = 0.f;
                 int ch = -1;
                 if (act && in_box(g, si, p.shift[j], Tx, Ty, Tz)) {
                     const double4 xj = p.xs[j];
                     const double dx = xi.x - (xj.x + sh.x), dy = xi.y - (xj.y + sh.y), dz = xi.z - (xj.z + sh.z);
                     const double d2 = dx * dx + dy * dy + dz * dz;
                     const int cj = sd.chan[(int)xj.w];
                     if (d2 <= p.ratm2 && d2 > 0.0 && cj >= 0) {
                         const double *yj = p.Y + ((size_t)j * p.ne + ti) * NR;
                         double c6 = 0.0;
#pragma unroll
                         for (int b = 0; b < NR; ++b) c6 += yj[b] * wi[b];
                         r = (float)sqrt(d2);
                         float fc, dfc;
                         surr_cutoff(r, inv_rc, fc, dfc);
                         wgt = (float)c6 * fc;
                         ch = cj;
                     }
                 }
#pragma unroll
                 for (int c = 0; c < SURR_MAXCH; ++c) {
                     if (c >= nch) break;
                     unsigned m = __ballot_sync(0xffffffffu, ch == c);
                     while (m) {
                         const int b = __ffs(m) - 1;
                         m &= m - 1u;
                         const float rb = __shfl_sync(0xffffffffu, r, b);
                         const float wb = __shfl_sync(0xffffffffu, wgt, b);
                         const float d = rb - mu_k;
                         acc[c] = fmaf(wb, __expf(-d * d * sd.inv2s2), acc[c]);
                     }
                 }
             });
    float *out = sd.G + (size_t)i * nch * SURR_NRBF;
#pragma unroll
    for (int c = 0; c < SURR_MAXCH; ++c)
        if (c < nch) out[c * SURR_NRBF + lane] = acc[c];
}

// Backward, one warp per atom and one neighbour per lane. With phi_k = exp(-(r - mu_k)^2
// / (2 sigma^2)), psi_k = phi_k fc and g_k = dE/dG_i[c_j][k] + dE/dG_j[c_i][k]:
//     sum_k g_k psi_k  = fc S0,   sum_k g_k psi_k' = dfc S0 - 2 fc S1 / (2 sigma^2)
//     S0 = sum_k g_k phi_k,       S1 = sum_k g_k phi_k (r - mu_k)
// so each neighbour costs 32 exponentials and two FMAs per radial function; the atom's own
// dE/dG rows sit in shared memory (rows padded to 33 floats: lanes reading different
// channels at the same k hit different banks), the neighbour's row is read as 8 float4.
// In-range neighbours are first compacted into a per-warp queue, so that the radial loop
// always runs with 32 busy lanes.
struct SurrNb {
    int j, ch;
    float r, c6, dc6, dx, dy, dz;
};

template <int NR>
__global__ void __launch_bounds__(256, 2) k_desc_bwd(KP p, SurrDesc sd) {
    constexpr int PITCH = SURR_NRBF + 1;
    __shared__ float Ds[8][SURR_MAXCH * PITCH];
    __shared__ SurrNb Q[8][64];
    const int warp_in_block = threadIdx.x >> 5;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= p.n) return;
    const SG &g = p.sg[p.sid[i]];
    float *Dw = Ds[warp_in_block];
    SurrNb *q = Q[warp_in_block];
    const float *din = sd.dEdG + (size_t)i * sd.nch * SURR_NRBF;
    for (int c = 0; c < sd.nch; ++c) Dw[c * PITCH + lane] = din[c * SURR_NRBF + lane];
    __syncwarp();
    const double4 xi = p.xs[i];
    const int4 si = p.shift[i];
    const int ti = (int)xi.w;
    const int chi = sd.chan[ti];
    double wi[NR], dwi[NR];
#pragma unroll
    for (int a = 0; a < NR; ++a) {
        wi[a] = p.w[(size_t)i * NR + a];
        dwi[a] = p.dw[(size_t)i * NR + a];
    }
    const float inv_rc = (float)(1.0 / sqrt(p.ratm2));
    const float a2 = sd.inv2s2;
    double fx = 0, fy = 0, fz = 0, gcn = 0, vxx = 0, vyy = 0, vzz = 0, vxy = 0, vxz = 0, vyz = 0;
    // one queued neighbour per lane: the radial sums and their contributions
    auto process = [&](bool valid) {
        if (!valid) return;
        const SurrNb nb = q[lane];
        float fc, dfc;
        surr_cutoff(nb.r, inv_rc, fc, dfc);
        const float4 *gj = reinterpret_cast<const float4 *>(sd.dEdG + ((size_t)nb.j * sd.nch + chi) * SURR_NRBF);
        const float *gi = Dw + nb.ch * PITCH;
        float s0 = 0.f, s1 = 0.f;
#pragma unroll
        for (int qd = 0; qd < SURR_NRBF / 4; ++qd) {
            const float4 v = __ldg(gj + qd);
            const float gv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int k = 4 * qd + t;
                const float u = nb.r - (sd.mu0 + sd.dmu * k);
                const float w = (gv[t] + gi[k]) * __expf(-u * u * a2);
                s0 += w;
                s1 = fmaf(w, u, s1);
            }
        }
        // dE/dr / r and dE/dC6_ij
        const double fs = (double)nb.c6 * ((double)dfc * s0 - 2.0 * (double)a2 * (double)fc * s1) / (double)nb.r;
        const double dx = nb.dx, dy = nb.dy, dz = nb.dz;
        fx += fs * dx;
        fy += fs * dy;
        fz += fs * dz;
        vxx += fs * dx * dx;
        vyy += fs * dy * dy;
        vzz += fs * dz * dz;
        vxy += fs * dx * dy;
        vxz += fs * dx * dz;
        vyz += fs * dy * dz;
        gcn += (double)(fc * s0) * (double)nb.dc6; // dE/dC6_ij dC6_ij/dCN_i
    };
    int count = 0; // queued neighbours (warp-uniform)
    traverse(p, g, p.bin_s[i], p.stencils + g.sta_off, g.sta_n,
             [&](int j, int Tx, int Ty, int Tz, const double3 &sh, bool act) {
                 bool keep = false;
                 SurrNb nb;
                 if (act && chi >= 0 && in_box(g, si, p.shift[j], Tx, Ty, Tz)) {
                     const double4 xj = p.xs[j];
                     const double dx = xi.x - (xj.x + sh.x), dy = xi.y - (xj.y + sh.y), dz = xi.z - (xj.z + sh.z);
                     const double d2 = dx * dx + dy * dy + dz * dz;
                     const int ch = sd.chan[(int)xj.w];
                     if (d2 <= p.ratm2 && d2 > 0.0 && ch >= 0) {
                         const double *yj = p.Y + ((size_t)j * p.ne + ti) * NR;
                         double c6 = 0.0, dc6 = 0.0;
#pragma unroll
                         for (int b = 0; b < NR; ++b) {
                             c6 += yj[b] * wi[b];
                             dc6 += yj[b] * dwi[b]; // dC6_ij/dCN_i
                         }
                         nb = SurrNb{j, ch, (float)sqrt(d2), (float)c6, (float)dc6, (float)dx, (float)dy, (float)dz};
                         keep = true;
                     }
                 }
                 const unsigned m = __ballot_sync(0xffffffffu, keep);
                 if (keep) q[count + __popc(m & ((1u << lane) - 1u))] = nb;
                 count += __popc(m);
                 if (count >= 32) {
                     __syncwarp();
                     process(true);
                     __syncwarp();
                     if (lane < count - 32) q[lane] = q[32 + lane];
                     count -= 32;
                     __syncwarp();
                 }
             });
    __syncwarp();
    process(lane < count);
    fx = warp_sum(fx);
    fy = warp_sum(fy);
    fz = warp_sum(fz);
    gcn = warp_sum(gcn);
    vxx = warp_sum(vxx);
    vyy = warp_sum(vyy);
    vzz = warp_sum(vzz);
    vxy = warp_sum(vxy);
    vxz = warp_sum(vxz);
    vyz = warp_sum(vyz);
    if (lane == 0) {
        // the surrogate's share enters through the ATM apex arrays (entry arrays stay zero
        // for atoms the surrogate covers)
        p.fa[3 * i] += fx;
        p.fa[3 * i + 1] += fy;
        p.fa[3 * i + 2] += fz;
        p.ga[i] += gcn;
        const double sc = -1.0 / (2.0 * g.vol);
        double *v = p.va + 6 * (size_t)i;
        v[0] += vxx * sc;
        v[1] += vyy * sc;
        v[2] += vzz * sc;
        v[3] += vxy * sc;
        v[4] += vxz * sc;
        v[5] += vyz * sc;
    }
}

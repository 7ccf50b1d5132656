// Per-atom MLP of the learned ATM surrogate (layout and API in d3_mlp.h).
//
// Fused kernel k_mlp: one CTA of 8 warps per 128-row tile, each warp owns 16 rows end to
// end. The member's BF16 weights sit in shared memory (transposed, padded rows); the
// warp's input rows are normalised into shared memory and fed to mma.m16n8k16 through
// ldmatrix. Hidden activations never leave registers: the FP32 accumulator fragment of
// one layer is re-packed as the BF16 A fragment of the next (the m16n8 C layout of two
// adjacent n-tiles is the m16k16 A layout). SiLU derivatives are kept as FP16 pairs in
// the same fragment layout (layers 1 and 2 in the warp's shared scratch, which held the
// input rows until layer 1 consumed them; layer 3 in registers) for the backward pass,
// which runs the transposed GEMMs with ldmatrix.trans on the same weight tiles:
//     dZ3 = g w4 * silu'(Z3),  dH2 = dZ3 W3^T,  dZ2 = dH2 * silu'(Z2), ...,  dX = dZ1 W1^T
// with g = 1 at inference (dE/dX) and g = dLoss/dE when training.
//
// Training adds k_wgrad (dW = H^T dZ per 128-row split, mma with ldmatrix.trans on both
// operands; partial sums per split so that the reduction order is fixed) and k_adam.
#include "d3_mlp.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <stdexcept>
#include <string>

namespace d3mlp {

constexpr int P2 = HID + 8; // padded row of W2t / W3t (272 B: 68 words, 4 mod 32)

Layout make_layout(int nch) {
    if (nch < 1 || nch > MAXCH) throw std::invalid_argument("surrogate: channel count out of range");
    Layout L;
    L.nch = nch;
    L.in_dim = nch * NRBF + nch;
    L.in_pad = (L.in_dim + 15) / 16 * 16;
    L.p1 = L.in_pad + 8; // (in_pad/2 + 4) words: 4 mod 8 words -> conflict-free ldmatrix rows
    size_t o = 0;
    L.oW1 = o;
    o += (size_t)L.in_pad * HID;
    L.ob1 = o;
    o += HID;
    L.oW2 = o;
    o += (size_t)HID * HID;
    L.ob2 = o;
    o += HID;
    L.oW3 = o;
    o += (size_t)HID * HID;
    L.ob3 = o;
    o += HID;
    L.ow4 = o;
    o += HID;
    L.ob4 = o;
    o += 1;
    L.nparam = (o + 3) / 4 * 4;
    L.packed = (size_t)HID * L.p1 + 2 * (size_t)HID * P2;
    return L;
}

// per-warp scratch: the 16 staged input rows during layer 1, then the SiLU derivatives
// of layers 1 and 2 (FP16 pairs, 4 KB each, word-major so that lanes hit distinct banks)
static size_t warp_scratch(const Layout &L) { return std::max<size_t>((size_t)16 * L.p1 * 2, 8192); }

size_t smem_bytes(const Layout &L) {
    return L.packed * 2 + (4 * HID + 4) * sizeof(float) + (size_t)(THREADS / 32) * warp_scratch(L);
}

size_t acts_elems(const Layout &L, int B) { return (size_t)B * (L.in_pad + 5 * HID); }

// ------------------------------------------------------------------------------------
// warp-level MMA helpers
// ------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm4(uint32_t (&r)[4], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}

__device__ __forceinline__ void ldsm4t(uint32_t (&r)[4], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}

__device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ float2 unpack_bf16(uint32_t u) {
    __nv_bfloat162 v = *reinterpret_cast<__nv_bfloat162 *>(&u);
    return __bfloat1622float2(v);
}

// bias-initialised accumulators: columns nt*8 + 2 tig (+1), rows g and g + 8
__device__ __forceinline__ void init_acc(float (&acc)[16][4], const float *bias, int tig) {
#pragma unroll
    for (int nt = 0; nt < 16; ++nt) {
        const float2 b = bias ? *reinterpret_cast<const float2 *>(bias + nt * 8 + 2 * tig) : make_float2(0.f, 0.f);
        acc[nt][0] = b.x;
        acc[nt][1] = b.y;
        acc[nt][2] = b.x;
        acc[nt][3] = b.y;
    }
}

// acc += A (16 x 16*ksteps, fragments) * Wt^T, Wt rows = outputs (pitch `pitch`)
__device__ __forceinline__ void gemm_fwd_regA(float (&acc)[16][4], const uint32_t (&A)[8][4], const __nv_bfloat16 *wt,
                                              int pitch, int lane) {
    const int brow = (lane & 7) + ((lane >> 4) & 1) * 8, bcol = ((lane >> 3) & 1) * 8;
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
#pragma unroll
        for (int np = 0; np < 8; ++np) {
            uint32_t b[4];
            ldsm4(b, wt + (np * 16 + brow) * pitch + kk * 16 + bcol);
            mma(acc[2 * np], A[kk], b[0], b[1]);
            mma(acc[2 * np + 1], A[kk], b[2], b[3]);
        }
    }
}

// acc (16 x 128) += dA (16 x 128, fragments) * W^T where Wt (rows = the 128 outputs of the
// forward layer, pitch `pitch`) is read transposed: column block np*16 of the result
__device__ __forceinline__ void gemm_bwd_pair(float (&acc)[2][4], const uint32_t (&dA)[8][4], const __nv_bfloat16 *wt,
                                              int pitch, int np, int lane) {
    const int trow = (lane & 7) + ((lane >> 3) & 1) * 8, tcol = ((lane >> 4) & 1) * 8;
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
        uint32_t b[4];
        ldsm4t(b, wt + (kk * 16 + trow) * pitch + np * 16 + tcol);
        mma(acc[0], dA[kk], b[0], b[1]);
        mma(acc[1], dA[kk], b[2], b[3]);
    }
}

__device__ __forceinline__ void gemm_bwd_full(float (&acc)[16][4], const uint32_t (&dA)[8][4], const __nv_bfloat16 *wt,
                                              int pitch, int lane) {
#pragma unroll
    for (int nt = 0; nt < 16; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
    const int trow = (lane & 7) + ((lane >> 3) & 1) * 8, tcol = ((lane >> 4) & 1) * 8;
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
#pragma unroll
        for (int np = 0; np < 8; ++np) {
            uint32_t b[4];
            ldsm4t(b, wt + (kk * 16 + trow) * pitch + np * 16 + tcol);
            mma(acc[2 * np], dA[kk], b[0], b[1]);
            mma(acc[2 * np + 1], dA[kk], b[2], b[3]);
        }
    }
}

__device__ __forceinline__ void silu(float z, float &h, float &d) {
    const float s = __fdividef(1.0f, 1.0f + __expf(-z));
    h = z * s;
    d = s * fmaf(z, 1.0f - s, 1.0f);
}

// SiLU of the accumulators: BF16 A fragments of the activations; FP16 derivative pairs
// to the warp's shared scratch (word k of lane l at D[k*32 + l])
__device__ __forceinline__ void activate(const float (&acc)[16][4], uint32_t (&H)[8][4], __half2 *D, int lane) {
#pragma unroll
    for (int nt = 0; nt < 16; ++nt) {
        float h0, h1, h2, h3, d0, d1, d2, d3;
        silu(acc[nt][0], h0, d0);
        silu(acc[nt][1], h1, d1);
        silu(acc[nt][2], h2, d2);
        silu(acc[nt][3], h3, d3);
        H[nt >> 1][(nt & 1) * 2] = pack_bf16(h0, h1);
        H[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16(h2, h3);
        D[(2 * nt) * 32 + lane] = __floats2half2_rn(d0, d1);
        D[(2 * nt + 1) * 32 + lane] = __floats2half2_rn(d2, d3);
    }
}

// dZ = acc * silu'(Z) as BF16 A fragments
__device__ __forceinline__ void grad_frag(const float (&acc)[16][4], const __half2 *D, int lane, uint32_t (&dA)[8][4]) {
#pragma unroll
    for (int nt = 0; nt < 16; ++nt) {
        const float2 d01 = __half22float2(D[(2 * nt) * 32 + lane]), d23 = __half22float2(D[(2 * nt + 1) * 32 + lane]);
        dA[nt >> 1][(nt & 1) * 2] = pack_bf16(acc[nt][0] * d01.x, acc[nt][1] * d01.y);
        dA[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16(acc[nt][2] * d23.x, acc[nt][3] * d23.y);
    }
}

// store A fragments (16 rows x 128) to a row-major [row][128] BF16 array
__device__ __forceinline__ void store_frag(uint16_t *dst, const uint32_t (&F)[8][4], int g, int tig) {
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
        uint32_t *r0 = reinterpret_cast<uint32_t *>(dst + (size_t)g * HID + kk * 16 + 2 * tig);
        uint32_t *r8 = reinterpret_cast<uint32_t *>(dst + (size_t)(g + 8) * HID + kk * 16 + 2 * tig);
        r0[0] = F[kk][0];
        r8[0] = F[kk][1];
        r0[4] = F[kk][2];
        r8[4] = F[kk][3];
    }
}

struct KArgs {
    int nch, in_pad, p1;
    size_t scratch; // bytes of shared scratch per warp
    size_t ob1, ob2, ob3, ow4, ob4, nparam, packed;
    int members;
    const float *master;
    const uint16_t *wpacked;
    const float *mean, *inv_std;
    const float *G;
    const int *center;
    int rows;
    float *E;
    float *dX;
    // training
    const float *target;
    const int *idx;
    uint16_t *acts;
    float *partial;
    float *loss;
    int splits;
};

template <bool TRAIN>
__global__ void __launch_bounds__(THREADS, 1) k_mlp(KArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ float red[THREADS / 32][HID + 2];
    const int p1 = a.p1, in_pad = a.in_pad, nfeat = a.nch * NRBF;
    __nv_bfloat16 *w1t = reinterpret_cast<__nv_bfloat16 *>(smem);
    __nv_bfloat16 *w2t = w1t + HID * p1;
    __nv_bfloat16 *w3t = w2t + HID * P2;
    float *vb1 = reinterpret_cast<float *>(w3t + HID * P2);
    float *vb2 = vb1 + HID, *vb3 = vb2 + HID, *vw4 = vb3 + HID; // vw4[HID] = b4
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3;
    unsigned char *scratch = reinterpret_cast<unsigned char *>(vw4 + HID + 4) + (size_t)warp * a.scratch;
    __nv_bfloat16 *xw = reinterpret_cast<__nv_bfloat16 *>(scratch); // layer-1 input rows
    __half2 *dsm1 = reinterpret_cast<__half2 *>(scratch);             // silu'(Z1), after layer 1
    __half2 *dsm2 = dsm1 + 32 * 32;                                    // silu'(Z2)
    const int nrows = a.rows;
    const int ntiles = (nrows + TILE - 1) / TILE;
    const int m_lo = TRAIN ? (int)blockIdx.y : 0, m_hi = TRAIN ? (int)blockIdx.y + 1 : a.members;
    const size_t act_stride = (size_t)nrows * (in_pad + 5 * HID);
    for (int m = m_lo; m < m_hi; ++m) {
        __syncthreads();
        {
            const uint4 *src = reinterpret_cast<const uint4 *>(a.wpacked + (size_t)m * a.packed);
            uint4 *dst = reinterpret_cast<uint4 *>(smem);
            const int nvec = (int)(a.packed * 2 / 16);
            for (int k = tid; k < nvec; k += THREADS) dst[k] = src[k];
            const float *mp = a.master + (size_t)m * a.nparam;
            for (int k = tid; k < HID; k += THREADS) {
                vb1[k] = mp[a.ob1 + k];
                vb2[k] = mp[a.ob2 + k];
                vb3[k] = mp[a.ob3 + k];
                vw4[k] = mp[a.ow4 + k];
            }
            if (tid == 0) vw4[HID] = mp[a.ob4];
        }
        __syncthreads();
        const float b4 = vw4[HID];
        const int t_lo = blockIdx.x, t_step = TRAIN ? ntiles : gridDim.x;
        for (int tile = t_lo; tile < ntiles; tile += t_step) {
            const int r0 = tile * TILE + warp * 16;
            // ---- stage the warp's 16 input rows (normalised descriptor + one-hot channel)
            for (int lr = 0; lr < 16; ++lr) {
                const int r = r0 + lr;
                const bool valid = r < nrows;
                const int src = valid ? (TRAIN ? a.idx[(size_t)m * nrows + r] : r) : 0;
                const float *gr = a.G + (size_t)src * nfeat;
                const int cen = valid ? a.center[src] : -1;
                __nv_bfloat16 *xr = xw + lr * p1;
                for (int c = 2 * lane; c < in_pad; c += 64) {
                    float v0 = 0.f, v1 = 0.f;
                    if (valid) {
                        if (c < nfeat) {
                            const float2 gv = *reinterpret_cast<const float2 *>(gr + c);
                            v0 = (gv.x - a.mean[c]) * a.inv_std[c];
                            v1 = (gv.y - a.mean[c + 1]) * a.inv_std[c + 1];
                        } else {
                            v0 = (c - nfeat == cen) ? 1.f : 0.f;
                            v1 = (c + 1 - nfeat == cen) ? 1.f : 0.f;
                        }
                    }
                    *reinterpret_cast<__nv_bfloat162 *>(xr + c) = __floats2bfloat162_rn(v0, v1);
                }
            }
            __syncwarp();
            uint16_t *actm = TRAIN ? a.acts + (size_t)m * act_stride : nullptr;
            if (TRAIN) {
                // X rows for the weight gradient of layer 1
                const int vpr = in_pad / 8;
                for (int v = lane; v < 16 * vpr; v += 32) {
                    const int lr = v / vpr, c = (v % vpr) * 8;
                    *reinterpret_cast<uint4 *>(actm + (size_t)(r0 + lr) * in_pad + c) =
                        *reinterpret_cast<const uint4 *>(xw + lr * p1 + c);
                }
            }
            // ---- layer 1: Z1 = X W1 + b1
            float acc[16][4];
            init_acc(acc, vb1, tig);
            {
                const int arow = (lane & 7) + ((lane >> 3) & 1) * 8, acol = ((lane >> 4) & 1) * 8;
                const int brow = (lane & 7) + ((lane >> 4) & 1) * 8, bcol = ((lane >> 3) & 1) * 8;
                for (int ks = 0; ks < in_pad / 16; ++ks) {
                    uint32_t af[4];
                    ldsm4(af, xw + arow * p1 + ks * 16 + acol);
#pragma unroll
                    for (int np = 0; np < 8; ++np) {
                        uint32_t b[4];
                        ldsm4(b, w1t + (np * 16 + brow) * p1 + ks * 16 + bcol);
                        mma(acc[2 * np], af, b[0], b[1]);
                        mma(acc[2 * np + 1], af, b[2], b[3]);
                    }
                }
            }
            uint32_t H[8][4];
            __half2 D3[16][2];
            __syncwarp(); // every lane is done reading the input rows the derivatives overwrite
            activate(acc, H, dsm1, lane);
            if (TRAIN) store_frag(actm + (size_t)nrows * in_pad + (size_t)r0 * HID, H, g, tig);
            // ---- layer 2
            init_acc(acc, vb2, tig);
            gemm_fwd_regA(acc, H, w2t, P2, lane);
            activate(acc, H, dsm2, lane);
            if (TRAIN) store_frag(actm + (size_t)nrows * (in_pad + HID) + (size_t)r0 * HID, H, g, tig);
            // ---- layer 3 and the output projection (FP32 activations)
            init_acc(acc, vb3, tig);
            gemm_fwd_regA(acc, H, w3t, P2, lane);
            float eg = 0.f, eg8 = 0.f;
#pragma unroll
            for (int nt = 0; nt < 16; ++nt) {
                const float2 w = *reinterpret_cast<const float2 *>(vw4 + nt * 8 + 2 * tig);
                float h0, h1, h2, h3, d0, d1, d2, d3;
                silu(acc[nt][0], h0, d0);
                silu(acc[nt][1], h1, d1);
                silu(acc[nt][2], h2, d2);
                silu(acc[nt][3], h3, d3);
                eg = fmaf(h0, w.x, fmaf(h1, w.y, eg));
                eg8 = fmaf(h2, w.x, fmaf(h3, w.y, eg8));
                D3[nt][0] = __floats2half2_rn(d0, d1);
                D3[nt][1] = __floats2half2_rn(d2, d3);
                if (TRAIN) {
                    H[nt >> 1][(nt & 1) * 2] = pack_bf16(h0, h1);
                    H[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16(h2, h3);
                }
            }
            eg += __shfl_xor_sync(0xffffffffu, eg, 1);
            eg += __shfl_xor_sync(0xffffffffu, eg, 2);
            eg8 += __shfl_xor_sync(0xffffffffu, eg8, 1);
            eg8 += __shfl_xor_sync(0xffffffffu, eg8, 2);
            const float Eg = eg + b4, Eg8 = eg8 + b4;
            const int rg = r0 + g, rg8 = r0 + g + 8;
            float sg = 1.f, sg8 = 1.f; // dOut/dE of rows g, g + 8
            if (TRAIN) {
                const float inv_b = 1.0f / (float)nrows;
                const int sr = a.idx[(size_t)m * nrows + rg], sr8 = a.idx[(size_t)m * nrows + rg8];
                const float e0 = Eg - a.target[sr], e8 = Eg8 - a.target[sr8];
                sg = 2.f * e0 * inv_b;
                sg8 = 2.f * e8 * inv_b;
                if (tig == 0) {
                    a.E[(size_t)m * nrows + rg] = Eg;
                    a.E[(size_t)m * nrows + rg8] = Eg8;
                }
                // w4 / b4 gradient and loss of the tile
                float l = (tig == 0) ? e0 * e0 + e8 * e8 : 0.f;
                float db = (tig == 0) ? sg + sg8 : 0.f;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    l += __shfl_xor_sync(0xffffffffu, l, o);
                    db += __shfl_xor_sync(0xffffffffu, db, o);
                }
#pragma unroll
                for (int nt = 0; nt < 16; ++nt) {
                    const float2 h01 = unpack_bf16(H[nt >> 1][(nt & 1) * 2]);
                    const float2 h23 = unpack_bf16(H[nt >> 1][(nt & 1) * 2 + 1]);
                    float s0 = sg * h01.x + sg8 * h23.x, s1 = sg * h01.y + sg8 * h23.y;
#pragma unroll
                    for (int o = 4; o < 32; o <<= 1) {
                        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
                        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                    }
                    if (g == 0) {
                        red[warp][nt * 8 + 2 * tig] = s0;
                        red[warp][nt * 8 + 2 * tig + 1] = s1;
                    }
                }
                if (lane == 0) {
                    red[warp][HID] = db;
                    red[warp][HID + 1] = l;
                }
            } else if (tig == 0) {
                if (rg < nrows) a.E[(size_t)m * nrows + rg] = Eg;
                if (rg8 < nrows) a.E[(size_t)m * nrows + rg8] = Eg8;
            }
            if (TRAIN || a.dX) {
                // ---- backward: dZ3 = s w4 silu'(Z3)
                uint32_t dA[8][4];
#pragma unroll
                for (int nt = 0; nt < 16; ++nt) {
                    const float2 w = *reinterpret_cast<const float2 *>(vw4 + nt * 8 + 2 * tig);
                    const float2 d01 = __half22float2(D3[nt][0]), d23 = __half22float2(D3[nt][1]);
                    dA[nt >> 1][(nt & 1) * 2] = pack_bf16(sg * w.x * d01.x, sg * w.y * d01.y);
                    dA[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16(sg8 * w.x * d23.x, sg8 * w.y * d23.y);
                }
                if (TRAIN) store_frag(actm + (size_t)nrows * (in_pad + 4 * HID) + (size_t)r0 * HID, dA, g, tig);
                gemm_bwd_full(acc, dA, w3t, P2, lane); // dH2
                grad_frag(acc, dsm2, lane, dA);        // dZ2
                if (TRAIN) store_frag(actm + (size_t)nrows * (in_pad + 3 * HID) + (size_t)r0 * HID, dA, g, tig);
                gemm_bwd_full(acc, dA, w2t, P2, lane); // dH1
                grad_frag(acc, dsm1, lane, dA);        // dZ1
                if (TRAIN) store_frag(actm + (size_t)nrows * (in_pad + 2 * HID) + (size_t)r0 * HID, dA, g, tig);
                if (!TRAIN) {
                    // dX = dZ1 W1^T over the descriptor columns, times inv_std; summed over
                    // members (same CTA, members in order: deterministic)
                    for (int np = 0; np < nfeat / 16; ++np) {
                        float acc2[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
                        gemm_bwd_pair(acc2, dA, w1t, p1, np, lane);
#pragma unroll
                        for (int j = 0; j < 2; ++j) {
                            const int c = np * 16 + j * 8 + 2 * tig;
                            const float i0 = a.inv_std[c], i1 = a.inv_std[c + 1];
                            if (rg < nrows) {
                                float2 *o = reinterpret_cast<float2 *>(a.dX + (size_t)rg * nfeat + c);
                                float2 v = make_float2(acc2[j][0] * i0, acc2[j][1] * i1);
                                if (m > 0) {
                                    const float2 q = *o;
                                    v.x += q.x;
                                    v.y += q.y;
                                }
                                *o = v;
                            }
                            if (rg8 < nrows) {
                                float2 *o = reinterpret_cast<float2 *>(a.dX + (size_t)rg8 * nfeat + c);
                                float2 v = make_float2(acc2[j][2] * i0, acc2[j][3] * i1);
                                if (m > 0) {
                                    const float2 q = *o;
                                    v.x += q.x;
                                    v.y += q.y;
                                }
                                *o = v;
                            }
                        }
                    }
                }
            }
            if (TRAIN) {
                __syncthreads();
                for (int k = tid; k < HID + 2; k += THREADS) {
                    float s = 0.f;
                    for (int w = 0; w < THREADS / 32; ++w) s += red[w][k];
                    if (k < HID)
                        a.partial[((size_t)m * a.splits + tile) * a.nparam + a.ow4 + k] = s;
                    else if (k == HID)
                        a.partial[((size_t)m * a.splits + tile) * a.nparam + a.ob4] = s;
                    else
                        a.loss[(size_t)m * a.splits + tile] = s;
                }
            }
            __syncwarp();
        }
    }
}

// ------------------------------------------------------------------------------------
// weight gradients: P[m][split][W_l] = H_{l-1}^T dZ_l over the split's 128 rows,
// P[m][split][b_l] = column sums of dZ_l. Grid: x = 64-row blocks of W1, W2, W3; y = split;
// z = member. 4 warps, each 16 rows of the 64-row block by all 128 columns.
// ------------------------------------------------------------------------------------
struct WArgs {
    int in_pad;
    size_t oW1, ob1, oW2, ob2, oW3, ob3, nparam;
    const uint16_t *acts;
    int B, splits;
    float *partial;
};

constexpr int WG_LDA = 72, WG_LDB = HID + 8;

__global__ void __launch_bounds__(128) k_wgrad(WArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16 *As = reinterpret_cast<__nv_bfloat16 *>(smem); // [128][72]
    __nv_bfloat16 *Bs = As + 128 * WG_LDA;                        // [128][136]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int nb1 = (a.in_pad + 63) / 64;
    const int bx = blockIdx.x;
    int layer, mt;
    if (bx < nb1) {
        layer = 0;
        mt = bx;
    } else if (bx < nb1 + 2) {
        layer = 1;
        mt = bx - nb1;
    } else {
        layer = 2;
        mt = bx - nb1 - 2;
    }
    const int s = blockIdx.y, m = blockIdx.z;
    const size_t B = (size_t)a.B;
    const uint16_t *base = a.acts + (size_t)m * B * (a.in_pad + 5 * HID);
    const uint16_t *X = base, *H1 = X + B * a.in_pad, *H2 = H1 + B * HID, *dZ1 = H2 + B * HID, *dZ2 = dZ1 + B * HID,
                   *dZ3 = dZ2 + B * HID;
    const uint16_t *act = layer == 0 ? X : (layer == 1 ? H1 : H2);
    const uint16_t *dz = layer == 0 ? dZ1 : (layer == 1 ? dZ2 : dZ3);
    const int lda = layer == 0 ? a.in_pad : HID, M = lda;
    const size_t oW = layer == 0 ? a.oW1 : (layer == 1 ? a.oW2 : a.oW3);
    const size_t ob = layer == 0 ? a.ob1 : (layer == 1 ? a.ob2 : a.ob3);
    const int k0 = s * 128, mbase = mt * 64;
    for (int v = tid; v < 128 * 8; v += 128) {
        const int r = v >> 3, c = (v & 7) * 8;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (mbase + c < M) val = *reinterpret_cast<const uint4 *>(act + (size_t)(k0 + r) * lda + mbase + c);
        *reinterpret_cast<uint4 *>(As + r * WG_LDA + c) = val;
    }
    for (int v = tid; v < 128 * 16; v += 128) {
        const int r = v >> 4, c = (v & 15) * 8;
        *reinterpret_cast<uint4 *>(Bs + r * WG_LDB + c) = *reinterpret_cast<const uint4 *>(dz + (size_t)(k0 + r) * HID + c);
    }
    __syncthreads();
    float acc[16][4];
#pragma unroll
    for (int nt = 0; nt < 16; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
    const int mrow0 = warp * 16;
    const int arow = (lane & 7) + ((lane >> 4) & 1) * 8, acol = ((lane >> 3) & 1) * 8;
    const int brow = (lane & 7) + ((lane >> 3) & 1) * 8, bcol = ((lane >> 4) & 1) * 8;
#pragma unroll 2
    for (int ks = 0; ks < 8; ++ks) {
        uint32_t af[4];
        ldsm4t(af, As + (ks * 16 + arow) * WG_LDA + mrow0 + acol);
#pragma unroll
        for (int np = 0; np < 8; ++np) {
            uint32_t b[4];
            ldsm4t(b, Bs + (ks * 16 + brow) * WG_LDB + np * 16 + bcol);
            mma(acc[2 * np], af, b[0], b[1]);
            mma(acc[2 * np + 1], af, b[2], b[3]);
        }
    }
    float *P = a.partial + ((size_t)m * a.splits + s) * a.nparam;
    const int mr = mbase + mrow0 + g;
#pragma unroll
    for (int nt = 0; nt < 16; ++nt) {
        const int col = nt * 8 + 2 * tig;
        if (mr < M) *reinterpret_cast<float2 *>(P + oW + (size_t)mr * HID + col) = make_float2(acc[nt][0], acc[nt][1]);
        if (mr + 8 < M)
            *reinterpret_cast<float2 *>(P + oW + (size_t)(mr + 8) * HID + col) = make_float2(acc[nt][2], acc[nt][3]);
    }
    if (mt == 0) {
        float sum = 0.f;
        for (int r = 0; r < 128; ++r) sum += __bfloat162float(Bs[r * WG_LDB + tid]);
        P[ob + tid] = sum;
    }
}

// ------------------------------------------------------------------------------------
// parameter packing and Adam
// ------------------------------------------------------------------------------------
__device__ __forceinline__ long long packed_index(int in_pad, int p1, size_t oW2, size_t ob1, size_t ob2, size_t oW3,
                                                  size_t ob3, size_t p) {
    if (p < ob1) {
        const size_t k = p / HID, n = p % HID;
        return (long long)(n * p1 + k);
    }
    if (p >= oW2 && p < ob2) {
        const size_t q = p - oW2, k = q / HID, n = q % HID;
        return (long long)((size_t)HID * p1 + n * P2 + k);
    }
    if (p >= oW3 && p < ob3) {
        const size_t q = p - oW3, k = q / HID, n = q % HID;
        return (long long)((size_t)HID * p1 + (size_t)HID * P2 + n * P2 + k);
    }
    return -1;
}

struct PArgs {
    int in_pad, p1;
    size_t ob1, oW2, ob2, oW3, ob3, ob4, nparam, packed;
    int members;
};

__global__ void k_pack(PArgs a, const float *master, uint16_t *packed) {
    const size_t total = (size_t)a.members * a.nparam;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t m = i / a.nparam, p = i % a.nparam;
        const long long q = packed_index(a.in_pad, a.p1, a.oW2, a.ob1, a.ob2, a.oW3, a.ob3, p);
        if (q >= 0) packed[m * a.packed + q] = __bfloat16_as_ushort(__float2bfloat16_rn(master[i]));
    }
}

__global__ void k_adam(PArgs a, float *master, uint16_t *packed, float *m1, float *m2, const float *partial, int splits,
                       float lr, float beta1, float beta2, float eps, float wd, float bc1, float bc2) {
    const size_t total = (size_t)a.members * a.nparam;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t m = i / a.nparam, p = i % a.nparam;
        if (p > a.ob4) continue; // row padding of the parameter vector
        float gs = 0.f;
        for (int s = 0; s < splits; ++s) gs += partial[(m * splits + s) * a.nparam + p];
        const float mm = beta1 * m1[i] + (1.f - beta1) * gs;
        const float vv = beta2 * m2[i] + (1.f - beta2) * gs * gs;
        m1[i] = mm;
        m2[i] = vv;
        const long long q = packed_index(a.in_pad, a.p1, a.oW2, a.ob1, a.ob2, a.oW3, a.ob3, p);
        float w = master[i];
        if (q >= 0) w -= lr * wd * w;
        w -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
        master[i] = w;
        if (q >= 0) packed[m * a.packed + q] = __bfloat16_as_ushort(__float2bfloat16_rn(w));
    }
}

// ------------------------------------------------------------------------------------
// host wrappers
// ------------------------------------------------------------------------------------
static void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("surrogate MLP: ") + what + ": " + cudaGetErrorString(e));
}

// the dynamic shared memory attribute is set once per device and size, so that calls
// inside a stream capture make no attribute calls
template <typename F>
static void ensure_smem(F fn, size_t bytes, size_t *cache) {
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) dev = 0;
    if (cache[dev] >= bytes) return;
    check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), "smem attribute");
    cache[dev] = bytes;
}

static KArgs kargs(const Net &net) {
    KArgs a{};
    const Layout &L = net.L;
    a.nch = L.nch;
    a.in_pad = L.in_pad;
    a.p1 = L.p1;
    a.ob1 = L.ob1;
    a.ob2 = L.ob2;
    a.ob3 = L.ob3;
    a.ow4 = L.ow4;
    a.ob4 = L.ob4;
    a.nparam = L.nparam;
    a.packed = L.packed;
    a.scratch = warp_scratch(L);
    a.members = net.members;
    a.master = net.master;
    a.wpacked = net.packed;
    a.mean = net.mean;
    a.inv_std = net.inv_std;
    return a;
}

void infer(const Net &net, const float *G, const int *center, int rows, float *E, float *dX, int sms, cudaStream_t s) {
    if (rows <= 0) return;
    static size_t cache[64] = {0};
    const size_t sm = smem_bytes(net.L);
    ensure_smem(k_mlp<false>, sm, cache);
    KArgs a = kargs(net);
    a.G = G;
    a.center = center;
    a.rows = rows;
    a.E = E;
    a.dX = dX;
    const int ntiles = (rows + TILE - 1) / TILE;
    const int grid = std::max(1, std::min(ntiles, std::max(1, sms)));
    k_mlp<false><<<grid, THREADS, sm, s>>>(a);
    check(cudaGetLastError(), "k_mlp launch");
}

void train_fwdbwd(const Net &net, const float *G, const int *center, const float *target, const int *idx, int B,
                  float *E, uint16_t *acts, float *partial, float *loss, cudaStream_t s) {
    if (B <= 0 || B % TILE) throw std::invalid_argument("surrogate training: batch must be a positive multiple of 128");
    static size_t cache[64] = {0};
    const size_t sm = smem_bytes(net.L);
    ensure_smem(k_mlp<true>, sm, cache);
    KArgs a = kargs(net);
    a.G = G;
    a.center = center;
    a.rows = B;
    a.E = E;
    a.target = target;
    a.idx = idx;
    a.acts = acts;
    a.partial = partial;
    a.loss = loss;
    a.splits = B / TILE;
    k_mlp<true><<<dim3(B / TILE, net.members), THREADS, sm, s>>>(a);
    check(cudaGetLastError(), "k_mlp (train) launch");
}

void wgrad(const Net &net, const uint16_t *acts, int B, float *partial, cudaStream_t s) {
    if (B <= 0 || B % TILE) throw std::invalid_argument("surrogate training: batch must be a positive multiple of 128");
    static size_t cache[64] = {0};
    const size_t sm = (size_t)128 * (WG_LDA + WG_LDB) * 2;
    ensure_smem(k_wgrad, sm, cache);
    const Layout &L = net.L;
    WArgs a{};
    a.in_pad = L.in_pad;
    a.oW1 = L.oW1;
    a.ob1 = L.ob1;
    a.oW2 = L.oW2;
    a.ob2 = L.ob2;
    a.oW3 = L.oW3;
    a.ob3 = L.ob3;
    a.nparam = L.nparam;
    a.acts = acts;
    a.B = B;
    a.splits = B / TILE;
    a.partial = partial;
    const int nb = (L.in_pad + 63) / 64 + 4;
    k_wgrad<<<dim3(nb, B / TILE, net.members), 128, sm, s>>>(a);
    check(cudaGetLastError(), "k_wgrad launch");
}

static PArgs pargs(const Layout &L, int members) {
    PArgs a{};
    a.in_pad = L.in_pad;
    a.p1 = L.p1;
    a.ob1 = L.ob1;
    a.oW2 = L.oW2;
    a.ob2 = L.ob2;
    a.oW3 = L.oW3;
    a.ob3 = L.ob3;
    a.ob4 = L.ob4;
    a.nparam = L.nparam;
    a.packed = L.packed;
    a.members = members;
    return a;
}

void adam(const Layout &L, int members, float *master, uint16_t *packed, float *m1, float *m2, const float *partial,
          int splits, float lr, float beta1, float beta2, float eps, float weight_decay, int step, cudaStream_t s) {
    const float bc1 = 1.f - powf(beta1, (float)step), bc2 = 1.f - powf(beta2, (float)step);
    const size_t total = (size_t)members * L.nparam;
    const int grid = (int)std::min<size_t>((total + 255) / 256, 4096);
    k_adam<<<grid, 256, 0, s>>>(pargs(L, members), master, packed, m1, m2, partial, splits, lr, beta1, beta2, eps,
                                weight_decay, bc1, bc2);
    check(cudaGetLastError(), "k_adam launch");
}

void pack(const Layout &L, int members, const float *master, uint16_t *packed, cudaStream_t s) {
    check(cudaMemsetAsync(packed, 0, (size_t)members * L.packed * 2, s), "memset packed");
    const size_t total = (size_t)members * L.nparam;
    const int grid = (int)std::min<size_t>((total + 255) / 256, 4096);
    k_pack<<<grid, 256, 0, s>>>(pargs(L, members), master, packed);
    check(cudaGetLastError(), "k_pack launch");
}

} // namespace d3mlp

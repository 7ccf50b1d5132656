// Per-atom MLP of the learned ATM surrogate: an ensemble of networks
//     in -> 128 -> 128 -> 128 -> 1, SiLU after each hidden layer,
// hidden GEMMs on the tensor cores with BF16 weights and activations and FP32
// accumulation; biases and the 128 -> 1 projection in FP32.
//
// Input row r: the descriptor G[r][nch*32] normalised as (G - mean) * inv_std, followed
// by a one-hot of the atom's own channel, zero-padded to in_pad (a multiple of 16).
//
// Parameters of one member, FP32 master copy (offsets in `Layout`):
//     W1[in_pad][128] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] w4[128] b4
// and the packed BF16 copy the kernels read, transposed (out-major) and row-padded so
// that ldmatrix reads are free of bank conflicts:
//     W1t[128][in_pad + 8] W2t[128][136] W3t[128][136]
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace d3mlp {

constexpr int HID = 128;
constexpr int NRBF = 32;
constexpr int TILE = 128;   // rows per CTA tile: 8 warps x 16 rows
constexpr int THREADS = 256;
constexpr int MAXCH = 8;

struct Layout {
    int nch = 0, in_dim = 0, in_pad = 0, p1 = 0;
    size_t oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0, ow4 = 0, ob4 = 0, nparam = 0;
    size_t packed = 0; // bf16 elements per member
};

Layout make_layout(int nch);

struct Net {
    Layout L;
    int members = 0;
    const float *master = nullptr;           // [members][nparam]
    const uint16_t *packed = nullptr;        // [members][packed]
    const float *mean = nullptr;             // [nch*32]
    const float *inv_std = nullptr;          // [nch*32]
};

// Dynamic shared memory of the fused kernel.
size_t smem_bytes(const Layout &L);

// Inference over `rows` descriptor rows: E[m*rows + r] = output of member m (network
// units); dX[r*nch*32 + f] = sum over members of dE_m/dG[r][f] (descriptor units), when
// dX is not null. `sms` bounds the persistent grid.
void infer(const Net &net, const float *G, const int *center, int rows, float *E, float *dX, int sms,
           cudaStream_t s);

// Training, one mini-batch of B rows per member (B a multiple of 128): member m reads
// rows idx[m*B + r] of G/center/target (target already normalised). Loss per member:
// mean over the batch of (E - target)^2.
//   train_fwdbwd: forward + backward through the activations; writes the activations
//       the weight gradients need into `acts` (per member: X[B][in_pad], H1, H2, dZ1, dZ2,
//       dZ3 [B][128], BF16), the w4/b4 partial gradients of each 128-row tile into
//       partial[(m*splits + tile)*nparam + ...] and each tile's summed squared error into
//       loss[m*splits + tile] (splits = B/128).
//   wgrad: W1..W3 and b1..b3 partial gradients of each 128-row split into `partial`.
//   adam: sums the partials over splits, Adam update of the FP32 master (decoupled weight
//       decay on the weight matrices), refreshes the packed BF16 copy.
size_t acts_elems(const Layout &L, int B);
void train_fwdbwd(const Net &net, const float *G, const int *center, const float *target, const int *idx, int B,
                  float *E, uint16_t *acts, float *partial, float *loss, cudaStream_t s);
void wgrad(const Net &net, const uint16_t *acts, int B, float *partial, cudaStream_t s);
void adam(const Layout &L, int members, float *master, uint16_t *packed, float *m1, float *m2, const float *partial,
          int splits, float lr, float beta1, float beta2, float eps, float weight_decay, int step, cudaStream_t s);
void pack(const Layout &L, int members, const float *master, uint16_t *packed, cudaStream_t s);

} // namespace d3mlp

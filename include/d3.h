/*
 * d3.h -- C ABI of the B200-native DFT-D3 dispersion engine (libd3.so).
 *
 * Drop-in for the C API of LASP-D3 (src/d3.h of that project): the nine entry points
 * below keep the reference's names, argument types (float I/O, uint16_t elements,
 * enums passed as int), units and ownership rules, so its Python cffi binding
 * (src/d3_cffi.py), Fortran iso_c_binding interfaces (src/fortran_d3.f90) and C/C++
 * callers link against this library unchanged.
 *
 * Units and conventions (as the reference):
 *   coordinates and cell in Angstrom, cell rows are lattice vectors;
 *   cutoffs in bohr (not converted);
 *   energy in eV (negative = binding), forces in eV/Angstrom in the caller's atom
 *   order, stress in eV/Angstrom^3 (already divided by the signed cell volume),
 *   row-major 3x3.
 * Threading: a handle must be used from one thread at a time. Work runs on the
 * current CUDA device.
 *
 * Deliberate deviations from the reference, all on error paths:
 *   - set_atoms with more atoms than the handle capacity prints an error and returns
 *     (the reference calls exit(), src/d3_buffer.cu:380-383);
 *   - an element that was not given at init is rejected (the reference silently maps
 *     it through a re-built element list, src/d3_buffer.cu:389-422);
 *   - atomic numbers outside the parameter table are rejected at init.
 */
#ifndef D3_B200_H
#define D3_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef float real_t; /* src/d3_types.h:7 */

typedef enum { ZERO_DAMPING = 0, BJ_DAMPING = 1 } damping_type_t; /* src/d3_types.h:16-19 */

typedef enum {
    PBE = 0,
    PBE0 = 1,
    B3LYP = 2,
    BLYP = 3,
    BP86 = 4,
    REVPBE = 5,
    CUSTOM = 99
} functional_t; /* src/d3_types.h:21-29 */

typedef void d3_handle_t; /* src/d3.h:9 */

/* ---------------- reference ABI (src/d3.h:36-128) ---------------- */

/* One-shot evaluation without ATM (replaces src/d3.h:36-38, src/d3.cu:236-251). */
void compute_dispersion_energy(real_t atoms[][3], uint16_t *elements, uint64_t num_atoms, real_t cell[3][3],
                               real_t cutoff_radius, real_t CN_cutoff_radius, damping_type_t damping_type,
                               functional_t functional_type, real_t *energy, real_t *force, real_t *stress);

/* Handle for repeated evaluations, two-body + CN only (replaces src/d3.h:60-62). */
d3_handle_t *init_d3_handle(uint16_t *elements, uint64_t num_elements, uint64_t max_length, real_t cutoff_radius,
                            real_t coordination_number_cutoff, damping_type_t damping_type,
                            functional_t functional_type);

/* Handle with the ATM three-body term within atm_cutoff (bohr) (replaces src/d3.h:64-66). */
d3_handle_t *init_d3_handle_with_atm(uint16_t *elements, uint64_t length_elements, uint64_t max_length,
                                     real_t cutoff_radius, real_t coordination_number_cutoff, real_t atm_cutoff,
                                     damping_type_t damping_type, functional_t functional_type);

/* Coordinates [length][3] in Angstrom and atomic numbers (replaces src/d3.h:82). */
void set_atoms(d3_handle_t *handle, real_t *coords, uint16_t *elements, uint64_t length);

/* Cell, rows = lattice vectors, Angstrom (replaces src/d3.h:90). */
void set_cell(d3_handle_t *handle, real_t cell[3][3]);

/* Release the handle after synchronising its work (replaces src/d3.h:97). */
void free_d3_handle(d3_handle_t *handle);

/* Kept for ABI compatibility: every evaluation starts from cleared intermediates
   (replaces src/d3.h:106). */
void clear_d3_handle(d3_handle_t *handle);

/* Energy (eV), forces [n][3] (eV/A), stress [9] (eV/A^3) (replaces src/d3.h:115). */
void compute_dispersion_energy_from_handle(d3_handle_t *handle, real_t *energy, real_t *force, real_t *stress);

/* Same, returning the status word: 0 success; bit 0 neighbour-list overflow (as the
   reference's COMPUTE_NEIGHBOR_LIST_OVERFLOW); 1 for a NULL handle or an internal error
   (replaces src/d3.h:127-128, src/d3.cu:130-226). Additional bits of this engine:
   0x02 non-finite input, 0x04 degenerate cell, 0x08 lattice shift out of range,
   0x10 CUDA error, 0x20 atoms or cell not set. */
uint16_t compute_dispersion_energy_from_handle_status(d3_handle_t *handle, real_t *energy, real_t *force,
                                                      real_t *stress);

/* ---------------- additive extensions (no reference counterpart) ---------------- */

/* Parameter table layout: 5 references / 95 elements (reference default) or the
   7-reference / 103-element layout of USE_EXTENDED_PARAMETERS. */
enum { D3_TABLE_5REF = 0, D3_TABLE_7REF = 1 };

/* Handle with double-precision cutoffs and the table layout chosen at run time;
   rc_atm <= 0 disables ATM. */
d3_handle_t *d3_init_handle_ex(const uint16_t *elements, uint64_t n_elements, uint64_t max_length, double rc,
                               double rc_cn, double rc_atm, int damping_type, int functional_type, int table);

/* FP64 input/output path: Angstrom in, eV / eV/A / eV/A^3 out, same conventions. */
int d3_set_atoms_f64(d3_handle_t *handle, const double *coords, const uint16_t *elements, uint64_t length);
int d3_set_cell_f64(d3_handle_t *handle, const double cell[9]);
uint16_t d3_compute_f64(d3_handle_t *handle, double *energy, double *force, double *stress);

/* Options (value 0/1): */
enum {
    D3_OPT_ATM_FORCE_SCALED = 1, /* 1: apply the 1/2, 1/6 repeated-index ATM factors to forces too
                                    (forces = -dE/dx); 0 (default): reference convention */
    D3_OPT_SMOOTH_CN = 2,        /* tanh^3 CN cutoff (reference compile-time SMOOTH_CUTOFF_CN) */
    D3_OPT_PRECISION = 3,        /* 0 (default): FP64 throughout (plain form); 1: FP32 pair and
                                    triplet arithmetic with FP64 C6 weights, dE/dCN and final
                                    reductions (precision form) */
    D3_OPT_BIN_DIVISOR = 4,      /* cell-list bin width = smallest cutoff / value (1..32, default 6) */
    D3_OPT_ATM_TILE = 5,         /* ATM partner tile entries (0 = automatic) */
    D3_OPT_ATM_CTAS_PER_SM = 6,  /* persistent ATM CTAs per SM (0 = occupancy limit) */
    D3_OPT_ATM_SCHEDULE = 8,     /* precision-form ATM: 0 (default) block pairs, each triplet
                                    visited once; 1 mirror-symmetric, each triplet twice */
    D3_OPT_ATM_LIST_CAPACITY = 9, /* ATM half-list capacity in entries (0 = estimated from the
                                    density, the default). A synchronous evaluation whose
                                    list overflows grows it and runs again; an asynchronous
                                    one (d3_compute_async, graph replays) sets status bit 0
                                    and leaves the ATM terms out instead */
    D3_OPT_PAIR_KERNEL = 10,     /* two-body pass: 0 (default) compact groups of 32 atoms with
                                    staged partners (one thread per atom); 1 one warp per atom
                                    (also used for sharded evaluations and handles of more
                                    than 8 elements) */
    D3_OPT_ATMB_WARPS = 11,      /* precision-form block-pair ATM kernel: warps per CTA, 0 =
                                    automatic (8), 2..12; above 8 each warp stages one y
                                    block at a time instead of two. With
                                    D3_OPT_ATM_CTAS_PER_SM = 2, two CTAs per SM when they fit */
    D3_OPT_ATMB_LIST_CAPACITY = 12, /* longest half list (entries) the block-pair kernel takes,
                                    0 = as many as the shared memory allows (4,096..8,192);
                                    longer lists go to the mirror-symmetric kernel */
    D3_OPT_ATMB_SPLIT = 13,      /* CTAs of the block-pair kernel sharing one apex, each taking
                                    every S-th block row (0 = automatic: more than one only
                                    when the apexes are fewer than about 3 per CTA, e.g. the
                                    96-atom water box; 1..64) */
    D3_OPT_ATMB_FINE_SKIP = 14   /* block-pair kernel: 1 (default) skips out-of-range visits
                                    per two steps, 0 per four steps (more overlap of the
                                    packed pairs) */
};
int d3_set_option(d3_handle_t *handle, int option, int value);

/* Damping parameters for CUSTOM (or to override a functional): s6, s8 and
   (sr6, sr8) for zero damping or (a1, a2) for BJ damping. */
int d3_set_functional_params(d3_handle_t *handle, double s6, double s8, double p1, double p2);

/* Batching form: many independent periodic structures in one handle, evaluated by one
   launch per pass (the ATM pass is one persistent launch over all structures' apexes).
   d3_init_batch sizes the handle for up to max_structures structures holding together
   up to max_total_atoms atoms. d3_set_batch_f64 takes the atom counts per structure,
   the concatenated coordinates [n][3] and elements [n] (structure by structure, Angstrom)
   and one cell per structure [n_structures][9] (Angstrom, rows = lattice vectors).
   d3_compute_batch_f64 returns energies [n_structures] (eV), forces [n][3] (eV/A, same
   order as given) and stresses [n_structures][9] (eV/A^3). The single-structure calls
   refuse a handle that holds more than one structure. */
d3_handle_t *d3_init_batch(const uint16_t *elements, uint64_t n_elements, uint64_t max_structures,
                           uint64_t max_total_atoms, double rc, double rc_cn, double rc_atm, int damping_type,
                           int functional_type, int table);
int d3_set_batch_f64(d3_handle_t *handle, uint64_t n_structures, const uint64_t *atom_counts, const double *coords,
                     const uint16_t *elements, const double *cells);
uint16_t d3_compute_batch_f64(d3_handle_t *handle, double *energies, double *forces, double *stresses);
int d3_num_structures(d3_handle_t *handle);

/* Replace the positions of the atoms already set (same count and elements) from device
   memory (double, Angstrom, [n][3]), ordered on cuda_stream; with d3_compute_async this
   lets an MD loop run without host copies and be captured in a CUDA graph. */
int d3_set_positions_device(d3_handle_t *handle, const double *coords_dev, void *cuda_stream);

/* Enqueue one evaluation on a CUDA stream (cudaStream_t passed as void*, NULL = the
   handle's stream) with no host synchronisation; results stay on the device at
   d3_device_results(): energies [S], forces [3n], stresses [9S] (double, eV units; S = 1
   for a single-structure handle). The neighbour-list capacity must already be sufficient (run one
   d3_compute_f64 or compute_dispersion_energy_from_handle_status first). */
uint16_t d3_compute_async(d3_handle_t *handle, void *cuda_stream);
const double *d3_device_results(d3_handle_t *handle);
/* Status word of the last enqueued evaluation (synchronise its stream first): how an
   asynchronous or graph-replayed evaluation reports a list overflow (bit 0) or bad input
   (bit 1). d3_atm_list_capacity: the ATM half-list capacity now allocated (entries). */
uint16_t d3_fetch_status(d3_handle_t *handle);
int64_t d3_atm_list_capacity(d3_handle_t *handle);
/* Stream-ordered device-to-device copy of the results of the last enqueued evaluation
   (energies [S], forces [n][3], stresses [S][9], double) to a caller buffer; it can be
   captured in a CUDA graph together with d3_compute_async (MD loops). */
int d3_copy_results_device(d3_handle_t *handle, double *results_dev, void *cuda_stream);

/* Copy the device results of the last evaluation to host arrays (energies [S], forces
   [n][3], stresses [S][9]; any may be NULL). Synchronise the evaluation's stream first. */
int d3_fetch_results(d3_handle_t *handle, double *energies, double *forces, double *stresses);

/* Device time (ms, CUDA events on the evaluation's stream) of each pass of the last
   evaluation: [0] wrap+bin, [1] CN + C6 weights, [2] two-body, [3] ATM list,
   [4] ATM triplets, [5] chain rule, [6] finalize; returns the number written.
   counters (may be NULL) receives 4 values: ATM in-range triplet visits (two per
   triplet), two-body in-range ordered pairs, CN in-range ordered pairs, 0. */
int d3_pass_times(d3_handle_t *handle, float *ms, int cap, uint64_t *counters);

/* Number of kernels one evaluation launches. */
int d3_launches_per_eval(d3_handle_t *handle);

/* Self-check of the refined reciprocal square root, reciprocal and inverse cube
   root used by the ATM kernel: max relative error against CUDA's double-precision
   functions over [1e-12, 1e14], written to max_rel_err[6] (one Newton step:
   rsqrt, rcp, rcbrt; two Newton steps: rsqrt, rcp, rcbrt). */
int d3_selftest_math(double *max_rel_err);

/* Measured FMA throughput (TFLOP/s, 2 flops per FMA) of the FP64 (fp64 = 1) or FP32
   pipe of the current device: the denominator of the engine's roofline figures. */
double d3_peak_probe(int fp64);

/* Coordination numbers of one periodic structure without any device allocation (no
   counterpart in the reference). For callers that must not allocate device memory
   where they call the library -- e.g. an MD-engine plugin inside its time-step loop,
   where cudaMalloc would synchronise the device, or an application whose memory is all
   owned by its own pool allocator. Inputs and outputs are caller-owned device buffers:
   coords [n][3] (double, Angstrom), elements [n] (atomic numbers), cn [n] (double,
   written). cell is a host array (Angstrom, rows = lattice vectors), cn_cutoff in bohr,
   table D3_TABLE_5REF or D3_TABLE_7REF. Work is enqueued on cuda_stream (NULL = the
   default stream) with no host synchronisation. At most D3_NOALLOC_MAX_ATOMS atoms:
   larger sizes are rejected with an error (return 1, see d3_last_error). The only
   scratch is a fixed array in device memory shared by all calls on a device (held until
   the process exits): calls that overlap on the GPU race on it. The first call on each
   device does a one-time set-up and should come before any stream capture; that set-up
   does not survive cudaDeviceReset. Returns 0 on success. Atoms whose element is outside
   the table get CN = NaN and contribute nothing to the others. Every image within the
   cutoff of the positions wrapped into the cell is used (the handle API follows the
   reference's image box over the positions as given; both agree for atoms given inside
   the cell); the smooth-cutoff CN option has no counterpart here. The work is bounded
   before launch: cells so thin that more than D3_NOALLOC_MAX_IMAGES images, or more than
   2^36 pair-image tests, would be needed are rejected with an error. */
#define D3_NOALLOC_MAX_ATOMS 8192
#define D3_NOALLOC_MAX_IMAGES 4096
int d3_coordination_numbers_noalloc(const double *coords, const uint16_t *elements, uint64_t num_atoms,
                                    const double cell[9], double cn_cutoff, int table, double *cn,
                                    void *cuda_stream);

/* ---- Learned ATM surrogate (no counterpart in the reference) ----------------------
   Per-atom ATM energy from an ensemble of MLPs over per-atom descriptors:
     G_i[c][k] = sum over neighbours j of channel c within rc_ATM of
                 C6_ij exp(-(r_ij - mu_k)^2 / (2 sigma^2)) (1 + cos(pi r_ij / rc_ATM)) / 2
   with 32 centres mu_k uniform in 0.8 .. 21 A, sigma = 0.7 A, C6_ij the exact
   CN-dependent coefficient. Network input: (G - mean) * inv_std, then a one-hot of the
   atom's own channel. Each member: in -> 128 -> 128 -> 128 -> 1, SiLU, BF16 hidden
   weights on the tensor cores, FP32 accumulation. E_i (eV) = e_scale * mean over members
   + e_shift[channel of i]. Atoms whose ensemble standard deviation (population, eV)
   exceeds the threshold (default 2e-4 eV) take their exact share instead: all triplets
   through them, each weighted 1/3, by the exact ATM kernel. Forces, stress and dE/dCN
   are the analytic derivatives of that energy (forces = -dE/dx, so repeated-index
   triplets are force-scaled in the fallback share).

   Parameter vector of one member (FP32, d3_mlp_layout gives the offsets):
     W1[in_pad][128] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] w4[128] b4
   with in_pad = 16-aligned (33 * nch), W[in][out] (row = input). */
#define D3_OPT_ATM_SURROGATE 7 /* d3_set_option value 1: evaluate ATM through the surrogate */
int d3_set_surrogate(d3_handle_t *handle, const int *channel_z, int n_channels, int members, const float *params,
                     const float *mean, const float *inv_std, const float *e_shift, float e_scale);
int d3_set_surrogate_threshold(d3_handle_t *handle, double std_threshold_ev);
/* atoms that took the exact fallback in the last evaluation */
int d3_surrogate_flagged(d3_handle_t *handle);
/* After an evaluation: descriptors of the handle's atoms for the given channels, in
   the caller's atom order, into device memory: G_dev [n][32 * n_channels] (float),
   center_dev [n] (channel of each atom, -1 if none), e_atm_dev [n] (double, eV: the
   per-atom ATM energy of the last evaluation, one third of every triplet through the
   atom). Any output may be NULL. */
int d3_surrogate_descriptors(d3_handle_t *handle, const int *channel_z, int n_channels, float *G_dev,
                             int *center_dev, double *e_atm_dev, void *cuda_stream);

/* Network kernels on caller device buffers (training and standalone evaluation).
   d3_mlp_layout: out[12] = in_dim, in_pad, oW1, ob1, oW2, ob2, oW3, ob3, ow4, ob4,
   nparam (floats per member), packed (BF16 elements per member of the packed copy).
   d3_mlp_pack: BF16 packed copy of the FP32 parameters [members][nparam].
   d3_mlp_forward: E_dev [members][rows] network outputs; dX_dev (may be NULL)
   [rows][32 * n_channels] = sum over members of dE/dG.
   d3_mlp_train_batch: forward, backward and weight gradients of one mini-batch of
   B rows (a multiple of 128) per member, member m reading rows idx_dev[m * B + r];
   target_dev holds normalised targets; loss = mean squared error per member. Writes
   E_dev [members][B], the partial gradients partial_dev [members][B/128][nparam] and
   loss_dev [members][B/128] (summed squared errors per 128-row split); acts_dev is
   scratch of d3_mlp_acts_elems(n_channels, B) BF16 elements per member.
   d3_mlp_adam: sums the partial gradients, Adam step (step counts from 1) with
   decoupled weight decay on the weight matrices, refreshes the packed copy. */
int d3_mlp_layout(int n_channels, uint64_t *out);
uint64_t d3_mlp_acts_elems(int n_channels, int B);
int d3_mlp_pack(int n_channels, int members, const float *params_dev, uint16_t *packed_dev, void *cuda_stream);
int d3_mlp_forward(int n_channels, int members, const float *params_dev, const uint16_t *packed_dev,
                   const float *mean_dev, const float *inv_std_dev, const float *G_dev, const int *center_dev,
                   int rows, float *E_dev, float *dX_dev, void *cuda_stream);
int d3_mlp_train_batch(int n_channels, int members, const float *params_dev, const uint16_t *packed_dev,
                       const float *mean_dev, const float *inv_std_dev, const float *G_dev, const int *center_dev,
                       const float *target_dev, const int *idx_dev, int B, float *E_dev, uint16_t *acts_dev,
                       float *partial_dev, float *loss_dev, void *cuda_stream);
int d3_mlp_adam(int n_channels, int members, float *params_dev, uint16_t *packed_dev, float *m1_dev, float *m2_dev,
                const float *partial_dev, int splits, float lr, float beta1, float beta2, float eps,
                float weight_decay, int step, void *cuda_stream);

/* Sharded evaluation of one structure by `world` cooperating processes, one per GPU (no
   counterpart in the reference). Every rank holds the same handle contents (atoms, cell,
   options). d3_shard_begin computes the coordination numbers and C6 weights of every atom
   and the two-body and ATM terms of this rank's share of the atoms (every world-th one),
   and writes this rank's part of dE/dCN (d3_shard_length(handle) doubles) to dedcn_dev.
   The caller sums dedcn_dev over the ranks (an all-reduce); d3_shard_end then runs the
   dE/dCN chain rule for this rank's share and writes this rank's part of the results
   (energies [S], forces [n][3], stresses [S][9], double, eV units, the layout of
   d3_device_results) to results_dev; the sum of results_dev over the ranks is the result.
   results_dev must hold 10 S + 3 n doubles, S = d3_num_structures(handle) and
   n = d3_shard_length(handle): d3_shard_end writes that many whatever the buffer's size.
   d3_shard_begin synchronises cuda_stream (it checks the neighbour-list capacity); the
   learned surrogate is not available here. Returns the status word. */
uint64_t d3_shard_length(d3_handle_t *handle);
uint16_t d3_shard_begin(d3_handle_t *handle, int rank, int world, double *dedcn_dev, void *cuda_stream);
uint16_t d3_shard_end(d3_handle_t *handle, const double *dedcn_dev, double *results_dev, void *cuda_stream);

/* Last error message of this thread ("" if none). */
const char *d3_last_error(void);

/* Diagnostics (caller atom order): coordination numbers, dE/dCN (hartree), per-atom
   energies (hartree, reference sign); ATM half list as rows (apex, j, Tx, Ty, Tz) with
   the reference's lattice shifts; wrap shifts and bin index of each atom. */
int d3_debug_atom_arrays(d3_handle_t *handle, double *cn, double *dedcn, double *energy_atoms);
int64_t d3_debug_atm_pairs(d3_handle_t *handle, int64_t *rows, int64_t cap);
int d3_debug_bins(d3_handle_t *handle, int64_t *wrap_shift, int64_t *bin_index, int *num_bins);
/* Per-pass terms of the last evaluation, D3_DEBUG_TERM_COLUMNS doubles per atom (caller
   order; hartree and bohr, the reference's sign conventions): [0] two-body energy (half
   of every ordered pair of the atom), [1] its dE/dCN, [2..4] its force, [5..10] its
   virial; [11] ATM apex share (a third of the energy of every triplet whose largest
   index is the atom), [12] the atom's dE/dCN from those triplets, [13..15] its force
   from them, [16..21] their virial; [22..24] dE/dCN chain-rule force, [25..30] its
   virial. Virials are xx yy zz xy xz yz, already divided by the cell volume (two-body
   and chain rule: also by 2). Diagnostics for parity tests (no reference counterpart). */
#define D3_DEBUG_TERM_COLUMNS 31
int d3_debug_pass_terms(d3_handle_t *handle, double *terms);

#ifdef __cplusplus
}
#endif

#endif /* D3_B200_H */

// Internal engine interface for the B200 D3 dispersion path.
//
// The engine replaces the reference's d3.cu driver, d3_buffer device storage and the
// d3_kernel passes (LASP-D3 src/d3.cu:130-226, src/d3_buffer.cu, src/d3_kernel.cu):
//   wrap + bin (GPU counting sort) -> CN -> per-atom Gaussian C6 weights ->
//   [ATM half-list build -> ATM triplets] + two-body -> dE/dCN chain rule -> reductions.
// Everything for one evaluation runs on one stream with no host synchronisation until
// the final device-to-host copy.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "d3_geometry.h"

namespace d3 {

constexpr double ANG2BOHR = 1.0 / 0.52917726;   // src/d3.cu:50 (here in double)
constexpr double HARTREE_EV = 27.211396641308;   // src/d3.cu:205
constexpr int MAX_NREF = 7;
constexpr int MAX_TYPES = 32;

// status bits (0 = success, bit 0 = neighbour-list overflow as in the reference's
// d3_internal.h:7, other bits are additions of this engine)
enum : uint16_t {
    ST_OK = 0,
    ST_LIST_OVERFLOW = 1u << 0,
    ST_BAD_INPUT = 1u << 1,      // non-finite coordinate or cell
    ST_BAD_CELL = 1u << 2,       // degenerate cell
    ST_SHIFT_RANGE = 1u << 3,    // lattice shift outside the packed range
    ST_CUDA_ERROR = 1u << 4,
    ST_NOT_READY = 1u << 5,      // atoms or cell not set
};

struct FuncParams {
    double s6, s8, p1, p2; // zero: p1 = sr6, p2 = sr8; BJ: p1 = a1, p2 = a2
};

struct Options {
    bool atm_force_scaled = false; // false: reference convention (ATM forces not scaled
                                   // by the 1/2, 1/6 repeated-index factors)
    bool smooth_cn = false;        // tanh^3 CN cutoff (reference SMOOTH_CUTOFF_CN)
    int precision = 0;             // 0: FP64 plain form; 1: FP32 pair/triplet arithmetic with
                                   // FP64 weights, dE/dCN and reductions (precision form)
    // tunables (set by the autotuner or the caller)
    double bin_divisor = 6.0;      // bin width = smallest cutoff / bin_divisor
    int atm_tile = 0;              // ATM partner tile entries (0: largest that fits, <= 128)
    int atm_ctas_per_sm = 0;       // persistent ATM CTAs per SM (0: occupancy limit)
    bool atm_surrogate = false;    // learned ATM surrogate with exact fallback (needs a model)
    int atm_schedule = 0;          // precision-form ATM: 0 block pairs (each triplet once),
                                   // 1 mirror-symmetric full square (each triplet twice)
    long long atm_list_capacity = 0; // ATM half-list entries to allocate (0: estimate from the
                                     // density); a synchronous evaluation regrows on overflow
    int pair_kernel = 0;           // two-body pass: 0 atom groups with staged partners,
                                   // 1 one warp per atom
    int atmb_warps = 0;            // block-pair ATM: warps per CTA (0: automatic; above 8
                                   // with one y buffer per warp)
    int atmb_mcap = 0;             // block-pair ATM: longest list it takes (0: automatic)
    int atmb_split = 0;            // block-pair ATM: CTAs sharing one apex (0: automatic,
                                   // more than one only when apexes are fewer than CTAs)
    int atmb_fine_skip = 1;        // block-pair ATM: skip out-of-range visits per packed pair
                                   // of steps (1) or per four steps (0)
};

// Learned ATM surrogate: network parameters and normalisation (network in d3_mlp.h).
// Per-atom ATM energy (eV) of atom i = e_scale * mean_m(net_m(x_i)) + e_shift[channel(i)];
// atoms whose ensemble standard deviation (population, eV) exceeds the threshold take
// their exact share instead (all triplets through them, weight 1/3 each).
struct SurrogateModel {
    std::vector<int> channel_z;   // atomic number of each neighbour/centre channel
    int members = 0;
    std::vector<float> master;    // [members][nparam] FP32 parameters
    std::vector<float> mean;      // [nch*32] descriptor normalisation
    std::vector<float> inv_std;   // [nch*32]
    std::vector<float> e_shift;   // [nch] eV
    float e_scale = 1.0f;         // eV per network unit
};

struct Engine;

Engine *engine_create(const uint16_t *elements, uint64_t n_elements, uint64_t max_atoms, double rc, double rc_cn,
                      double rc_atm, bool use_atm, int damping, int functional, bool extended, std::string &err,
                      uint64_t max_structs = 1);
void engine_destroy(Engine *e);
int engine_set_atoms(Engine *e, const double *pos_bohr, const uint16_t *Z, uint64_t n, std::string &err);
int engine_set_cell(Engine *e, const double cell_bohr[9], const float cell_bohr_f[9], std::string &err);
// many independent structures in one handle: counts[k] atoms each, concatenated
// positions (bohr), elements and cells (bohr, 9 per structure)
int engine_set_batch(Engine *e, uint64_t nstruct, const uint64_t *counts, const double *pos_bohr, const uint16_t *Z,
                     const double *cells_bohr, const float *cells_f, std::string &err);
// replace positions from device memory (Angstrom, caller order; same atoms), stream-ordered
int engine_set_positions_device(Engine *e, const double *coords_ang_dev, cudaStream_t stream);
int engine_num_structures(const Engine *e);
// copy the device results of the last evaluation (caller synchronises its stream first)
void engine_fetch_results(Engine *e, double *energies, double *forces, double *stresses);
void engine_set_options(Engine *e, const Options &o);
Options engine_get_options(const Engine *e);
void engine_set_functional_params(Engine *e, const FuncParams &p);
// Runs the whole evaluation on `stream` (the engine's own stream when null) and,
// when sync is true, waits and copies results to the host outputs: energies [S] (eV),
// forces [3n] (eV/A, caller order), stresses [9S] (eV/A^3). Returns the status word.
uint16_t engine_compute(Engine *e, double *energy_ev, double *forces_ev_a, double *stress_ev_a3,
                        cudaStream_t stream, bool sync);
// device-resident results of the last evaluation (eV units, caller order)
const double *engine_device_results(const Engine *e); // [S energies, 3n forces, 9S stresses]
uint64_t engine_num_atoms(const Engine *e);

// per-pass device times (ms) of the last evaluation, from CUDA events on its stream:
// [bin, cn+weights, two-body, atm-list, atm, chain, finalize]; work counters
// [atm in-range visits, two-body ordered pairs, cn ordered pairs, 0]
int engine_pass_times(Engine *e, float *ms, int cap, unsigned long long *counters);
int engine_launches_per_eval(const Engine *e);
// max relative error of the ATM kernel's refined rsqrt / reciprocal / inverse cube root:
// [one Newton step x3, two Newton steps x3]
int engine_selftest_math(double max_rel[6]);
// measured FMA throughput of the FP64 (fp64 = 1) or FP32 pipe, TFLOP/s
double engine_peak_probe(int fp64);

// learned ATM surrogate: load a model (every element of the handle must be a channel),
// set the fallback threshold (eV; default 2e-4), number of atoms that took the exact
// fallback in the last evaluation
int engine_set_surrogate(Engine *e, const SurrogateModel &m, std::string &err);
void engine_set_surrogate_threshold(Engine *e, double ev);
int engine_surrogate_flagged(Engine *e);
// descriptors of the current atoms (valid after an evaluation) for the given channels,
// written to device memory in caller order: G[n][nch*32], centre channel [n] (-1: not a
// channel) and the per-atom ATM energy of the last evaluation (eV, E/3 share of each
// triplet), each output skipped when null
int engine_surrogate_descriptors(Engine *e, const int *channel_z, int nch, float *G_dev, int *center_dev,
                                 double *e_atm_dev, cudaStream_t stream, std::string &err);
// Sharded evaluation of one structure by `world` processes: stage 1 (CN and weights of
// every atom; two-body and ATM of this rank's share) writes this rank's partial dE/dCN
// [n] (binned order) to G_out; the caller sums G over the ranks (all-reduce) and stage 2
// (chain rule of this rank's share, forces, reductions) writes this rank's partial
// results [S energies, 3n forces, 9S stresses] (eV units, caller order) to out_dev; the
// caller sums them over the ranks. Stage 1 synchronises its stream (list capacity).
uint16_t engine_shard_begin(Engine *e, int rank, int world, double *G_out, cudaStream_t stream, std::string &err);
uint16_t engine_shard_end(Engine *e, const double *G_in, double *out_dev, cudaStream_t stream, std::string &err);

// diagnostics for tests: coordination numbers, dE/dCN, per-atom energies (hartree),
// in the caller's atom order; ATM list (caller indices and reference lattice shifts)
int engine_debug_atom_arrays(Engine *e, double *cn, double *dedcn, double *energy_atoms);
int64_t engine_debug_atm_pairs(Engine *e, int64_t *out, int64_t cap);
int engine_debug_pass_terms(Engine *e, double *out);
long long engine_atm_capacity(const Engine *e);
uint16_t engine_fetch_status(Engine *e);
int engine_debug_bins(Engine *e, int64_t *wrap_shift, int64_t *bin_index, int nb_out[3]);

} // namespace d3

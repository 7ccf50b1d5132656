// C ABI of libd3.so: the reference's nine entry points (LASP-D3 src/d3.h:36-128,
// implemented there in src/d3.cu:14-251) plus additive d3_* extensions, on top of the
// engine in d3_engine.cu. No exception crosses this boundary.
#include "../../include/d3.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "d3_engine.h"
#include "d3_mlp.h"

namespace {

thread_local std::string g_last_error;

void set_error(const std::string &msg) {
    g_last_error = msg;
    fprintf(stderr, "Error: %s\n", msg.c_str());
}

struct Handle {
    d3::Engine *engine = nullptr;
    uint64_t n = 0;
    std::vector<double> f64_forces;
};

Handle *H(d3_handle_t *h) { return reinterpret_cast<Handle *>(h); }

// Angstrom -> bohr, float input widened to double (the reference converts in float,
// src/d3.cu:50-60; the FP64 engine keeps the conversion in double)
void to_bohr(const float *in, size_t m, std::vector<double> &out) {
    out.resize(m);
    for (size_t i = 0; i < m; ++i) out[i] = (double)in[i] * d3::ANG2BOHR;
}

d3_handle_t *make_handle(const uint16_t *elements, uint64_t n_el, uint64_t max_len, double rc, double rc_cn,
                         double rc_atm, bool use_atm, int damping, int functional, bool extended) {
    std::string err;
    d3::Engine *e = d3::engine_create(elements, n_el, max_len, rc, rc_cn, rc_atm, use_atm, damping, functional,
                                      extended, err);
    if (!e) {
        set_error(err);
        return nullptr;
    }
    Handle *h = new Handle();
    h->engine = e;
    return reinterpret_cast<d3_handle_t *>(h);
}

std::string status_message(unsigned st) {
    if (st & d3::ST_CUDA_ERROR) return "CUDA error during compute";
    if (st & d3::ST_NOT_READY) return "atoms or cell not set";
    if (st & d3::ST_BAD_CELL) return "degenerate cell (set_cell failed)";
    if (st & d3::ST_BAD_INPUT) return "non-finite coordinate or cell";
    if (st & d3::ST_SHIFT_RANGE) return "lattice shift outside the packed range";
    if (st & d3::ST_LIST_OVERFLOW) return "ATM neighbour list overflow";
    return "";
}

uint16_t compute_float(Handle *h, real_t *energy, real_t *force, real_t *stress) {
    if (d3::engine_num_structures(h->engine) > 1) {
        set_error("handle holds a batch of structures; use d3_compute_batch_f64");
        return d3::ST_BAD_INPUT;
    }
    const uint64_t n = d3::engine_num_atoms(h->engine);
    h->f64_forces.resize(3 * n);
    double e = 0, s[9] = {0};
    uint16_t st = d3::engine_compute(h->engine, &e, h->f64_forces.data(), s, nullptr, true);
    if (st & (d3::ST_CUDA_ERROR | d3::ST_NOT_READY | d3::ST_BAD_CELL)) {
        set_error(status_message(st));
        return st;
    }
    if (energy) *energy = (real_t)e;
    if (force)
        for (uint64_t i = 0; i < 3 * n; ++i) force[i] = (real_t)h->f64_forces[i];
    if (stress)
        for (int i = 0; i < 9; ++i) stress[i] = (real_t)s[i];
    return st;
}

} // namespace

namespace d3 {
// lets other translation units of the library report through d3_last_error()
void record_error(const std::string &msg) { g_last_error = msg; }
} // namespace d3

extern "C" {

d3_handle_t *init_d3_handle(uint16_t *elements, uint64_t num_elements, uint64_t max_length, real_t cutoff_radius,
                            real_t coordination_number_cutoff, damping_type_t damping_type,
                            functional_t functional_type) {
    return make_handle(elements, num_elements, max_length, cutoff_radius, coordination_number_cutoff, 0.0, false,
                       (int)damping_type, (int)functional_type, false);
}

d3_handle_t *init_d3_handle_with_atm(uint16_t *elements, uint64_t length_elements, uint64_t max_length,
                                     real_t cutoff_radius, real_t coordination_number_cutoff, real_t atm_cutoff,
                                     damping_type_t damping_type, functional_t functional_type) {
    return make_handle(elements, length_elements, max_length, cutoff_radius, coordination_number_cutoff, atm_cutoff,
                       true, (int)damping_type, (int)functional_type, false);
}

void set_atoms(d3_handle_t *handle, real_t *coords, uint16_t *elements, uint64_t length) {
    if (!handle) {
        set_error("handle is NULL in set_atoms");
        return;
    }
    std::vector<double> b;
    to_bohr(coords, 3 * length, b);
    std::string err;
    if (d3::engine_set_atoms(H(handle)->engine, b.data(), elements, length, err)) set_error(err);
}

void set_cell(d3_handle_t *handle, real_t cell[3][3]) {
    if (!handle) {
        set_error("handle is NULL in set_cell");
        return;
    }
    double c[9];
    float cf[9];
    const float a2b = 1.0f / 0.52917726f; // the reference's float conversion (src/d3.cu:79-85)
    for (int i = 0; i < 9; ++i) {
        c[i] = (double)cell[i / 3][i % 3] * d3::ANG2BOHR;
        cf[i] = cell[i / 3][i % 3] * a2b;
    }
    std::string err;
    if (d3::engine_set_cell(H(handle)->engine, c, cf, err)) set_error(err);
}

void free_d3_handle(d3_handle_t *handle) {
    if (!handle) {
        set_error("handle is NULL in free_d3_handle");
        return;
    }
    Handle *h = H(handle);
    d3::engine_destroy(h->engine);
    delete h;
}

void clear_d3_handle(d3_handle_t *handle) {
    if (!handle) set_error("handle is NULL in clear_d3_handle");
}

uint16_t compute_dispersion_energy_from_handle_status(d3_handle_t *handle, real_t *energy, real_t *force,
                                                      real_t *stress) {
    if (!handle) {
        set_error("handle is NULL in compute_dispersion_energy_from_handle");
        return 1;
    }
    return compute_float(H(handle), energy, force, stress);
}

void compute_dispersion_energy_from_handle(d3_handle_t *handle, real_t *energy, real_t *force, real_t *stress) {
    uint16_t st = compute_dispersion_energy_from_handle_status(handle, energy, force, stress);
    if (st != 0) fprintf(stderr, "Error: compute_dispersion_energy_from_handle failed with status %d\n", st);
}

void compute_dispersion_energy(real_t atoms[][3], uint16_t *elements, uint64_t num_atoms, real_t cell[3][3],
                               real_t cutoff_radius, real_t CN_cutoff_radius, damping_type_t damping_type,
                               functional_t functional_type, real_t *energy, real_t *force, real_t *stress) {
    // as the reference: a temporary handle without ATM (src/d3.cu:236-251)
    d3_handle_t *h = init_d3_handle(elements, num_atoms, num_atoms, cutoff_radius, CN_cutoff_radius, damping_type,
                                    functional_type);
    if (!h) return;
    set_atoms(h, (real_t *)atoms, elements, num_atoms);
    set_cell(h, cell);
    clear_d3_handle(h);
    compute_dispersion_energy_from_handle(h, energy, force, stress);
    free_d3_handle(h);
}

// ---------------- extensions ----------------

d3_handle_t *d3_init_handle_ex(const uint16_t *elements, uint64_t n_elements, uint64_t max_length, double rc,
                               double rc_cn, double rc_atm, int damping_type, int functional_type, int table) {
    return make_handle(elements, n_elements, max_length, rc, rc_cn, rc_atm, rc_atm > 0.0, damping_type,
                       functional_type, table == D3_TABLE_7REF);
}

int d3_set_atoms_f64(d3_handle_t *handle, const double *coords, const uint16_t *elements, uint64_t length) {
    if (!handle) {
        set_error("handle is NULL in d3_set_atoms_f64");
        return 1;
    }
    std::vector<double> b(3 * length);
    for (uint64_t i = 0; i < 3 * length; ++i) b[i] = coords[i] * d3::ANG2BOHR;
    std::string err;
    if (d3::engine_set_atoms(H(handle)->engine, b.data(), elements, length, err)) {
        set_error(err);
        return 1;
    }
    return 0;
}

int d3_set_cell_f64(d3_handle_t *handle, const double cell[9]) {
    if (!handle) {
        set_error("handle is NULL in d3_set_cell_f64");
        return 1;
    }
    double c[9];
    float cf[9];
    const float a2b = 1.0f / 0.52917726f;
    for (int i = 0; i < 9; ++i) {
        c[i] = cell[i] * d3::ANG2BOHR;
        cf[i] = (float)cell[i] * a2b;
    }
    std::string err;
    if (d3::engine_set_cell(H(handle)->engine, c, cf, err)) {
        set_error(err);
        return 1;
    }
    return 0;
}

uint16_t d3_compute_f64(d3_handle_t *handle, double *energy, double *force, double *stress) {
    if (!handle) {
        set_error("handle is NULL in d3_compute_f64");
        return 1;
    }
    if (d3::engine_num_structures(H(handle)->engine) > 1) {
        set_error("handle holds a batch of structures; use d3_compute_batch_f64");
        return d3::ST_BAD_INPUT;
    }
    uint16_t st = d3::engine_compute(H(handle)->engine, energy, force, stress, nullptr, true);
    if (st) set_error(status_message(st));
    return st;
}

int d3_set_option(d3_handle_t *handle, int option, int value) {
    if (!handle) {
        set_error("handle is NULL in d3_set_option");
        return 1;
    }
    d3::Options o = d3::engine_get_options(H(handle)->engine);
    switch (option) {
    case D3_OPT_ATM_FORCE_SCALED: o.atm_force_scaled = value != 0; break;
    case D3_OPT_SMOOTH_CN: o.smooth_cn = value != 0; break;
    case D3_OPT_BIN_DIVISOR:
        if (value < 1 || value > 32) {
            set_error("D3_OPT_BIN_DIVISOR takes 1..32");
            return 1;
        }
        o.bin_divisor = value;
        break;
    case D3_OPT_ATM_TILE: o.atm_tile = value < 0 ? 0 : value; break;
    case D3_OPT_ATM_CTAS_PER_SM: o.atm_ctas_per_sm = value < 0 ? 0 : value; break;
    case D3_OPT_ATM_SURROGATE: o.atm_surrogate = value != 0; break;
    case D3_OPT_ATM_SCHEDULE:
        if (value != 0 && value != 1) {
            set_error("D3_OPT_ATM_SCHEDULE takes 0 (block pairs) or 1 (mirror-symmetric)");
            return 1;
        }
        o.atm_schedule = value;
        break;
    case D3_OPT_ATM_LIST_CAPACITY: o.atm_list_capacity = value < 0 ? 0 : value; break;
    case D3_OPT_ATMB_WARPS:
        if (value < 0 || value > 12) {
            set_error("D3_OPT_ATMB_WARPS takes 0 (automatic) or 2..12");
            return 1;
        }
        o.atmb_warps = value;
        break;
    case D3_OPT_ATMB_LIST_CAPACITY: o.atmb_mcap = value < 0 ? 0 : value; break;
    case D3_OPT_ATMB_SPLIT: o.atmb_split = value < 0 ? 0 : value; break;
    case D3_OPT_ATMB_FINE_SKIP: o.atmb_fine_skip = value != 0; break;
    case D3_OPT_PAIR_KERNEL:
        if (value != 0 && value != 1) {
            set_error("D3_OPT_PAIR_KERNEL takes 0 (atom groups) or 1 (one warp per atom)");
            return 1;
        }
        o.pair_kernel = value;
        break;
    case D3_OPT_PRECISION:
        if (value != 0 && value != 1) {
            set_error("D3_OPT_PRECISION takes 0 (FP64) or 1 (FP32 pair/triplet arithmetic)");
            return 1;
        }
        o.precision = value;
        break;
    default: set_error("unknown option " + std::to_string(option)); return 1;
    }
    try {
        d3::engine_set_options(H(handle)->engine, o);
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
    return 0;
}

d3_handle_t *d3_init_batch(const uint16_t *elements, uint64_t n_elements, uint64_t max_structures,
                           uint64_t max_total_atoms, double rc, double rc_cn, double rc_atm, int damping_type,
                           int functional_type, int table) {
    std::string err;
    d3::Engine *e = d3::engine_create(elements, n_elements, max_total_atoms, rc, rc_cn, rc_atm, rc_atm > 0.0,
                                      damping_type, functional_type, table == D3_TABLE_7REF, err, max_structures);
    if (!e) {
        set_error(err);
        return nullptr;
    }
    Handle *h = new Handle();
    h->engine = e;
    return reinterpret_cast<d3_handle_t *>(h);
}

int d3_set_batch_f64(d3_handle_t *handle, uint64_t n_structures, const uint64_t *atom_counts, const double *coords,
                     const uint16_t *elements, const double *cells) {
    if (!handle || !atom_counts || !coords || !elements || !cells) {
        set_error("NULL argument in d3_set_batch_f64");
        return 1;
    }
    uint64_t n = 0;
    for (uint64_t k = 0; k < n_structures; ++k) n += atom_counts[k];
    std::vector<double> b(3 * n), cb(9 * n_structures);
    std::vector<float> cf(9 * n_structures);
    const float a2b = 1.0f / 0.52917726f;
    for (uint64_t i = 0; i < 3 * n; ++i) b[i] = coords[i] * d3::ANG2BOHR;
    for (uint64_t i = 0; i < 9 * n_structures; ++i) {
        cb[i] = cells[i] * d3::ANG2BOHR;
        cf[i] = (float)cells[i] * a2b;
    }
    std::string err;
    if (d3::engine_set_batch(H(handle)->engine, n_structures, atom_counts, b.data(), elements, cb.data(), cf.data(),
                             err)) {
        set_error(err);
        return 1;
    }
    return 0;
}

uint16_t d3_compute_batch_f64(d3_handle_t *handle, double *energies, double *forces, double *stresses) {
    if (!handle) {
        set_error("handle is NULL in d3_compute_batch_f64");
        return 1;
    }
    uint16_t st = d3::engine_compute(H(handle)->engine, energies, forces, stresses, nullptr, true);
    if (st & (d3::ST_CUDA_ERROR | d3::ST_NOT_READY))
        set_error(st & d3::ST_NOT_READY ? "atoms or cell not set" : "CUDA error during compute");
    return st;
}

int d3_set_positions_device(d3_handle_t *handle, const double *coords_dev, void *cuda_stream) {
    if (!handle || !coords_dev) {
        set_error("NULL argument in d3_set_positions_device");
        return 1;
    }
    return d3::engine_set_positions_device(H(handle)->engine, coords_dev, (cudaStream_t)cuda_stream);
}

int d3_fetch_results(d3_handle_t *handle, double *energies, double *forces, double *stresses) {
    if (!handle) {
        set_error("handle is NULL in d3_fetch_results");
        return 1;
    }
    try {
        d3::engine_fetch_results(H(handle)->engine, energies, forces, stresses);
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
    return 0;
}

int d3_num_structures(d3_handle_t *handle) { return handle ? d3::engine_num_structures(H(handle)->engine) : -1; }

int d3_set_functional_params(d3_handle_t *handle, double s6, double s8, double p1, double p2) {
    if (!handle) {
        set_error("handle is NULL in d3_set_functional_params");
        return 1;
    }
    d3::engine_set_functional_params(H(handle)->engine, d3::FuncParams{s6, s8, p1, p2});
    return 0;
}

uint16_t d3_compute_async(d3_handle_t *handle, void *cuda_stream) {
    if (!handle) {
        set_error("handle is NULL in d3_compute_async");
        return 1;
    }
    return d3::engine_compute(H(handle)->engine, nullptr, nullptr, nullptr, (cudaStream_t)cuda_stream, false);
}

const double *d3_device_results(d3_handle_t *handle) {
    return handle ? d3::engine_device_results(H(handle)->engine) : nullptr;
}

uint16_t d3_fetch_status(d3_handle_t *handle) {
    if (!handle) {
        set_error("handle is NULL in d3_fetch_status");
        return 1;
    }
    try {
        return d3::engine_fetch_status(H(handle)->engine);
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return d3::ST_CUDA_ERROR;
    }
}

int64_t d3_atm_list_capacity(d3_handle_t *handle) { return handle ? d3::engine_atm_capacity(H(handle)->engine) : -1; }

const char *d3_last_error(void) { return g_last_error.c_str(); }

int d3_pass_times(d3_handle_t *handle, float *ms, int cap, uint64_t *counters) {
    if (!handle) return -1;
    try {
        return d3::engine_pass_times(H(handle)->engine, ms, cap, reinterpret_cast<unsigned long long *>(counters));
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return -1;
    }
}

int d3_launches_per_eval(d3_handle_t *handle) {
    return handle ? d3::engine_launches_per_eval(H(handle)->engine) : -1;
}

double d3_peak_probe(int fp64) {
    try {
        return d3::engine_peak_probe(fp64);
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return -1.0;
    }
}

int d3_selftest_math(double *max_rel_err) {
    try {
        return d3::engine_selftest_math(max_rel_err);
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
}

int d3_debug_atom_arrays(d3_handle_t *handle, double *cn, double *dedcn, double *energy_atoms) {
    if (!handle) return 1;
    try {
        return d3::engine_debug_atom_arrays(H(handle)->engine, cn, dedcn, energy_atoms);
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
}

int d3_debug_pass_terms(d3_handle_t *handle, double *terms) {
    if (!handle || !terms) return 1;
    try {
        return d3::engine_debug_pass_terms(H(handle)->engine, terms);
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
}

int64_t d3_debug_atm_pairs(d3_handle_t *handle, int64_t *rows, int64_t cap) {
    if (!handle) return -1;
    try {
        return d3::engine_debug_atm_pairs(H(handle)->engine, rows, cap);
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return -1;
    }
}

int d3_debug_bins(d3_handle_t *handle, int64_t *wrap_shift, int64_t *bin_index, int *num_bins) {
    if (!handle) return 1;
    try {
        return d3::engine_debug_bins(H(handle)->engine, wrap_shift, bin_index, num_bins);
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
}

// ---- learned ATM surrogate ---------------------------------------------------------
int d3_set_surrogate(d3_handle_t *handle, const int *channel_z, int n_channels, int members, const float *params,
                     const float *mean, const float *inv_std, const float *e_shift, float e_scale) {
    if (!handle || !channel_z || !params || !mean || !inv_std || !e_shift || n_channels < 1 || members < 1) {
        set_error("invalid argument in d3_set_surrogate");
        return 1;
    }
    try {
        const d3mlp::Layout L = d3mlp::make_layout(n_channels);
        d3::SurrogateModel m;
        m.channel_z.assign(channel_z, channel_z + n_channels);
        m.members = members;
        m.master.assign(params, params + (size_t)members * L.nparam);
        const size_t nf = (size_t)n_channels * d3mlp::NRBF;
        m.mean.assign(mean, mean + nf);
        m.inv_std.assign(inv_std, inv_std + nf);
        m.e_shift.assign(e_shift, e_shift + n_channels);
        m.e_scale = e_scale;
        std::string err;
        if (d3::engine_set_surrogate(H(handle)->engine, m, err)) {
            set_error(err);
            return 1;
        }
        return 0;
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
}

int d3_set_surrogate_threshold(d3_handle_t *handle, double std_threshold_ev) {
    if (!handle || !(std_threshold_ev >= 0.0)) {
        set_error("invalid argument in d3_set_surrogate_threshold");
        return 1;
    }
    d3::engine_set_surrogate_threshold(H(handle)->engine, std_threshold_ev);
    return 0;
}

int d3_surrogate_flagged(d3_handle_t *handle) {
    if (!handle) return -1;
    try {
        return d3::engine_surrogate_flagged(H(handle)->engine);
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return -1;
    }
}

int d3_surrogate_descriptors(d3_handle_t *handle, const int *channel_z, int n_channels, float *G_dev,
                             int *center_dev, double *e_atm_dev, void *cuda_stream) {
    if (!handle || !channel_z) {
        set_error("invalid argument in d3_surrogate_descriptors");
        return 1;
    }
    std::string err;
    if (d3::engine_surrogate_descriptors(H(handle)->engine, channel_z, n_channels, G_dev, center_dev, e_atm_dev,
                                         (cudaStream_t)cuda_stream, err)) {
        set_error(err);
        return 1;
    }
    return 0;
}

int d3_mlp_layout(int n_channels, uint64_t *out) {
    try {
        const d3mlp::Layout L = d3mlp::make_layout(n_channels);
        const uint64_t v[12] = {(uint64_t)L.in_dim, (uint64_t)L.in_pad, L.oW1, L.ob1, L.oW2, L.ob2,
                                L.oW3, L.ob3, L.ow4, L.ob4, L.nparam, L.packed};
        for (int k = 0; k < 12; ++k) out[k] = v[k];
        return 0;
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
}

uint64_t d3_mlp_acts_elems(int n_channels, int B) {
    try {
        return d3mlp::acts_elems(d3mlp::make_layout(n_channels), B);
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 0;
    }
}

static d3mlp::Net mlp_net(int n_channels, int members, const float *params, const uint16_t *packed, const float *mean,
                          const float *inv_std) {
    d3mlp::Net net;
    net.L = d3mlp::make_layout(n_channels);
    net.members = members;
    net.master = params;
    net.packed = packed;
    net.mean = mean;
    net.inv_std = inv_std;
    return net;
}

static int sm_count() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

int d3_mlp_pack(int n_channels, int members, const float *params_dev, uint16_t *packed_dev, void *cuda_stream) {
    try {
        d3mlp::pack(d3mlp::make_layout(n_channels), members, params_dev, packed_dev, (cudaStream_t)cuda_stream);
        return 0;
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
}

int d3_mlp_forward(int n_channels, int members, const float *params_dev, const uint16_t *packed_dev,
                   const float *mean_dev, const float *inv_std_dev, const float *G_dev, const int *center_dev,
                   int rows, float *E_dev, float *dX_dev, void *cuda_stream) {
    try {
        d3mlp::infer(mlp_net(n_channels, members, params_dev, packed_dev, mean_dev, inv_std_dev), G_dev, center_dev,
                     rows, E_dev, dX_dev, sm_count(), (cudaStream_t)cuda_stream);
        return 0;
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
}

int d3_mlp_train_batch(int n_channels, int members, const float *params_dev, const uint16_t *packed_dev,
                       const float *mean_dev, const float *inv_std_dev, const float *G_dev, const int *center_dev,
                       const float *target_dev, const int *idx_dev, int B, float *E_dev, uint16_t *acts_dev,
                       float *partial_dev, float *loss_dev, void *cuda_stream) {
    try {
        const d3mlp::Net net = mlp_net(n_channels, members, params_dev, packed_dev, mean_dev, inv_std_dev);
        d3mlp::train_fwdbwd(net, G_dev, center_dev, target_dev, idx_dev, B, E_dev, acts_dev, partial_dev, loss_dev,
                            (cudaStream_t)cuda_stream);
        d3mlp::wgrad(net, acts_dev, B, partial_dev, (cudaStream_t)cuda_stream);
        return 0;
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
}

int d3_mlp_adam(int n_channels, int members, float *params_dev, uint16_t *packed_dev, float *m1_dev, float *m2_dev,
                const float *partial_dev, int splits, float lr, float beta1, float beta2, float eps,
                float weight_decay, int step, void *cuda_stream) {
    try {
        d3mlp::adam(d3mlp::make_layout(n_channels), members, params_dev, packed_dev, m1_dev, m2_dev, partial_dev,
                    splits, lr, beta1, beta2, eps, weight_decay, step, (cudaStream_t)cuda_stream);
        return 0;
    } catch (const std::exception &ex) {
        set_error(ex.what());
        return 1;
    }
}

// ---- sharded evaluation ---------------------------------------------------------------
uint64_t d3_shard_length(d3_handle_t *handle) { return handle ? d3::engine_num_atoms(H(handle)->engine) : 0; }

uint16_t d3_shard_begin(d3_handle_t *handle, int rank, int world, double *dedcn_dev, void *cuda_stream) {
    if (!handle) {
        set_error("handle is NULL in d3_shard_begin");
        return 1;
    }
    std::string err;
    const uint16_t st = d3::engine_shard_begin(H(handle)->engine, rank, world, dedcn_dev, (cudaStream_t)cuda_stream, err);
    if (!err.empty()) set_error(err);
    return st;
}

uint16_t d3_shard_end(d3_handle_t *handle, const double *dedcn_dev, double *results_dev, void *cuda_stream) {
    if (!handle) {
        set_error("handle is NULL in d3_shard_end");
        return 1;
    }
    std::string err;
    const uint16_t st = d3::engine_shard_end(H(handle)->engine, dedcn_dev, results_dev, (cudaStream_t)cuda_stream, err);
    if (!err.empty()) set_error(err);
    return st;
}

int d3_copy_results_device(d3_handle_t *handle, double *results_dev, void *cuda_stream) {
    if (!handle || !results_dev) {
        set_error("NULL argument in d3_copy_results_device");
        return 1;
    }
    const double *src = d3::engine_device_results(H(handle)->engine);
    const size_t S = (size_t)d3::engine_num_structures(H(handle)->engine), n = d3::engine_num_atoms(H(handle)->engine);
    const cudaError_t e = cudaMemcpyAsync(results_dev, src, sizeof(double) * (10 * S + 3 * n), cudaMemcpyDeviceToDevice,
                                          (cudaStream_t)cuda_stream);
    if (e != cudaSuccess) {
        set_error(std::string("d3_copy_results_device: ") + cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

} // extern "C"

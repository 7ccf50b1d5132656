// Coordination numbers without any device allocation.
//
// d3_coordination_numbers_noalloc() computes the D3 coordination numbers (the first
// pass of the dispersion evaluation) for one periodic structure. Unlike the handle API
// it never allocates device memory: its only scratch is the file-scope array below,
// sized for D3_NOALLOC_MAX_ATOMS atoms. It exists for callers that must not allocate
// at the point where they call us -- for example a molecular-dynamics engine plugin
// invoked inside its time-step loop, where cudaMalloc would synchronise the device and
// stall the engine's other streams, or an application that has handed all device memory
// to its own pool allocator and forbids allocations outside it.
//
// Rules for callers:
//   * the first call on each device performs a one-time set-up on that device (it looks
//     up the scratch array's device address and loads the covalent-radius table into
//     constant memory); make that first call before any stream capture;
//   * every call shares the one scratch array of the device, which keeps the previous
//     call's contents; calls whose work overlaps on the GPU (different streams, or
//     different host threads) race on it and must be serialised by the caller;
//   * the device holds the scratch array (256 KiB) until the process exits;
//   * the set-up is cached per device and does not survive cudaDeviceReset: after a reset
//     in the same process this entry point must not be called again;
//   * images: every periodic image within the cutoff of the WRAPPED positions is used.
//     The handle API instead reproduces the reference's image box over the positions as
//     given (unwrapped); the two agree when the atoms are given inside the cell, and can
//     differ for atoms given outside it. The smooth-cutoff CN option has no counterpart.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/d3.h"
#include "d3_geometry.h"
#include "d3_synth_params.h"

namespace d3 {
void record_error(const std::string &msg);
}

namespace {

constexpr int MAX_DEVICES = 64;
constexpr double ANG2BOHR_NA = 1.0 / 0.52917726;

// Scratch of the no-allocation path: per atom, the position wrapped into the cell
// (bohr) and the covalent radius. Each call writes every slot it reads first.
static __device__ __align__(256) double g_d3_noalloc_scratch[4 * D3_NOALLOC_MAX_ATOMS];

// K2-scaled covalent radii (bohr) by atomic number, for the 5- and 7-reference layouts
static __constant__ double c_noalloc_rcov[2][128];

struct NoallocGeom {
    double h[9], inv[9];
    int half[3];
    double rcn2;
};

__global__ void k_noalloc_wrap(const double *coords, const uint16_t *elements, int n, NoallocGeom g, int table,
                               double *scratch) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = coords[3 * i] * ANG2BOHR_NA, y = coords[3 * i + 1] * ANG2BOHR_NA, z = coords[3 * i + 2] * ANG2BOHR_NA;
    double s[3];
    for (int k = 0; k < 3; ++k) s[k] = floor(x * g.inv[k] + y * g.inv[3 + k] + z * g.inv[6 + k]);
    double *o = scratch + 4 * (size_t)i;
    o[0] = x - (s[0] * g.h[0] + s[1] * g.h[3] + s[2] * g.h[6]);
    o[1] = y - (s[0] * g.h[1] + s[1] * g.h[4] + s[2] * g.h[7]);
    o[2] = z - (s[0] * g.h[2] + s[1] * g.h[5] + s[2] * g.h[8]);
    const int Z = elements[i];
    o[3] = (Z < 128) ? c_noalloc_rcov[table][Z] : -1.0;
}

__global__ void k_noalloc_cn(int n, NoallocGeom g, const double *scratch, double *cn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *xi = scratch + 4 * (size_t)i;
    if (!(xi[3] > 0.0)) {
        cn[i] = NAN; // element outside the parameter table
        return;
    }
    double acc = 0.0;
    for (int j = 0; j < n; ++j) {
        const double *xj = scratch + 4 * (size_t)j;
        if (!(xj[3] > 0.0)) continue; // an atom outside the table contributes nothing
        const double rsum = xi[3] + xj[3];
        for (int tz = -g.half[2]; tz <= g.half[2]; ++tz)
            for (int ty = -g.half[1]; ty <= g.half[1]; ++ty)
                for (int tx = -g.half[0]; tx <= g.half[0]; ++tx) {
                    const double dx = xi[0] - (xj[0] + tx * g.h[0] + ty * g.h[3] + tz * g.h[6]);
                    const double dy = xi[1] - (xj[1] + tx * g.h[1] + ty * g.h[4] + tz * g.h[7]);
                    const double dz = xi[2] - (xj[2] + tx * g.h[2] + ty * g.h[5] + tz * g.h[8]);
                    const double d2 = dx * dx + dy * dy + dz * dz;
                    if (d2 <= g.rcn2 && d2 > 0.0) acc += 1.0 / (1.0 + exp(-16.0 * (rsum / sqrt(d2) - 1.0)));
                }
    }
    cn[i] = acc;
}

std::mutex g_setup_mutex;
double *g_scratch_ptr[MAX_DEVICES] = {};

int fail(const std::string &m) {
    d3::record_error(m);
    fprintf(stderr, "Error: %s\n", m.c_str());
    return 1;
}

// once per device, with that device current
int setup_device(int dev, double **out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_ptr[dev]) {
        *out = g_scratch_ptr[dev];
        return 0;
    }
    double *ptr = nullptr;
    cudaError_t err = cudaGetSymbolAddress((void **)&ptr, g_d3_noalloc_scratch);
    if (err != cudaSuccess || !ptr)
        return fail(std::string("d3_coordination_numbers_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(err));
    double rc[2][128];
    for (int t = 0; t < 2; ++t) {
        const int ne = t ? D3_NE_EXTENDED : D3_NE_ORIGINAL;
        const int nr = t ? D3_NREF_EXTENDED : D3_NREF_ORIGINAL;
        // the generator fills whole tables; only the covalent radii are kept here
        static float c6[D3_NE_EXTENDED * D3_NE_EXTENDED * D3_NREF_EXTENDED * D3_NREF_EXTENDED * 3];
        float r0[D3_NE_EXTENDED * D3_NE_EXTENDED], rcov[D3_NE_EXTENDED], r2r4[D3_NE_EXTENDED];
        d3_synth_fill(D3_SYNTH_SEED, ne, nr, t, c6, r0, rcov, r2r4);
        for (int Z = 0; Z < 128; ++Z) {
            const int slot = t ? Z - 1 : Z;
            rc[t][Z] = (slot >= 0 && slot < ne && Z < 118) ? (double)rcov[slot] : -1.0;
        }
    }
    err = cudaMemcpyToSymbol(c_noalloc_rcov, rc, sizeof(rc));
    if (err != cudaSuccess)
        return fail(std::string("d3_coordination_numbers_noalloc: loading the radius table failed: ") +
                    cudaGetErrorString(err));
    g_scratch_ptr[dev] = ptr;
    *out = ptr;
    return 0;
}

} // namespace

extern "C" int d3_coordination_numbers_noalloc(const double *coords, const uint16_t *elements, uint64_t num_atoms,
                                               const double cell[9], double cn_cutoff, int table, double *cn,
                                               void *cuda_stream) {
    if (!coords || !elements || !cell || !cn) return fail("d3_coordination_numbers_noalloc: NULL argument");
    if (num_atoms == 0) return fail("d3_coordination_numbers_noalloc: no atoms");
    if (num_atoms > (uint64_t)D3_NOALLOC_MAX_ATOMS)
        return fail("d3_coordination_numbers_noalloc: " + std::to_string(num_atoms) + " atoms exceed the maximum of " +
                    std::to_string(D3_NOALLOC_MAX_ATOMS) + "; use the handle API for larger systems");
    if (table != D3_TABLE_5REF && table != D3_TABLE_7REF) return fail("d3_coordination_numbers_noalloc: unknown table");
    if (!(cn_cutoff > 0.0) || !std::isfinite(cn_cutoff)) return fail("d3_coordination_numbers_noalloc: bad cutoff");
    double hb[9];
    for (int k = 0; k < 9; ++k) {
        if (!std::isfinite(cell[k])) return fail("d3_coordination_numbers_noalloc: non-finite cell");
        hb[k] = cell[k] * ANG2BOHR_NA;
    }
    const d3::CellGeom geom = d3::make_geom(hb);
    if (!(std::fabs(geom.volume) > 1e-12)) return fail("d3_coordination_numbers_noalloc: degenerate cell");
    NoallocGeom g;
    for (int k = 0; k < 9; ++k) {
        g.h[k] = geom.h[k];
        g.inv[k] = geom.inv[k];
    }
    // wrapped atoms lie inside the cell, so images up to floor(rc / height) + 1 cells
    // away cover every pair within the cutoff. The kernel visits every image of every
    // pair, so the work is bounded before launch: at most D3_NOALLOC_MAX_IMAGES images
    // and n^2 x images <= 2^36 pair-image tests (about a second on one GPU)
    double images = 1.0;
    for (int k = 0; k < 3; ++k) {
        const double reach = std::floor(cn_cutoff / geom.height[k]) + 1.0;
        if (!(reach <= 64.0)) return fail("d3_coordination_numbers_noalloc: cell too thin for the cutoff");
        g.half[k] = (int)reach;
        images *= 2.0 * reach + 1.0;
    }
    if (images > (double)D3_NOALLOC_MAX_IMAGES || (double)num_atoms * (double)num_atoms * images > 68719476736.0)
        return fail("d3_coordination_numbers_noalloc: " + std::to_string((long long)images) + " periodic images for " +
                    std::to_string(num_atoms) + " atoms exceed the work bound of this entry point (at most " +
                    std::to_string(D3_NOALLOC_MAX_IMAGES) +
                    " images and 2^36 pair-image tests); use the handle API, whose cell list scales");
    g.rcn2 = cn_cutoff * cn_cutoff;
    // arguments are valid: only now touch the device
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return fail(std::string("d3_coordination_numbers_noalloc: no usable device: ") + cudaGetErrorString(err));
    double *scratch = nullptr;
    if (setup_device(dev, &scratch)) return 1;
    // an error left by earlier work of this thread would otherwise be reported as ours
    err = cudaGetLastError();
    if (err != cudaSuccess)
        return fail(std::string("d3_coordination_numbers_noalloc: CUDA error pending from earlier work: ") +
                    cudaGetErrorString(err));
    cudaStream_t s = (cudaStream_t)cuda_stream;
    const int n = (int)num_atoms, T = 128, blocks = (n + T - 1) / T;
    k_noalloc_wrap<<<blocks, T, 0, s>>>(coords, elements, n, g, table, scratch);
    k_noalloc_cn<<<blocks, T, 0, s>>>(n, g, scratch, cn);
    err = cudaGetLastError();
    if (err != cudaSuccess)
        return fail(std::string("d3_coordination_numbers_noalloc: launch failed: ") + cudaGetErrorString(err));
    return 0;
}

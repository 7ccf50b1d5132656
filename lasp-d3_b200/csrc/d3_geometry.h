// Host-side cell geometry for the D3 engine: cell inverse, perpendicular heights,
// the reference's image box and workload decision, bin grid choice and the
// row-compressed bin stencil used by every pair traversal on the device.
#pragma once
#include <cstdint>
#include <vector>

namespace d3 {

// One stencil row: bin offsets (dxlo..dxhi, dy, dz) relative to the home bin.
// Along x the neighbour bins of a row are contiguous in the binned atom order
// (x is the fastest bin index), so a row expands to a few contiguous atom ranges.
struct StencilRow {
    int dy, dz, dxlo, dxhi;
};

struct CellGeom {
    double h[9];     // rows = lattice vectors, bohr
    double inv[9];   // inverse of h (row-vector convention: frac = x * inv)
    double height[3];
    double volume;   // signed determinant, as the reference uses it
};

CellGeom make_geom(const double h[9]);

// Reference image box (calculate_cell_repeats, src/d3_buffer.cu:63-84) and workload
// decision (set_cell, src/d3_buffer.cu:431-477), from the float cell in bohr with the
// reference's float-operand inverse. Returns true for ALL_ITERATE.
bool reference_box(const float cell_f[9], float rc, float rc_cn, int64_t mcb[3]);

// Bins per direction for a target bin width, capped so the bin count stays bounded.
void choose_bins(const CellGeom &g, double target_width, int64_t max_bins, int nb[3]);

// All bin offsets whose closest possible point pair is within r (+ margin),
// compressed into x-rows. Exact convex-QP distance between parallelepiped bins.
std::vector<StencilRow> build_stencil(const CellGeom &g, const int nb[3], double r);

// Stencil of a block of gy x gz bin rows (offsets relative to the block's first row): for
// every row offset the union of the x ranges its member rows need (the block's own x
// extent is added at run time). Each row offset appears once.
std::vector<StencilRow> merge_block_stencil(const std::vector<StencilRow> &st, int gy, int gz);

} // namespace d3

#include <map>
// Host-side cell geometry (see d3_geometry.h).
#include "d3_geometry.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <map>

namespace d3 {

CellGeom make_geom(const double h[9]) {
    CellGeom g;
    for (int i = 0; i < 9; ++i) g.h[i] = h[i];
    const double *m = h;
    double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                 m[2] * (m[3] * m[7] - m[4] * m[6]);
    g.volume = det;
    double id = 1.0 / det;
    g.inv[0] = (m[4] * m[8] - m[5] * m[7]) * id;
    g.inv[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    g.inv[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    g.inv[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    g.inv[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    g.inv[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    g.inv[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    g.inv[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    g.inv[8] = (m[0] * m[4] - m[1] * m[3]) * id;
    // perpendicular height along lattice direction k = 1 / |column k of inv|
    for (int k = 0; k < 3; ++k) {
        double s = g.inv[0 * 3 + k] * g.inv[0 * 3 + k] + g.inv[1 * 3 + k] * g.inv[1 * 3 + k] +
                   g.inv[2 * 3 + k] * g.inv[2 * 3 + k];
        g.height[k] = 1.0 / std::sqrt(s);
    }
    return g;
}

bool reference_box(const float cf[9], float rc, float rc_cn, int64_t mcb[3]) {
    // matrix_inverse<float, double>: products and differences in float, widened
    float m[3][3];
    for (int i = 0; i < 9; ++i) m[i / 3][i % 3] = cf[i];
    float det_f = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                  m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    volatile float t[9];
    t[0] = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    t[1] = m[0][2] * m[2][1] - m[0][1] * m[2][2];
    t[2] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
    t[3] = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    t[4] = m[0][0] * m[2][2] - m[0][2] * m[2][0];
    t[5] = m[0][2] * m[1][0] - m[0][0] * m[1][2];
    t[6] = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    t[7] = m[0][1] * m[2][0] - m[0][0] * m[2][1];
    t[8] = m[0][0] * m[1][1] - m[0][1] * m[1][0];
    double id = 1.0 / (double)det_f;
    double inv[3][3];
    for (int i = 0; i < 9; ++i) inv[i / 3][i % 3] = (double)t[i] * id;
    double larger = rc_cn > rc ? rc_cn : rc;
    bool all_iterate = false;
    for (int i = 0; i < 3; ++i) {
        double vn = std::sqrt(inv[i][0] * inv[i][0] + inv[i][1] * inv[i][1] + inv[i][2] * inv[i][2]);
        uint64_t ng = (uint64_t)std::floor((1.0 / vn) / larger);
        if (ng <= 2) all_iterate = true;
    }
    float cut = (float)larger;
    for (int i = 0; i < 3; ++i) {
        double nrm = std::sqrt(inv[0][i] * inv[0][i] + inv[1][i] * inv[1][i] + inv[2][i] * inv[2][i]);
        mcb[i] = ((int64_t)(int)(cut * nrm) + 1) * 2 + 1;
    }
    return all_iterate;
}

void choose_bins(const CellGeom &g, double target, int64_t max_bins, int nb[3]) {
    for (int k = 0; k < 3; ++k) nb[k] = std::max(1, (int)std::floor(g.height[k] / target));
    while ((int64_t)nb[0] * nb[1] * nb[2] > max_bins) {
        int k = 0;
        for (int j = 1; j < 3; ++j)
            if (nb[j] > nb[k]) k = j;
        nb[k] = std::max(1, nb[k] / 2);
    }
}

namespace {

// min over u in [-1,1]^3 of (d+u)^T G (d+u): exact, by enumerating which coordinates
// sit on a bound (27 active sets) and solving the free ones.
double min_dist2(const double G[3][3], const double d[3]) {
    double best = std::numeric_limits<double>::infinity();
    for (int code = 0; code < 27; ++code) {
        int st[3] = {code % 3, (code / 3) % 3, code / 9}; // 0 free, 1 lower, 2 upper
        double v[3];
        int fr[3], nf = 0;
        for (int k = 0; k < 3; ++k) {
            if (st[k] == 1)
                v[k] = d[k] - 1.0;
            else if (st[k] == 2)
                v[k] = d[k] + 1.0;
            else {
                v[k] = 0.0;
                fr[nf++] = k;
            }
        }
        // solve G_ff x_f = -G_fc v_c  (x_f = d_f + u_f)
        double rhs[3], A[3][3];
        for (int a = 0; a < nf; ++a) {
            rhs[a] = 0;
            for (int k = 0; k < 3; ++k)
                if (st[k] != 0) rhs[a] -= G[fr[a]][k] * v[k];
            for (int b = 0; b < nf; ++b) A[a][b] = G[fr[a]][fr[b]];
        }
        double x[3] = {0, 0, 0};
        bool ok = true;
        if (nf == 1) {
            x[0] = rhs[0] / A[0][0];
        } else if (nf == 2) {
            double det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
            if (std::fabs(det) < 1e-300) ok = false;
            else {
                x[0] = (rhs[0] * A[1][1] - A[0][1] * rhs[1]) / det;
                x[1] = (A[0][0] * rhs[1] - rhs[0] * A[1][0]) / det;
            }
        } else if (nf == 3) {
            x[0] = x[1] = x[2] = 0.0; // unconstrained minimum of a PD form is the origin
        }
        if (!ok) continue;
        for (int a = 0; a < nf; ++a) {
            double u = x[a] - d[fr[a]];
            if (u < -1.0 || u > 1.0) {
                ok = false;
                break;
            }
            v[fr[a]] = x[a];
        }
        if (!ok) continue;
        double q = 0;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) q += v[a] * G[a][b] * v[b];
        best = std::min(best, q);
    }
    return best;
}

} // namespace

std::vector<StencilRow> build_stencil(const CellGeom &g, const int nb[3], double r) {
    double M[3][3];
    for (int k = 0; k < 3; ++k)
        for (int c = 0; c < 3; ++c) M[k][c] = g.h[k * 3 + c] / nb[k];
    double G[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) G[a][b] = M[a][0] * M[b][0] + M[a][1] * M[b][1] + M[a][2] * M[b][2];
    const double rr = r * (1.0 + 1e-9) + 1e-6;
    const double r2 = rr * rr;
    int ext[3];
    for (int k = 0; k < 3; ++k) ext[k] = (int)std::ceil(rr / (g.height[k] / nb[k])) + 1;
    std::vector<StencilRow> rows;
    for (int dz = -ext[2]; dz <= ext[2]; ++dz)
        for (int dy = -ext[1]; dy <= ext[1]; ++dy) {
            int lo = 1, hi = 0;
            for (int dx = -ext[0]; dx <= ext[0]; ++dx) {
                double d[3] = {(double)dx, (double)dy, (double)dz};
                if (min_dist2(G, d) <= r2) {
                    if (lo > hi) lo = hi = dx;
                    else hi = dx;
                }
            }
            if (lo <= hi) rows.push_back({dy, dz, lo, hi});
        }
    return rows;
}

std::vector<StencilRow> merge_block_stencil(const std::vector<StencilRow> &st, int gy, int gz) {
    std::map<std::pair<int, int>, std::pair<int, int>> m; // (dz, dy) -> (lo, hi)
    for (int oz = 0; oz < gz; ++oz)
        for (int oy = 0; oy < gy; ++oy)
            for (const StencilRow &r : st) {
                const auto key = std::make_pair(r.dz + oz, r.dy + oy);
                auto it = m.find(key);
                if (it == m.end())
                    m.emplace(key, std::make_pair(r.dxlo, r.dxhi));
                else {
                    it->second.first = std::min(it->second.first, r.dxlo);
                    it->second.second = std::max(it->second.second, r.dxhi);
                }
            }
    std::vector<StencilRow> out;
    out.reserve(m.size());
    for (const auto &kv : m) out.push_back({kv.first.second, kv.first.first, kv.second.first, kv.second.second});
    return out;
}

} // namespace d3

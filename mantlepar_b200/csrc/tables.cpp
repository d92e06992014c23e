// Host construction of the per-mesh stage tables (see tables.hpp).
//
// The arithmetic follows the reference's setup code so that the tables equal
// the reference's per-cell tables up to the rounding of vertex coordinates:
//   Gauss-Legendre rule (PetscDTGaussQuadrature, src/core/integral.cpp:7-20)
//   bilinear maps and Jacobian (src/core/integral.cpp:91-121)
//   stencil centre, moments, inverse, smoothness (tensorstencilpoly.cpp:146-231,318-368,383-398)
//   limiter points (state_reconstruction.cpp:152-168)
//   normal-line samples (diffusiveflux.cpp:23-84,255-334; 4 samples, extent 0.9)
#include "tables.hpp"
#include "geometry.hpp"

#include "../../include/mantlepar/mp.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <vector>

namespace mp {
namespace {

using namespace geo;

struct Grid {
    double dx, dy;
    V2 vert(int I, int J) const { return V2{(double)I * dx, (double)J * dy}; }
    Quad cell(int I, int J) const { return Quad{{vert(I, J), vert(I + 1, J), vert(I + 1, J + 1), vert(I, J + 1)}}; }
};

// Normal-line samples of a uniform rectangular mesh (diffusiveflux.cpp:255-334,
// numberOfSamples 4, extentFraction 0.9): the available ray distance across
// an edge is the cell size normal to it.
void fill_diffusion(StageHot& t, double dx, double dy, double h, const std::vector<double>& gw) {
    typedef long double ld;
    const int N = 4;
    const ld frac = 0.9L;
    derivative_weights(N, true, t.dif_c_int);
    derivative_weights(N + 1, false, t.dif_c_bnd);
    const double size[2] = {dy, dx};      // across horizontal / vertical edges
    const double len[2] = {dx, dy};
    for (int o = 0; o < 2; ++o) {
        t.dif_ds[o][0] = (double)(frac * size[o] * (2.0L / (N - 1)));
        t.dif_ds[o][1] = (double)(frac * size[o] * (1.0L / N));
        for (int q = 0; q < kNQ; ++q) t.dif_w[o][q] = (double)((ld)len[o] * gw[q] / 2);
    }
    const double Y = t.Y, X = t.X;
    // Interior: offsets (k - 1.5) ds along the edge normal, which points from
    // the left cell into the right one: down for horizontal edges (left cell
    // above), +x for vertical edges (left cell at smaller x).
    for (int k = 0; k < N; ++k) {
        const ld off = (ld)k - (N - 1) / 2.0L;
        const double sh = (double)(off * t.dif_ds[0][0] / h), sv = (double)(off * t.dif_ds[1][0] / h);
        t.dif_pos_int[0][k] = k < N / 2 ? -Y - sh : Y - sh;
        t.dif_pos_int[1][k] = k < N / 2 ? X + sv : -X + sv;
    }
    // Walls: interior samples at (N - k) ds inside, farthest first.
    for (int k = 0; k < N; ++k) {
        const double dh = (double)((ld)(N - k) * t.dif_ds[0][1] / h), dv = (double)((ld)(N - k) * t.dif_ds[1][1] / h);
        t.dif_pos_bnd[0][k] = -Y + dh;   // bottom wall: the cell above it
        t.dif_pos_bnd[1][k] = Y - dh;    // top wall: the cell below it
        t.dif_pos_bnd[2][k] = -X + dv;   // left wall
        t.dif_pos_bnd[3][k] = X - dv;    // right wall
    }
}

}  // namespace

int build_stage_tables(int nx, int ny, double x0, double x1, double y0, double y1, StageTables& t) {
    if (nx < 2 || ny < 2) return MP_ERR_ARG_SIZ;
    const double dx = (x1 - x0) / (double)nx, dy = (y1 - y0) / (double)ny;
    if (!(dx > 0) || !(dy > 0) || !std::isfinite(dx) || !std::isfinite(dy)) return MP_ERR_ARG_OUTOFRANGE;
    const Grid g{dx, dy};
    const Quad target = g.cell(0, 0);
    std::vector<double> p1, w1, gp, gw;
    gauss_legendre(1, p1, w1);
    gauss_legendre(kNQ, gp, gw);
    const double area = cell_integral(target, p1, w1, [](V2) { return 1.0; });
    const double h = std::sqrt(area);
    const V2 c{0.5 * dx, 0.5 * dy};   // target centre = centre of the 3x3 stencil

    StencilBuild big;
    if (!big.build(g, -1, -1, 3, 2, h, -1, -1)) return MP_ERR_ARG_WRONG;
    for (int r = 0; r < 9; ++r) for (int m = 0; m < 9; ++m) t.C9[r][m] = big.coef[(size_t)r * 9 + m];
    for (int r = 1; r < 9; ++r) for (int s = 1; s < 9; ++s) t.S9[r - 1][s - 1] = big.sigma[(size_t)r * 9 + s];
    for (int tpos = 0; tpos < 4; ++tpos) {
        StencilBuild small;
        if (!small.build(g, 0, 0, 2, 1, h, tpos % 2, tpos / 2)) return MP_ERR_ARG_WRONG;
        if (tpos == 0) for (int r = 0; r < 4; ++r) for (int m = 0; m < 4; ++m) t.C4[r][m] = small.coef[(size_t)r * 4 + m];
        for (int r = 1; r < 4; ++r) for (int s = 1; s < 4; ++s) t.S4[tpos][r - 1][s - 1] = small.target[(size_t)r * 4 + s];
    }
    {
        int k = 0;
        for (int r = 0; r < 8; ++r)
            for (int c = r; c < 8; ++c) t.SF9[k++] = c == r ? t.S9[r][r] : 2.0 * t.S9[r][c];
        for (int tpos = 0; tpos < 4; ++tpos) {
            k = 0;
            for (int r = 0; r < 3; ++r)
                for (int c = r; c < 3; ++c) t.SF4[tpos][k++] = c == r ? t.S4[tpos][r][r] : 2.0 * t.S4[tpos][r][c];
        }
    }
    t.X = 0.5 * dx / h;
    t.Y = 0.5 * dy / h;
    t.scan_guard = 1e36 / (16.0 * std::max(1.0, t.X * t.X) * std::max(1.0, t.Y * t.Y));
    fill_diffusion(t, dx, dy, h, gw);
    t.y0 = y0; t.dy = dy; t.hn = h;
    t.epsA = 1e-2 * area;
    t.area = area;
    t.len_h = dx;
    t.len_v = dy;
    for (int q = 0; q < kNQ; ++q) { t.gq[q] = gp[q]; t.gw[q] = gw[q]; }
    for (int b = 0; b < kNQ; ++b)
        for (int a = 0; a < kNQ; ++a) {
            const V2 r{gp[a], gp[b]};
            t.cw[b * kNQ + a] = gw[a] * gw[b] * jacobian(r, target) / area;
            t.cwp[b * kNQ + a] = gw[a] * gw[b] * jacobian(r, target);
        }
    for (int q = 0; q < kNQ; ++q) { t.gx[q] = t.X * gp[q]; t.gy[q] = t.Y * gp[q]; }
    // Limiter points per class: class = cj*3 + ci, ci in {0: left wall, 1, 2: right wall}.
    int at = 0, nl = 0;
    for (int cls = 0; cls < 9; ++cls) {
        t.pt_off[cls] = at;
        const int ci = cls % 3, cj = cls / 3;
        std::vector<V2> pts;
        std::vector<unsigned char> kind;
        auto add = [&](V2 p, unsigned char k) { pts.push_back(V2{(p.x - c.x) / h, (p.y - c.y) / h}); kind.push_back(k); };
        add(bilinear(V2{0, 0}, target), 0);
        for (double a : gp) for (double b : gp) add(bilinear(V2{a, b}, target), 0);
        for (int e = 0; e < 4; ++e) {
            const V2 a = target[e], b = target[(e + 1) % 4];
            for (double r : gp) add(lerp_edge(r, a, b), 0);
            const bool wall = (e == 0 && cj == 0) || (e == 1 && ci == 2) || (e == 2 && cj == 2) || (e == 3 && ci == 0);
            const int ni = e == 1 ? 1 : (e == 3 ? -1 : 0), nj = e == 0 ? -1 : (e == 2 ? 1 : 0);
            std::vector<V2> s;
            if (wall) left_samples(a, b, target, nullptr, gp, s);
            else { const Quad other = g.cell(ni, nj); left_samples(a, b, target, &other, gp, s); }
            for (const V2& q : s) add(q, 1);
        }
        if (at + (int)pts.size() > kMaxPoints) return MP_ERR_ARG_SIZ;
        for (size_t k = 0; k < pts.size(); ++k) { t.pt_x[at] = pts[k].x; t.pt_y[at] = pts[k].y; t.pt_kind[at] = kind[k]; ++at; }
        // Group the points after the centre into 5-point lines. Each group of
        // 5 consecutive points (a Gauss row, an edge, or one sample depth of
        // an edge) shares one normalised coordinate; its other coordinate is
        // X*g_q or Y*g_q up to the rounding of the bilinear map.
        t.line_off[cls] = nl;
        std::vector<std::array<double, 3>> lines;  // dir, fixed coordinate, kind
        // 5x5 Gauss points were added with a outer (x), b inner (y): regroup into rows.
        for (int b = 0; b < kNQ; ++b) {
            double eta = 0;
            for (int a = 0; a < kNQ; ++a) eta += pts[1 + a * kNQ + b].y;
            lines.push_back({0.0, eta / kNQ, 0.0});
        }
        size_t k = 1 + kNQ * kNQ;
        for (int e = 0; e < 4; ++e) {
            const bool row = (e == 0 || e == 2);
            // edge points, then samples: for each Gauss point, the left-side
            // samples (2 interior / 4 boundary) -- regroup by depth.
            double fixed = 0;
            for (int q = 0; q < kNQ; ++q) fixed += row ? pts[k + q].y : pts[k + q].x;
            lines.push_back({row ? 0.0 : 1.0, fixed / kNQ, 0.0});
            k += kNQ;
            size_t ns = 0;
            while (k + ns < pts.size() && kind[k + ns] == 1) ++ns;
            const size_t per = ns / kNQ;   // samples per Gauss point
            for (size_t d = 0; d < per; ++d) {
                double f = 0;
                for (int q = 0; q < kNQ; ++q) f += row ? pts[k + q * per + d].y : pts[k + q * per + d].x;
                lines.push_back({row ? 0.0 : 1.0, f / kNQ, 1.0});
            }
            k += ns;
        }
        if (nl + (int)lines.size() > kMaxLines) return MP_ERR_ARG_SIZ;
        for (const auto& l : lines) { t.line_dir[nl] = (unsigned char)l[0]; t.line_c[nl] = l[1]; t.line_kind[nl] = (unsigned char)l[2]; ++nl; }
    }
    t.pt_off[9] = at;
    t.line_off[9] = nl;
    return MP_OK;
}

}  // namespace mp

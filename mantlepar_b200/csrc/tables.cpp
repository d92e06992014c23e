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

#include "../../include/mantlepar/mp.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <vector>

namespace mp {
namespace {

typedef long double ld;
struct V2 { double x, y; };
typedef std::array<V2, 4> Quad;

void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0); w.assign(n, 0.0);
    const ld pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < (n + 1) / 2; ++k) {
        ld z = std::cos(pi * (k + 0.75L) / (n + 0.5L)), deriv = 1;
        for (int it = 0; it < 100; ++it) {
            ld p_prev = 1, p = z;
            for (int m = 2; m <= n; ++m) { const ld next = ((2 * m - 1) * z * p - (m - 1) * p_prev) / m; p_prev = p; p = next; }
            if (n == 1) { p = z; p_prev = 1; }
            deriv = n * (z * p - p_prev) / (z * z - 1);
            const ld step = p / deriv;
            z -= step;
            if (std::fabs(step) < 1e-19L) break;
        }
        ld p_prev = 1, p = z;
        for (int m = 2; m <= n; ++m) { const ld next = ((2 * m - 1) * z * p - (m - 1) * p_prev) / m; p_prev = p; p = next; }
        if (n == 1) { p = z; p_prev = 1; }
        deriv = n * (z * p - p_prev) / (z * z - 1);
        const ld weight = 2 / ((1 - z * z) * deriv * deriv);
        x[n - 1 - k] = (double)z; x[k] = (double)-z;
        w[n - 1 - k] = (double)weight; w[k] = (double)weight;
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

V2 lerp_edge(double r, V2 a, V2 b) {
    const double s = 0.5 * (1.0 - r), t = 0.5 * (1.0 + r);
    return V2{s * a.x + t * b.x, s * a.y + t * b.y};
}
V2 bilinear(V2 r, const Quad& c) { return lerp_edge(r.y, lerp_edge(r.x, c[0], c[1]), lerp_edge(r.x, c[3], c[2])); }
double jacobian(V2 r, const Quad& c) {
    const double s = 0.5 * (1.0 + r.x), t = 0.5 * (1.0 + r.y);
    const double xi_x = 0.5 * ((1.0 - t) * (c[1].x - c[0].x) + t * (c[2].x - c[3].x));
    const double xi_y = 0.5 * ((1.0 - t) * (c[1].y - c[0].y) + t * (c[2].y - c[3].y));
    const double et_x = 0.5 * ((1.0 - s) * (c[3].x - c[0].x) + s * (c[2].x - c[1].x));
    const double et_y = 0.5 * ((1.0 - s) * (c[3].y - c[0].y) + s * (c[2].y - c[1].y));
    return xi_x * et_y - xi_y * et_x;
}
template <class F>
double cell_integral(const Quad& c, const std::vector<double>& p, const std::vector<double>& w, F&& f) {
    double sum = 0.0;
    for (size_t j = 0; j < p.size(); ++j)
        for (size_t i = 0; i < p.size(); ++i) {
            const V2 r{p[i], p[j]};
            sum += w[i] * w[j] * jacobian(r, c) * f(bilinear(r, c));
        }
    return sum;
}

double power(double x, int k) { double r = 1; for (int i = 0; i < k; ++i) r *= x; return r; }
double falling(int degree, int d) { double r = 1; for (int k = 0; k < d; ++k) r *= (double)(degree - k); return r; }
double horner_derivative(const double* c, int si, int sj, double x, double y, int dx, int dy) {
    if (dx >= si || dy >= sj) return 0;
    double result = 0;
    for (int j = sj; j-- > dy;) {
        double row = 0;
        for (int i = si; i-- > dx;) row = row * x + c[j * si + i] * falling(i, dx);
        result = result * y + row * falling(j, dy);
    }
    return result;
}

bool solve_identity(int n, std::vector<double> A, std::vector<double>& X) {
    X.assign((size_t)n * n, 0.0);
    for (int k = 0; k < n; ++k) X[(size_t)k * n + k] = 1.0;
    for (int k = 0; k < n; ++k) {
        int piv = k;
        for (int r = k + 1; r < n; ++r) if (std::fabs(A[(size_t)r * n + k]) > std::fabs(A[(size_t)piv * n + k])) piv = r;
        if (A[(size_t)piv * n + k] == 0.0) return false;
        if (piv != k)
            for (int c = 0; c < n; ++c) { std::swap(A[(size_t)k * n + c], A[(size_t)piv * n + c]); std::swap(X[(size_t)k * n + c], X[(size_t)piv * n + c]); }
        for (int r = k + 1; r < n; ++r) {
            const double f = A[(size_t)r * n + k] / A[(size_t)k * n + k];
            for (int c = k + 1; c < n; ++c) A[(size_t)r * n + c] -= f * A[(size_t)k * n + c];
            for (int c = 0; c < n; ++c) X[(size_t)r * n + c] -= f * X[(size_t)k * n + c];
        }
    }
    for (int k = n - 1; k >= 0; --k)
        for (int c = 0; c < n; ++c) {
            double s = X[(size_t)k * n + c];
            for (int j = k + 1; j < n; ++j) s -= A[(size_t)k * n + j] * X[(size_t)j * n + c];
            X[(size_t)k * n + c] = s / A[(size_t)k * n + k];
        }
    return true;
}

struct Grid {
    double dx, dy;
    V2 vert(int I, int J) const { return V2{(double)I * dx, (double)J * dy}; }
    Quad cell(int I, int J) const { return Quad{{vert(I, J), vert(I + 1, J), vert(I + 1, J + 1), vert(I, J + 1)}}; }
};

// Basis coefficients and smoothness matrices of an si x sj stencil whose
// lower-left cell is (I0, J0) on the grid, normalised by h.
struct StencilBuild {
    int si, sj, n;
    V2 center;
    std::vector<double> coef;   // [cell*n + m]
    std::vector<double> sigma;  // reference square
    std::vector<double> target; // target-cell smoothness

    void smoothness(const Quad& nc, int gp, int order, std::vector<double>& m) const {
        std::vector<double> p, w;
        gauss_legendre(gp, p, w);
        const double area = cell_integral(nc, p, w, [](V2) { return 1.0; });
        m.assign((size_t)n * n, 0.0);
        std::vector<double> der(n);
        for (int qy = 0; qy < gp; ++qy)
            for (int qx = 0; qx < gp; ++qx) {
                const V2 r{p[qx], p[qy]};
                const V2 x = bilinear(r, nc);
                const double weight = w[qx] * w[qy] * (jacobian(r, nc) / area);
                for (int dy = 0; dy < sj; ++dy)
                    for (int dx = 0; dx < si; ++dx) {
                        if (dx + dy == 0 || dx + dy > order) continue;
                        for (int c = 0; c < n; ++c) der[c] = horner_derivative(&coef[(size_t)c * n], si, sj, x.x, x.y, dx, dy);
                        for (int r2 = 0; r2 < n; ++r2)
                            for (int c = 0; c <= r2; ++c) m[(size_t)r2 * n + c] += weight * der[r2] * der[c];
                    }
            }
        for (int r2 = 0; r2 < n; ++r2)
            for (int c = 0; c <= r2; ++c) m[(size_t)c * n + r2] = m[(size_t)r2 * n + c];
    }

    bool build(const Grid& g, int I0, int J0, int size, int order, double h, int ti, int tj) {
        si = sj = size; n = si * sj;
        std::vector<Quad> cells((size_t)n);
        for (int j = 0; j < sj; ++j) for (int i = 0; i < si; ++i) cells[(size_t)j * si + i] = g.cell(I0 + i, J0 + j);
        const V2 anchor = cells.front()[0];
        const V2 outer[4] = {anchor, cells[(size_t)si - 1][1], cells.back()[2], cells[(size_t)(sj - 1) * si][3]};
        double off[2] = {0, 0};
        for (const V2& q : outer) { off[0] += (q.x - anchor.x) / 4; off[1] += (q.y - anchor.y) / 4; }
        center = V2{anchor.x + off[0], anchor.y + off[1]};
        auto normalise = [&](const Quad& q) {
            Quad o;
            for (int k = 0; k < 4; ++k) o[k] = V2{(q[k].x - center.x) / h, (q[k].y - center.y) / h};
            return o;
        };
        const int gp = std::max(3, size);
        std::vector<double> p, w;
        gauss_legendre(gp, p, w);
        std::vector<double> M((size_t)n * n);
        for (int c = 0; c < n; ++c) {
            const Quad nc = normalise(cells[c]);
            const double area = cell_integral(nc, p, w, [](V2) { return 1.0; });
            for (int j = 0; j < sj; ++j)
                for (int i = 0; i < si; ++i)
                    M[(size_t)c * n + (size_t)j * si + i] = cell_integral(nc, p, w, [i, j](V2 x) { return power(x.x, i) * power(x.y, j); }) / area;
        }
        std::vector<double> inv;
        if (!solve_identity(n, M, inv)) return false;
        coef.assign((size_t)n * n, 0.0);
        for (int c = 0; c < n; ++c) for (int m = 0; m < n; ++m) coef[(size_t)c * n + m] = inv[(size_t)m * n + c];
        const Quad ref{{V2{-0.5, -0.5}, V2{0.5, -0.5}, V2{0.5, 0.5}, V2{-0.5, 0.5}}};
        smoothness(ref, gp, order, sigma);
        if (ti >= 0) smoothness(normalise(cells[(size_t)tj * si + ti]), std::max(3, 2 * (size - 1)), order, target);
        return true;
    }
};

// Normal-line sample points on the LEFT side of an edge (a->b, CCW for the
// left cell), 4 samples per Gauss point at extent 0.9; `right` may be null.
double ray_exit(const Quad& c, int face, V2 o, V2 d) {
    ld exit = std::numeric_limits<ld>::infinity();
    for (int f = 0; f < 4; ++f) {
        if (f == face) continue;
        const V2 a = c[f], b = c[(f + 1) % 4];
        const ld tx = (ld)b.x - a.x, ty = (ld)b.y - a.y, rx = (ld)o.x - a.x, ry = (ld)o.y - a.y;
        const ld inside = tx * ry - ty * rx, rate = tx * d.y - ty * d.x;
        if (rate < 0) exit = std::min(exit, inside / (-rate));
    }
    return (double)exit;
}
int face_index(const Quad& c, V2 a, V2 b, bool rev) {
    for (int f = 0; f < 4; ++f) {
        const V2 p = c[f], q = c[(f + 1) % 4];
        const V2 u = rev ? b : a, v = rev ? a : b;
        if (p.x == u.x && p.y == u.y && q.x == v.x && q.y == v.y) return f;
    }
    return 0;
}
void left_samples(V2 a, V2 b, const Quad& left, const Quad* right, const std::vector<double>& gp, std::vector<V2>& out) {
    const int N = 4;
    const double frac = 0.9;
    const double ddx = b.x - a.x, ddy = b.y - a.y;
    const double scale = std::max(std::fabs(ddx), std::fabs(ddy));
    const double ux = ddx / scale, uy = ddy / scale, norm = std::sqrt(ux * ux + uy * uy);
    const V2 nrm{uy / norm, -ux / norm};
    const int lf = face_index(left, a, b, false), rf = right ? face_index(*right, a, b, true) : 0;
    const bool boundary = right == nullptr;
    const int count = boundary ? N + 1 : N;
    for (double r : gp) {
        const V2 p = lerp_edge(r, a, b);
        double avail = ray_exit(left, lf, p, V2{-nrm.x, -nrm.y});
        if (right) avail = std::min(avail, ray_exit(*right, rf, p, nrm));
        const double spacing = (double)((ld)frac * avail * (boundary ? 1.0L / N : 2.0L / (N - 1)));
        for (int k = 0; k < count; ++k) {
            const bool left_side = boundary ? (k + 1 != count) : (k < count / 2);
            if (!left_side) continue;
            const ld offset = boundary ? (ld)k - N : (ld)k - (N - 1) / 2.0L;
            const ld dist = offset * spacing;
            out.push_back(V2{(double)((ld)p.x + dist * nrm.x), (double)((ld)p.y + dist * nrm.y)});
        }
    }
}

}  // namespace

namespace {

// diffusiveflux.cpp:203-253: first-derivative weights on uniform nodes 0..n
// at n/2 (middle) or n (end), long double intermediates.
void derivative_weights(int count, bool middle, double* w) {
    typedef long double ld;
    const int n = count - 1;
    if (middle) {
        ld factor = std::exp2(1.0L - n);
        for (int k = 3; k <= n; k += 2) factor *= (ld)k / (k - 1);
        if ((count / 2) % 2) factor = -factor;
        ld choose = 1;
        for (int i = 0; i < count / 2; ++i) {
            const ld den = (ld)n - 2.0L * i;
            w[i] = (double)(factor * choose / (den * den));
            w[n - i] = -w[i];
            choose *= (ld)(n - i) / (i + 1);
            factor = -factor;
        }
    } else {
        ld harmonic = 0;
        for (int j = 1; j <= n; ++j) harmonic += 1.0L / j;
        w[n] = (double)harmonic;
        ld choose = 1, sign = n % 2 ? -1 : 1;
        for (int i = 0; i < n; ++i) {
            w[i] = (double)(sign * choose / (n - i));
            choose *= (ld)(n - i) / (i + 1);
            sign = -sign;
        }
    }
}

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

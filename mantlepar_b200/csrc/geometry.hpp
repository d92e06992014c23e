// Host geometry of logically rectangular quad meshes, shared by the uniform
// table builder (tables.cpp) and the per-cell tables of general quad meshes
// (quad_tables.cpp). The arithmetic follows the reference's setup code:
//   Gauss-Legendre rule (PetscDTGaussQuadrature, src/core/integral.cpp:7-20)
//   bilinear maps and Jacobian (src/core/integral.cpp:91-121)
//   stencil centre, moments, inverse, smoothness (tensorstencilpoly.cpp:146-231,318-368,383-398)
//   normal-line samples (diffusiveflux.cpp:23-84,203-334; 4 samples, extent 0.9)
#ifndef MP_GEOMETRY_HPP
#define MP_GEOMETRY_HPP

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <utility>
#include <vector>

namespace mp {
namespace geo {

typedef long double ld;
struct V2 { double x, y; };
typedef std::array<V2, 4> Quad;

inline void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
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

// The rule of n points, computed once per n (n <= 16) and shared.
inline const std::pair<std::vector<double>, std::vector<double>>& gauss_rule_cached(int n) {
    static const auto rules = [] {
        std::vector<std::pair<std::vector<double>, std::vector<double>>> r(17);
        for (int k = 1; k <= 16; ++k) gauss_legendre(k, r[k].first, r[k].second);
        return r;
    }();
    return rules[n];
}

inline V2 lerp_edge(double r, V2 a, V2 b) {
    const double s = 0.5 * (1.0 - r), t = 0.5 * (1.0 + r);
    return V2{s * a.x + t * b.x, s * a.y + t * b.y};
}
inline V2 bilinear(V2 r, const Quad& c) { return lerp_edge(r.y, lerp_edge(r.x, c[0], c[1]), lerp_edge(r.x, c[3], c[2])); }
inline double jacobian(V2 r, const Quad& c) {
    const double s = 0.5 * (1.0 + r.x), t = 0.5 * (1.0 + r.y);
    const double xi_x = 0.5 * ((1.0 - t) * (c[1].x - c[0].x) + t * (c[2].x - c[3].x));
    const double xi_y = 0.5 * ((1.0 - t) * (c[1].y - c[0].y) + t * (c[2].y - c[3].y));
    const double et_x = 0.5 * ((1.0 - s) * (c[3].x - c[0].x) + s * (c[2].x - c[1].x));
    const double et_y = 0.5 * ((1.0 - s) * (c[3].y - c[0].y) + s * (c[2].y - c[1].y));
    return xi_x * et_y - xi_y * et_x;
}
template <class F>
inline double cell_integral(const Quad& c, const std::vector<double>& p, const std::vector<double>& w, F&& f) {
    double sum = 0.0;
    for (size_t j = 0; j < p.size(); ++j)
        for (size_t i = 0; i < p.size(); ++i) {
            const V2 r{p[i], p[j]};
            sum += w[i] * w[j] * jacobian(r, c) * f(bilinear(r, c));
        }
    return sum;
}

inline double power(double x, int k) { double r = 1; for (int i = 0; i < k; ++i) r *= x; return r; }
inline double falling(int degree, int d) { double r = 1; for (int k = 0; k < d; ++k) r *= (double)(degree - k); return r; }
inline double horner_derivative(const double* c, int si, int sj, double x, double y, int dx, int dy) {
    if (dx >= si || dy >= sj) return 0;
    double result = 0;
    for (int j = sj; j-- > dy;) {
        double row = 0;
        for (int i = si; i-- > dx;) row = row * x + c[j * si + i] * falling(i, dx);
        result = result * y + row * falling(j, dy);
    }
    return result;
}

inline bool solve_identity(int n, std::vector<double> A, std::vector<double>& X) {
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

// Basis coefficients and smoothness matrices of an si x sj stencil whose
// lower-left cell is (I0, J0) of a mesh (any type with Quad cell(I, J)),
// normalised by h.
struct StencilBuild {
    int si, sj, n;
    V2 center;
    std::vector<double> coef;   // [cell*n + m]
    std::vector<double> sigma;  // reference square
    std::vector<double> target; // target-cell smoothness

    void smoothness(const Quad& nc, int gp, int order, std::vector<double>& m) const {
        const std::vector<double>& p = gauss_rule_cached(gp).first;
        const std::vector<double>& w = gauss_rule_cached(gp).second;
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

    template <class Mesh>
    bool build(const Mesh& g, int I0, int J0, int size, int order, double h, int ti, int tj) {
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
        const std::vector<double>& p = gauss_rule_cached(gp).first;
        const std::vector<double>& w = gauss_rule_cached(gp).second;
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
inline double ray_exit(const Quad& c, int face, V2 o, V2 d) {
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
inline int face_index(const Quad& c, V2 a, V2 b, bool rev) {
    for (int f = 0; f < 4; ++f) {
        const V2 p = c[f], q = c[(f + 1) % 4];
        const V2 u = rev ? b : a, v = rev ? a : b;
        if (p.x == u.x && p.y == u.y && q.x == v.x && q.y == v.y) return f;
    }
    return 0;
}
inline void left_samples(V2 a, V2 b, const Quad& left, const Quad* right, const std::vector<double>& gp, std::vector<V2>& out) {
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

// diffusiveflux.cpp:203-253: first-derivative weights on uniform nodes 0..n
// at n/2 (middle) or n (end), long double intermediates.
inline void derivative_weights(int count, bool middle, double* w) {
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

}  // namespace geo
}  // namespace mp

#endif

// CPU oracle: restated per-cell numerics of the ML-WENO reconstruction.
// TEST INFRASTRUCTURE ONLY -- the checker for the CUDA transport kernels.
//
// Restates, with the reference's long double internals:
//   src/core/integral.cpp:7-121       Gauss rule, edge geometry, bilinear maps
//   src/core/mesh.cpp:12-25           SplitMix64 stateless noise
//   src/mlweno/tensorstencilpoly.cpp  moments, stencil inverse, smoothness,
//                                     centred evaluation (:146-231,:293-459)
//   src/mlweno/reconstruction.cpp     candidate filtering and log-space
//                                     nonlinear weights (:109-355,:477-502)
//   src/mlweno/diffusiveflux.cpp      normal-line sample geometry (:23-84,:255-334)
//   src/mlweno/advectiveflux.cpp      linear-law Lax-Friedrichs edge and
//                                     boundary flux integrals (:8-267)
// The Gauss-Legendre rule stands in for PETSc's PetscDTGaussQuadrature
// (PETSc 3.23+, not vendored): Newton iteration on P_n in long double, the
// published Golub-Welsch-free method; nodes agree with PETSc to ~1 ulp.
#ifndef MP_ORACLE_RESTATED_HPP
#define MP_ORACLE_RESTATED_HPP

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <memory>
#include <vector>

namespace orc {

typedef long double ld;
// Per-cell and per-face evaluation type. The reference evaluates these steps
// in long double (80-bit on x86-64); building with ORC_FP64_CELL evaluates
// the same steps in double, which measures how far the results move with the
// precision of the intermediates alone (tables and geometry stay long double).
#ifdef ORC_FP64_CELL
typedef double lc;
#else
typedef long double lc;
#endif

struct Pt { double x = 0, y = 0; };
typedef std::array<Pt, 4> Quad;

// Error codes of the transport oracle (mirroring the PETSc error classes the
// reference raises on this path).
enum Err {
    E_OK = 0, E_OUTOFRANGE = 63, E_FP = 72, E_WRONG = 62, E_WRONGSTATE = 73,
    E_SIZ = 60, E_NOT_CONVERGED = 91, E_PLIB = 77, E_PHASE = 100
};
struct Error { int code; const char* what; };
inline void require(bool ok, int code, const char* what) { if (!ok) throw Error{code, what}; }

// ---------------------------------------------------------------- geometry

// Gauss-Legendre nodes/weights on [-1,1], ascending nodes.
inline void gauss_rule(int n, std::vector<double>& pts, std::vector<double>& wts) {
    pts.assign(n, 0.0); wts.assign(n, 0.0);
    const ld pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < (n + 1) / 2; ++k) {
        ld x = std::cos(pi * (k + 0.75L) / (n + 0.5L));
        ld dp = 0;
        for (int it = 0; it < 100; ++it) {
            ld p0 = 1, p1 = x;
            for (int m = 2; m <= n; ++m) { ld p2 = ((2 * m - 1) * x * p1 - (m - 1) * p0) / m; p0 = p1; p1 = p2; }
            if (n == 1) { p1 = x; p0 = 1; }
            dp = n * (x * p1 - p0) / (x * x - 1);
            ld dx = p1 / dp;
            x -= dx;
            if (std::fabs(dx) < 1e-19L) break;
        }
        {
            ld p0 = 1, p1 = x;
            for (int m = 2; m <= n; ++m) { ld p2 = ((2 * m - 1) * x * p1 - (m - 1) * p0) / m; p0 = p1; p1 = p2; }
            if (n == 1) { p1 = x; p0 = 1; }
            dp = n * (x * p1 - p0) / (x * x - 1);
        }
        const ld w = 2 / ((1 - x * x) * dp * dp);
        pts[n - 1 - k] = (double)x; pts[k] = (double)-x;
        wts[n - 1 - k] = (double)w; wts[k] = (double)w;
    }
    if (n % 2 == 1) pts[n / 2] = 0.0;
}

// integral.cpp:62-89
inline void edge_geometry(Pt a, Pt b, double& length, Pt& normal) {
    const double dx = b.x - a.x, dy = b.y - a.y;
    const double scale = std::max(std::fabs(dx), std::fabs(dy));
    require(scale > 0, E_OUTOFRANGE, "Edge endpoints must be distinct");
    const double ux = dx / scale, uy = dy / scale;
    const double norm = std::sqrt(ux * ux + uy * uy);
    length = scale * norm;
    normal = Pt{uy / norm, -ux / norm};
}

// integral.cpp:91-98
inline Pt map_edge(double r, Pt a, Pt b) {
    const double s = 0.5 * (1.0 - r), t = 0.5 * (1.0 + r);
    return Pt{s * a.x + t * b.x, s * a.y + t * b.y};
}

// integral.cpp:100-107
inline Pt map_cell(Pt ref, const Quad& c) {
    const Pt lo = map_edge(ref.x, c[0], c[1]);
    const Pt hi = map_edge(ref.x, c[3], c[2]);
    return map_edge(ref.y, lo, hi);
}

// integral.cpp:109-121
inline double cell_jacobian(Pt ref, const Quad& c) {
    const double s = 0.5 * (1.0 + ref.x), t = 0.5 * (1.0 + ref.y);
    double dxi[2], deta[2];
    const double cx[4] = {c[0].x, c[1].x, c[2].x, c[3].x};
    const double cy[4] = {c[0].y, c[1].y, c[2].y, c[3].y};
    for (int d = 0; d < 2; ++d) {
        const double* v = d ? cy : cx;
        dxi[d] = 0.5 * ((1.0 - t) * (v[1] - v[0]) + t * (v[2] - v[3]));
        deta[d] = 0.5 * ((1.0 - s) * (v[3] - v[0]) + s * (v[2] - v[1]));
    }
    return dxi[0] * deta[1] - dxi[1] * deta[0];
}

// integral.h:49-78 (IntegrateCell) for a callback f(Pt).
template <class F>
inline double integrate_cell(const Quad& c, const std::vector<double>& p, const std::vector<double>& w, F&& f) {
    double sum = 0.0;
    for (size_t j = 0; j < p.size(); ++j)
        for (size_t i = 0; i < p.size(); ++i) {
            const Pt ref{p[i], p[j]};
            const Pt x = map_cell(ref, c);
            const double jac = cell_jacobian(ref, c);
            require(jac > 0, E_FP, "Cell mapping produced an invalid Jacobian");
            sum += w[i] * w[j] * jac * f(x);
        }
    return sum;
}

// mesh.cpp:12-25: stateless SplitMix64 finaliser, unit in [0,1).
inline uint64_t mix64(uint64_t v) {
    v += UINT64_C(0x9e3779b97f4a7c15);
    v = (v ^ (v >> 30)) * UINT64_C(0xbf58476d1ce4e5b9);
    v = (v ^ (v >> 27)) * UINT64_C(0x94d049bb133111eb);
    return v ^ (v >> 31);
}
inline double unit_noise(uint64_t key) { return (double)(mix64(key) >> 11) * 0x1.0p-53; }

// ------------------------------------------------------ tensor stencil poly

inline double ipow(double x, int k) { double r = 1; for (int i = 0; i < k; ++i) r *= x; return r; }
inline double falling(int degree, int d) { double r = 1; for (int k = 0; k < d; ++k) r *= (double)(degree - k); return r; }

// tensorstencilpoly.cpp:61-74 (Horner in normalised coordinates)
inline double normalized_derivative(const double* c, int si, int sj, double x, double y, int dx, int dy) {
    if (dx >= si || dy >= sj) return 0;
    double result = 0;
    for (int j = sj; j-- > dy;) {
        double row = 0;
        for (int i = si; i-- > dx;) row = row * x + c[(size_t)j * si + i] * falling(i, dx);
        result = result * y + row * falling(j, dy);
    }
    return result;
}

// Row-major dense solve A X = B with partial pivoting (stand-in for
// LAPACKE_dgesv, tensorstencilpoly.cpp:211). A is n x n, B is n x n.
inline void lu_solve(int n, std::vector<double>& A, std::vector<double>& B) {
    for (int k = 0; k < n; ++k) {
        int piv = k;
        double best = std::fabs(A[(size_t)k * n + k]);
        for (int r = k + 1; r < n; ++r) {
            const double v = std::fabs(A[(size_t)r * n + k]);
            if (v > best) { best = v; piv = r; }
        }
        require(best > 0, E_WRONG, "Stencil moment solve failed");
        if (piv != k) {
            for (int c = 0; c < n; ++c) { std::swap(A[(size_t)k * n + c], A[(size_t)piv * n + c]); std::swap(B[(size_t)k * n + c], B[(size_t)piv * n + c]); }
        }
        for (int r = k + 1; r < n; ++r) {
            const double f = A[(size_t)r * n + k] / A[(size_t)k * n + k];
            A[(size_t)r * n + k] = f;
            for (int c = k + 1; c < n; ++c) A[(size_t)r * n + c] -= f * A[(size_t)k * n + c];
            for (int c = 0; c < n; ++c) B[(size_t)r * n + c] -= f * B[(size_t)k * n + c];
        }
    }
    for (int k = n - 1; k >= 0; --k)
        for (int c = 0; c < n; ++c) {
            double s = B[(size_t)k * n + c];
            for (int j = k + 1; j < n; ++j) s -= A[(size_t)k * n + j] * B[(size_t)j * n + c];
            B[(size_t)k * n + c] = s / A[(size_t)k * n + k];
        }
}

// Geometry-dependent stencil tables (coefficients and smoothness matrices).
struct StencilTables {
    std::vector<double> coef;          // basis-major: coef[cell*n + monomial]
    std::vector<double> sigma;         // reference-square smoothness matrix
    std::vector<double> target_sigma;  // target-cell smoothness (if set)
};

struct StencilPoly {
    int si = 0, sj = 0, n = 0, order = 0;
    Pt center;
    double h = 0;
    const StencilTables* tab = nullptr;

    // tensorstencilpoly.cpp:318-368
    void build_smoothness(const std::vector<double>& coef, const Quad& nc, int gp, std::vector<double>& m) const {
        std::vector<double> p, w;
        gauss_rule(gp, p, w);
        const double area = integrate_cell(nc, p, w, [](Pt) { return 1.0; });
        require(area > 0, E_FP, "Smoothness integration area must be positive");
        std::vector<double> work((size_t)n * n, 0.0), der(n);
        for (size_t qy = 0; qy < p.size(); ++qy)
            for (size_t qx = 0; qx < p.size(); ++qx) {
                const Pt ref{p[qx], p[qy]};
                const Pt x = map_cell(ref, nc);
                const double weight = w[qx] * w[qy] * (cell_jacobian(ref, nc) / area);
                for (int dy = 0; dy < sj; ++dy)
                    for (int dx = 0; dx < si; ++dx) {
                        if (dx + dy == 0 || dx + dy > order) continue;
                        for (int c = 0; c < n; ++c) der[c] = normalized_derivative(coef.data() + (size_t)c * n, si, sj, x.x, x.y, dx, dy);
                        for (int r = 0; r < n; ++r)
                            for (int c = 0; c <= r; ++c) work[(size_t)r * n + c] += weight * der[r] * der[c];
                    }
            }
        for (int r = 0; r < n; ++r)
            for (int c = 0; c <= r; ++c) work[(size_t)c * n + r] = work[(size_t)r * n + c];
        m.swap(work);
    }

    Quad normalize(const Quad& q) const {
        Quad out;
        for (int k = 0; k < 4; ++k) out[k] = Pt{(q[k].x - center.x) / h, (q[k].y - center.y) / h};
        return out;
    }

    // Geometry part of tensorstencilpoly.cpp:146-176 (centre of the outer vertices).
    void place(const std::vector<Quad>& corners, int size_i, int size_j, int ord, double hh) {
        si = size_i; sj = size_j; n = si * sj; order = ord; h = hh;
        const Pt anchor = corners.front()[0];
        const Pt outer[4] = {anchor, corners[(size_t)si - 1][1], corners.back()[2], corners[(size_t)(sj - 1) * si][3]};
        double off[2] = {0, 0};
        for (const Pt& q : outer) { off[0] += (q.x - anchor.x) / 4; off[1] += (q.y - anchor.y) / 4; }
        center = Pt{anchor.x + off[0], anchor.y + off[1]};
    }

    // Tables of tensorstencilpoly.cpp:178-228 and :383-398 for this placement.
    void build_tables(const std::vector<Quad>& corners, int ti, int tj, bool target, StencilTables& t) const {
        const int gp = std::max(3, std::max(si, sj));
        std::vector<double> p, w;
        gauss_rule(gp, p, w);
        std::vector<double> moments((size_t)n * n, 0.0), inverse((size_t)n * n, 0.0);
        for (int cell = 0; cell < n; ++cell) {
            const Quad nc = normalize(corners[cell]);
            const double area = integrate_cell(nc, p, w, [](Pt) { return 1.0; });
            require(area > 0, E_FP, "Normalized cell area must be positive");
            for (int j = 0; j < sj; ++j)
                for (int i = 0; i < si; ++i) {
                    const double mom = integrate_cell(nc, p, w, [i, j](Pt x) { return ipow(x.x, i) * ipow(x.y, j); });
                    moments[(size_t)cell * n + (size_t)j * si + i] = mom / area;
                }
            inverse[(size_t)cell * n + cell] = 1;
        }
        lu_solve(n, moments, inverse);
        t.coef.assign((size_t)n * n, 0.0);
        for (int cell = 0; cell < n; ++cell)
            for (int m = 0; m < n; ++m) t.coef[(size_t)cell * n + m] = inverse[(size_t)m * n + cell];
        const Quad ref{{Pt{-0.5, -0.5}, Pt{0.5, -0.5}, Pt{0.5, 0.5}, Pt{-0.5, 0.5}}};
        build_smoothness(t.coef, ref, gp, t.sigma);
        if (target) {
            const Quad nc = normalize(corners[(size_t)tj * si + ti]);
            const int degree = (si - 1) + (sj - 1);
            build_smoothness(t.coef, nc, std::max(3, degree), t.target_sigma);
        }
    }

    // tensorstencilpoly.cpp:400-459 (value only)
    static double apply_smoothness(const std::vector<double>& m, const double* avg, int n) {
        lc diff[16];
        for (int i = 0; i < n; ++i) diff[i] = (lc)avg[i] - avg[0];
        lc sum = 0, mag = 0;
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) {
                const lc term = diff[r] * m[(size_t)r * n + c] * diff[c];
                sum += term;
                mag += std::fabs(term);
            }
        require(std::isfinite(sum) && std::isfinite(mag), E_FP, "Smoothness evaluation overflowed");
        const lc tol = 64 * (lc)std::numeric_limits<double>::epsilon() * mag;
        require(sum >= -tol, E_FP, "Smoothness quadratic form is negative beyond roundoff");
        return (double)std::max((lc)0, sum);
    }

    // tensorstencilpoly.cpp:293-316 + :247-270 (value, dx=dy=0)
    double evaluate(const double* avg, Pt p) const {
        double poly[16];
        for (int k = 0; k < n; ++k) poly[k] = 0;
        poly[0] = avg[0];
        const double* coef = tab->coef.data();
        for (int c = 0; c < n; ++c) {
            const double d = avg[c] - avg[0];
            for (int k = 0; k < n; ++k) poly[k] += d * coef[(size_t)c * n + k];
        }
        const double x = (p.x - center.x) / h, y = (p.y - center.y) / h;
        return normalized_derivative(poly, si, sj, x, y, 0, 0);
    }
};

// ---------------------------------------------------------- reconstruction

// One ML-WENO reconstruction of one target cell with the coupled solver's
// candidate set (state_reconstruction.cpp:64-68): large 3x3 order 2 at offset
// (-1,-1) with reference-square smoothness; small 2x2 order 1 at offsets
// (0,-1),(0,0),(-1,-1),(-1,0) with target-cell smoothness; epsilon 1e-2, s 1,
// no constant candidate; candidates leaving the domain are discarded
// (reconstruction.cpp:143-175).
struct Candidate {
    StencilPoly poly;
    int si = 0, sj = 0, start_i = 0, start_j = 0, order = 0, ti = 0, tj = 0;
    bool target_smooth = false;
    double linear = 1;
};

struct CandidateSet {
    std::vector<Candidate> cand;
};

inline int eta_of(int r) { return r == 1 ? 1 : (r == 2 ? 3 : 4); }

// log(sigma + eps*A) without forming eps*A (reconstruction.cpp:46-54).
inline lc log_denominator(double sigma, lc logReg) {
    if (sigma == 0) return logReg;
    const lc ls = std::log((lc)sigma);
    const lc hi = std::max(ls, logReg), lo = std::min(ls, logReg);
    return hi + std::log1p(std::exp(lo - hi));
}

struct Recon {
    const CandidateSet* set = nullptr;
    double target = 0;               // target cell average
    double w[5] = {0, 0, 0, 0, 0};   // nonlinear weights
    double centered[5][9];           // centred averages per candidate

    // reconstruction.cpp:275-355 + :212-265
    void update(const double* field, int nx, double area) {
        const size_t nc = set->cand.size();
        double sig[5];
        for (size_t k = 0; k < nc; ++k) {
            const Candidate& c = set->cand[k];
            for (int j = 0; j < c.sj; ++j)
                for (int i = 0; i < c.si; ++i) {
                    const double a = field[(size_t)(c.start_j + j) * nx + (c.start_i + i)];
                    require(std::isfinite(a), E_OUTOFRANGE, "Referenced cell averages must be finite");
                    centered[k][j * c.si + i] = a - target;
                }
            sig[k] = StencilPoly::apply_smoothness(c.target_smooth ? c.poly.tab->target_sigma : c.poly.tab->sigma, centered[k], c.poly.n);
        }
        const double eps = 1e-2;
        const int s = 1;
        lc logA[6];
        const lc logReg = std::log((lc)eps) + std::log((lc)area);
        for (size_t k = 0; k < nc; ++k) {
            const int r = set->cand[k].order + 1;
            const lc ex = (lc)s * r + eta_of(r);
            logA[k] = std::log((lc)set->cand[k].linear) - ex * log_denominator(sig[k], logReg);
            require(std::isfinite(logA[k]), E_FP, "Polynomial log weight is not finite");
        }
        logA[nc] = -std::numeric_limits<lc>::infinity();  // constant candidate disabled
        lc mx = logA[0];
        for (size_t k = 1; k <= nc; ++k) mx = std::max(mx, logA[k]);
        lc sum = 0;
        for (size_t k = 0; k <= nc; ++k) { logA[k] = std::exp(logA[k] - mx); sum += logA[k]; }
        require(std::isfinite(sum) && sum > 0, E_FP, "Invalid ML-WENO weight normalization");
        for (size_t k = 0; k < nc; ++k) w[k] = (double)(logA[k] / sum);
    }

    // reconstruction.cpp:477-502
    double evaluate(Pt p) const {
        lc result = target;
        for (size_t k = 0; k < set->cand.size(); ++k) {
            if (w[k] == 0) continue;
            result += (lc)w[k] * set->cand[k].poly.evaluate(centered[k], p);
        }
        require(std::isfinite(result), E_FP, "Reconstructed value is not representable");
        return (double)result;
    }
};

// ------------------------------------------------- diffusion sample points

// diffusiveflux.cpp:23-38
inline int find_face(const Quad& c, Pt a, Pt b, bool reverse) {
    for (int f = 0; f < 4; ++f) {
        const Pt p = c[f], q = c[(f + 1) % 4];
        const Pt u = reverse ? b : a, v = reverse ? a : b;
        if (p.x == u.x && p.y == u.y && q.x == v.x && q.y == v.y) return f;
    }
    throw Error{E_WRONG, "Edge must match the cell vertices with the required orientation"};
}

// diffusiveflux.cpp:43-72
inline double ray_distance(const Quad& c, int face, Pt o, Pt dir) {
    ld exit = std::numeric_limits<ld>::infinity();
    for (int f = 0; f < 4; ++f) {
        if (f == face) continue;
        const Pt a = c[f], b = c[(f + 1) % 4];
        const ld tx = (ld)b.x - a.x, ty = (ld)b.y - a.y;
        const ld rx = (ld)o.x - a.x, ry = (ld)o.y - a.y;
        const ld inside = tx * ry - ty * rx;
        require(std::isfinite(inside) && inside > 0, E_WRONG, "Edge quadrature point must lie strictly between the other cell faces");
        const ld rate = tx * dir.y - ty * dir.x;
        if (rate < 0) exit = std::min(exit, inside / (-rate));
    }
    const double d = (double)exit;
    require(d > 0, E_OUTOFRANGE, "Normal sampling requires positive available distance");
    return d;
}

struct Sampling {
    std::vector<Pt> samples;
    std::vector<int> sides;     // 0 left, 1 right, 2 boundary
    std::vector<double> spacing, weights, coefficients;
    std::vector<Pt> points;
    Pt normal;
    bool boundary = false;
    std::shared_ptr<const void> native;   // the reference's own sampling object (reference-backed build)
};

// diffusiveflux.cpp:203-253: first-derivative weights on the uniform nodes
// 0..n (n = count - 1), at n/2 (middle, count even) or at n (end).
inline std::vector<double> lagrange_derivative_weights(int count, bool middle) {
    const int n = count - 1;
    std::vector<double> w((size_t)count);
    auto real = [](ld v) {
        require(std::isfinite(v) && std::fabs(v) <= (ld)std::numeric_limits<double>::max(), E_FP,
                "Diffusion geometry, flux or derivative is not representable");
        return (double)v;
    };
    if (middle) {
        ld factor = std::exp2(1.0L - n);
        for (int k = 3; k <= n; k += 2) factor *= (ld)k / (k - 1);
        if ((count / 2) % 2) factor = -factor;
        ld choose = 1;
        for (int i = 0; i < count / 2; ++i) {
            const ld den = (ld)n - 2.0L * i;
            w[i] = real(factor * choose / (den * den));
            w[n - i] = -w[i];
            choose *= (ld)(n - i) / (i + 1);
            factor = -factor;
        }
    } else {
        ld harmonic = 0;
        for (int j = 1; j <= n; ++j) harmonic += 1.0L / j;
        w[n] = real(harmonic);
        ld choose = 1, sign = n % 2 ? -1 : 1;
        for (int i = 0; i < n; ++i) {
            w[i] = real(sign * choose / (n - i));
            choose *= (ld)(n - i) / (i + 1);
            sign = -sign;
        }
    }
    return w;
}

// Thermal boundary data at one Gauss point (EvaluateThermalBoundary,
// initialization.cpp:490-506): 0 zero flux, 1 prescribed temperature,
// 2 prescribed outward flux per unit length.
struct ThermalBC { int type = 0; double value = 0; };

// diffusiveflux.cpp:105-200 with the identity law (psi = T): the edge's
// diffusive flux and d flux / d sample per sample (zero at boundary slots).
inline void integrate_diffusion(const Sampling& s, const std::vector<double>& samples, double kappa,
                                const ThermalBC* bc, double& flux, std::vector<double>& deriv) {
    const size_t nq = s.points.size(), count = s.coefficients.size();
    auto real = [](lc v) {
        require(std::isfinite(v) && std::fabs(v) <= (lc)std::numeric_limits<double>::max(), E_FP,
                "Diffusion geometry, flux or derivative is not representable");
        return (double)v;
    };
    lc last_coef = 0;
    for (size_t k = 0; k + 1 < count; ++k) last_coef -= s.coefficients[k];
    lc integral = 0;
    deriv.assign(samples.size(), 0.0);
    std::vector<double> v(count);
    for (size_t q = 0; q < nq; ++q) {
        const double weight = s.weights[q];
        const int type = bc ? bc->type : -1;
        if (bc) {
            if (type == 0) continue;
            require(std::isfinite(bc->value), E_OUTOFRANGE, "Boundary data must be finite");
            if (type == 2) { integral += (lc)weight * bc->value; continue; }
        }
        require(std::isfinite(kappa) && kappa >= 0, E_OUTOFRANGE, "Diffusivity must be finite and nonnegative");
        for (size_t k = 0; k < count; ++k) {
            const size_t a = q * count + k;
            const double u = (bc && k + 1 == count) ? bc->value : samples[a];
            require(std::isfinite(u), E_OUTOFRANGE, "Diffusion sample state must be finite");
            v[k] = u;
        }
        lc gradient = 0;
        for (size_t k = 0; k + 1 < count; ++k) gradient += (lc)s.coefficients[k] * ((lc)v[k] - v.back());
        gradient /= s.spacing[q];
        require(std::isfinite(gradient), E_FP, "Sampled normal derivative overflowed");
        integral -= (lc)weight * kappa * gradient;
        const lc scale = -(lc)weight * kappa / s.spacing[q];
        for (size_t k = 0; k < count; ++k) {
            const lc coef = k + 1 == count ? last_coef : (lc)s.coefficients[k];
            const double partial = real(scale * coef * 1.0);
            if (!(bc && k + 1 == count)) deriv[q * count + k] = partial;
        }
    }
    flux = real(integral);
}

// diffusiveflux.cpp:255-334 with numberOfSamples N and extentFraction f.
inline void build_sampling(Pt a, Pt b, const Quad& left, const Quad* right,
                           const std::vector<double>& rp, const std::vector<double>& rw,
                           int N, double frac, Sampling& s) {
    double length;
    edge_geometry(a, b, length, s.normal);
    const int lf = find_face(left, a, b, false);
    const int rf = right ? find_face(*right, a, b, true) : 0;
    s.boundary = right == nullptr;
    const int count = s.boundary ? N + 1 : N;
    s.coefficients = lagrange_derivative_weights(count, !s.boundary);
    const size_t nq = rp.size();
    s.points.resize(nq); s.spacing.resize(nq); s.weights.resize(nq);
    s.samples.resize(nq * count); s.sides.resize(nq * count);
    const Pt inward{-s.normal.x, -s.normal.y};
    for (size_t q = 0; q < nq; ++q) {
        s.points[q] = map_edge(rp[q], a, b);
        double avail = ray_distance(left, lf, s.points[q], inward);
        if (right) avail = std::min(avail, ray_distance(*right, rf, s.points[q], s.normal));
        const ld sp = (ld)frac * avail * (s.boundary ? 1.0L / N : 2.0L / (N - 1));
        s.spacing[q] = (double)sp;
        s.weights[q] = (double)((ld)length * rw[q] / 2);
        for (int k = 0; k < count; ++k) {
            const ld off = s.boundary ? (ld)k - N : (ld)k - (N - 1) / 2.0L;
            const ld dist = off * s.spacing[q];
            const size_t at = q * count + k;
            s.samples[at] = Pt{(double)((ld)s.points[q].x + dist * s.normal.x),
                               (double)((ld)s.points[q].y + dist * s.normal.y)};
            s.sides[at] = s.boundary ? (k + 1 == count ? 2 : 0) : (k < count / 2 ? 0 : 1);
        }
    }
}

// ------------------------------------------------------- advective flux

// Advection boundary data of one edge point (AdvectiveBoundaryType):
// 0 prescribed state, 1 extrapolated state, 2 zero flux.
struct AdvectBC { int type = 1; double value = 0; };

// advectiveflux.cpp:8-18 (RealValue) and :41-48 (NormalVelocity).
inline double real_value(lc v) {
    require(std::isfinite(v) && std::fabs(v) <= (lc)std::numeric_limits<double>::max(), E_FP,
            "Advective flux or derivative is not representable");
    return (double)v;
}
inline double normal_velocity(Pt v, Pt n) { return real_value((lc)v.x * n.x + (lc)v.y * n.y); }

// advectiveflux.cpp:20-39 (CheckPoint) for the point fields the flux reads.
inline void check_point(Pt p, Pt v, Pt n) {
    require(std::isfinite(p.x) && std::isfinite(p.y) && std::isfinite(v.x) && std::isfinite(v.y) &&
            std::isfinite(n.x) && std::isfinite(n.y), E_OUTOFRANGE, "Flux position, velocity and normal must be finite");
    const double norm = std::hypot(n.x, n.y);
    require(std::isfinite(norm) && std::fabs(norm - 1) <= 128 * std::numeric_limits<double>::epsilon(), E_WRONG,
            "Advective flux requires a unit normal");
}

// LinearAdvectiveFlux (advectiveflux.cpp:272-285) through PhysicalFlux
// (:64-80): value (v.n) u, derivative v.n.
inline void linear_flux(double u, Pt v, Pt n, double& value, double& derivative) {
    require(std::isfinite(u), E_OUTOFRANGE, "Advective trace must be finite");
    derivative = normal_velocity(v, n);
    value = real_value((lc)derivative * u);
}

// advectiveflux.cpp:82-87 (relative roundoff allowance of a speed bound).
inline bool speed_bounds(double bound, double required) {
    return bound >= required || required - bound <= 64 * std::numeric_limits<double>::epsilon() * std::max(bound, required);
}

// IntegrateAdvectiveFlux (advectiveflux.cpp:327-338 via EdgeImpl :180-225 and
// FluxImpl :127-162) for the linear law: sum_q (w_q L / 2) Fhat_q with
// Fhat = (F(uL) + F(uR) - alpha (uR - uL)) / 2 in long double, alpha = the
// endpoint speed max(|F'(uL)|, |F'(uR)|) (local) or the supplied global speed.
inline double integrate_advective_flux(Pt a, Pt b, const std::vector<double>& rp, const std::vector<double>& rw,
                                       const std::vector<Pt>& vel, const std::vector<double>& left,
                                       const std::vector<double>& right, bool global, double global_speed) {
    double length; Pt normal;
    edge_geometry(a, b, length, normal);
    for (const Pt& v : vel) require(std::isfinite(v.x) && std::isfinite(v.y), E_OUTOFRANGE, "Edge velocity must be finite");
    if (global) require(std::isfinite(global_speed) && global_speed >= 0, E_OUTOFRANGE, "Global LF speed must be finite and nonnegative");
    lc sum = 0;
    for (size_t q = 0; q < rp.size(); ++q) {
        const Pt p = map_edge(rp[q], a, b);
        check_point(p, vel[q], normal);
        double fl, dl, fr, dr;
        linear_flux(left[q], vel[q], normal, fl, dl);
        linear_flux(right[q], vel[q], normal, fr, dr);
        const double speed = std::max(std::fabs(dl), std::fabs(dr));
        const double alpha = global ? global_speed : speed;
        require(speed_bounds(alpha, speed), E_OUTOFRANGE, "Supplied global LF speed is smaller than the current local bound");
        const lc jump = (lc)right[q] - left[q];
        const double flux = real_value(((lc)fl + fr - (lc)alpha * jump) / 2);
        const lc weight = (lc)rw[q] * length / 2;
        sum += weight * flux;
    }
    return real_value(sum);
}

// IntegrateAdvectiveBoundaryFlux (advectiveflux.cpp:426-437 via BoundaryImpl
// :227-267): the physical flux of the prescribed state (inflow) or of the
// interior trace (outflow), exactly zero at zero-flux points.
inline double integrate_advective_boundary_flux(Pt a, Pt b, const std::vector<double>& rp, const std::vector<double>& rw,
                                                const std::vector<Pt>& vel, const std::vector<double>& interior,
                                                const std::vector<AdvectBC>& data) {
    double length; Pt normal;
    edge_geometry(a, b, length, normal);
    for (const Pt& v : vel) require(std::isfinite(v.x) && std::isfinite(v.y), E_OUTOFRANGE, "Edge velocity must be finite");
    lc sum = 0;
    for (size_t q = 0; q < rp.size(); ++q) {
        require(data[q].type >= 0 && data[q].type <= 2, E_WRONG, "Unknown advection boundary policy");
        require(std::isfinite(interior[q]), E_OUTOFRANGE, "Interior boundary trace must be finite");
        const Pt p = map_edge(rp[q], a, b);
        check_point(p, vel[q], normal);
        if (data[q].type == 2) continue;
        const bool outflow = data[q].type == 1;
        double f, d;
        linear_flux(outflow ? interior[q] : data[q].value, vel[q], normal, f, d);
        const lc weight = (lc)rw[q] * length / 2;
        sum += weight * f;
    }
    return real_value(sum);
}

}  // namespace orc

#endif

// Host construction of the tables of a general quad mesh (see
// quad_tables.hpp): the vertices of the local rows and the normal-line
// sample spacing of every edge (long double ray exits), and -- with
// cell_tables -- the per-cell tables, whose arithmetic (the uniform
// builder's, geometry.hpp, applied to every cell's own stencil) the GPU
// builder in quad_table_kernels.cu reproduces bit for bit; the library
// builds the per-cell tables on the GPU, and this host form is the one the
// GPU tables are checked against.
#include "quad_tables.hpp"
#include "geometry.hpp"

#include "../../include/mantlepar/mp.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>

namespace mp {
namespace {

using namespace geo;

struct VertexMesh {
    int nx, ny;
    const double* xy;
    V2 vert(int I, int J) const {
        const size_t k = (size_t)J * (nx + 1) + I;
        return V2{xy[2 * k], xy[2 * k + 1]};
    }
    Quad cell(int I, int J) const { return Quad{{vert(I, J), vert(I + 1, J), vert(I + 1, J + 1), vert(I, J + 1)}}; }
};

// Corner average of a quad, formed like a stencil centre (anchor + mean offset).
V2 corner_centre(const Quad& q) {
    double off[2] = {0, 0};
    for (const V2& p : q) { off[0] += (p.x - q[0].x) / 4; off[1] += (p.y - q[0].y) / 4; }
    return V2{q[0].x + off[0], q[0].y + off[1]};
}

// Coefficients of a Q2 polynomial in (xi + dx, eta + dy), m = j*3 + i,
// re-expanded in (xi, eta): binomial expansion per axis.
void shift_q2(const double* a, double dx, double dy, double* out) {
    const double bin[3][3] = {{1, 0, 0}, {1, 1, 0}, {1, 2, 1}};
    double px[3] = {1, dx, dx * dx}, py[3] = {1, dy, dy * dy};
    for (int jn = 0; jn < 3; ++jn)
        for (int in = 0; in < 3; ++in) {
            double s = 0;
            for (int j = jn; j < 3; ++j)
                for (int i = in; i < 3; ++i) s += a[j * 3 + i] * bin[i][in] * px[i - in] * bin[j][jn] * py[j - jn];
            out[jn * 3 + in] = s;
        }
}

void fold(const std::vector<double>& S, int n, int first, double* out) {
    int k = 0;
    for (int r = first; r < n; ++r)
        for (int c = r; c < n; ++c) out[k++] = c == r ? S[(size_t)r * n + r] : 2.0 * S[(size_t)r * n + c];
}

// Normal-line sample spacing of the oriented edge a->b at the 5 Gauss points
// (diffusiveflux.cpp:255-334: the available ray distance inside the left
// cell, and inside the right one when there is one, times extent 0.9 and
// 2/(N-1) across an interior edge or 1/N at a wall, N = 4).
void edge_spacing(V2 a, V2 b, const Quad& left, const Quad* right, const std::vector<double>& gp, double* sp) {
    const int N = 4;
    const double frac = 0.9;
    const double ddx = b.x - a.x, ddy = b.y - a.y;
    const double scale = std::max(std::fabs(ddx), std::fabs(ddy));
    const double ux = ddx / scale, uy = ddy / scale, norm = std::sqrt(ux * ux + uy * uy);
    const V2 nrm{uy / norm, -ux / norm};
    const int lf = face_index(left, a, b, false), rf = right ? face_index(*right, a, b, true) : 0;
    for (size_t q = 0; q < gp.size(); ++q) {
        const V2 p = lerp_edge(gp[q], a, b);
        double avail = ray_exit(left, lf, p, V2{-nrm.x, -nrm.y});
        if (right) avail = std::min(avail, ray_exit(*right, rf, p, nrm));
        sp[q] = (double)((ld)frac * avail * (right ? 2.0L / (N - 1) : 1.0L / N));
    }
}

template <class F>
int parallel_rows(int rows, int threads, F&& f) {
    int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    nt = std::max(1, std::min(nt, rows));
    std::vector<int> codes(nt, 0);
    auto body = [&](int t) {
        for (int r = (int)((long long)rows * t / nt); r < (int)((long long)rows * (t + 1) / nt); ++r) {
            const int c = f(r);
            if (c) { codes[t] = c; return; }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(body, t);
    body(0);
    for (auto& th : pool) th.join();
    for (int c : codes) if (c) return c;
    return 0;
}

}  // namespace

int mesh_vertices(int nx, int ny, double x0, double x1, double y0, double y1, int family, double perturbation,
                  unsigned long long seed, double* xy) {
    if (nx < 1 || ny < 1 || !xy) return MP_ERR_ARG_SIZ;
    const double L = x1 - x0, H = y1 - y0;
    if (!(std::isfinite(x0) && std::isfinite(y0) && std::isfinite(L) && std::isfinite(H) && L > 0 && H > 0))
        return MP_ERR_ARG_OUTOFRANGE;
    if (family < 0 || family > 2) return MP_ERR_ARG_OUTOFRANGE;
    if (family == 1 && !(std::isfinite(perturbation) && perturbation >= 0 && perturbation < 0.25))
        return MP_ERR_ARG_OUTOFRANGE;
    const int M = nx + 1, N = ny + 1;
    const double hx = L / (double)(M - 1), hy = H / (double)(N - 1);
    const double pi = 3.14159265358979323846;
    auto noise = [](std::uint64_t key) {
        key += UINT64_C(0x9e3779b97f4a7c15);
        key = (key ^ (key >> 30)) * UINT64_C(0xbf58476d1ce4e5b9);
        key = (key ^ (key >> 27)) * UINT64_C(0x94d049bb133111eb);
        key ^= key >> 31;
        return 2.0 * ((double)(key >> 11) * 0x1.0p-53) - 1.0;
    };
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < M; ++i) {
            double px = x0 + (double)i * hx, py = y0 + (double)j * hy;
            if (family == 2) {
                const double s = (double)i / (M - 1), t = (double)j / (N - 1);
                px = x0 + L * std::sin(0.5 * pi * s);
                py = y0 + H * std::sin(0.5 * pi * t);
            } else if (family == 1 && i > 0 && i < M - 1 && j > 0 && j < N - 1) {
                const std::uint64_t index = (std::uint64_t)j * (std::uint64_t)M + (std::uint64_t)i;
                px += perturbation * hx * noise(seed + 2 * index);
                py += perturbation * hy * noise(seed + 2 * index + 1);
            }
            if (i == 0) px = x0;
            if (i == M - 1) px = x0 + L;
            if (j == 0) py = y0;
            if (j == N - 1) py = y0 + H;
            const size_t k = (size_t)j * M + i;
            xy[2 * k] = px;
            xy[2 * k + 1] = py;
        }
    return MP_OK;
}

int validate_quads(int nx, int ny, const double* xy, long long* bad) {
    const VertexMesh m{nx, ny, xy};
    const double tol = 64.0 * std::numeric_limits<double>::epsilon();
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const Quad q = m.cell(i, j);
            double xmin = q[0].x, xmax = xmin, ymin = q[0].y, ymax = ymin;
            bool ok = true;
            for (const V2& p : q) {
                ok = ok && std::isfinite(p.x) && std::isfinite(p.y);
                xmin = std::min(xmin, p.x); xmax = std::max(xmax, p.x);
                ymin = std::min(ymin, p.y); ymax = std::max(ymax, p.y);
            }
            const double sx = xmax - xmin, sy = ymax - ymin;
            ok = ok && std::isfinite(sx) && std::isfinite(sy) && sx > 0 && sy > 0;
            for (int k = 0; ok && k < 4; ++k) {
                const V2 p = q[k], nx_ = q[(k + 1) % 4], pv = q[(k + 3) % 4];
                const double ux = (nx_.x - p.x) / sx, uy = (nx_.y - p.y) / sy;
                const double vx = (pv.x - p.x) / sx, vy = (pv.y - p.y) / sy;
                ok = ux * vy - uy * vx > tol;
            }
            if (!ok) {
                if (bad) *bad = (long long)j * nx + i;
                return MP_ERR_ARG_WRONG;
            }
        }
    if (bad) *bad = -1;
    return MP_OK;
}

int build_quad_tables(int nx, int ny, const double* xy, int threads, QuadTables& t, int row0, int rows,
                      bool cell_tables) {
    if (nx < 2 || ny < 2) return MP_ERR_ARG_SIZ;
    if (rows < 0) { row0 = 0; rows = ny; }
    if (row0 < 0 || rows < 1 || row0 + rows > ny) return MP_ERR_ARG_OUTOFRANGE;
    // Tables of the local rows [row0, row0 + rows) of the global mesh, in local numbering.
    const size_t N = (size_t)nx * rows;
    const size_t NI = (size_t)nx * (rows + 1), NE = NI + (size_t)(nx + 1) * rows;
    t.nx = nx; t.ny = rows;
    t.xy.assign(xy + 2 * (size_t)row0 * (nx + 1), xy + 2 * (size_t)(row0 + rows + 1) * (nx + 1));
    const VertexMesh m{nx, ny, xy};
    std::vector<double> p1, w1, gp, gw;
    gauss_legendre(1, p1, w1);
    gauss_legendre(5, gp, gw);
    for (int q = 0; q < 5; ++q) { t.gq[q] = gp[q]; t.gw[q] = gw[q]; }
    for (int q = 0; q < 3; ++q) { t.gq3[q] = gauss_rule_cached(3).first[q]; t.gw3[q] = gauss_rule_cached(3).second[q]; }
    t.gq1 = p1[0]; t.gw1 = w1[0];
    derivative_weights(4, true, t.dif_c_int);
    derivative_weights(5, false, t.dif_c_bnd);
    t.spacing.assign(5 * NE, 0.0);
    const size_t NC = cell_tables ? N : 0;
    t.G0.assign(kQG0 * NC, 0.0);
    t.S9.assign(kQS9 * NC, 0.0);
    t.T4.assign(kQT4 * NC, 0.0);
    t.S4.assign(kQS4 * NC, 0.0);
    t.geo.assign(kQGeo * NC, 0.0);
    const int offi[4] = {0, 0, -1, -1}, offj[4] = {-1, 0, -1, 0};
    int st = !cell_tables ? 0 : parallel_rows(rows, threads, [&](int jl) -> int {
        const int j = row0 + jl;
        for (int i = 0; i < nx; ++i) {
            const size_t cell = (size_t)jl * nx + i;
            const Quad target = m.cell(i, j);
            const double area = cell_integral(target, p1, w1, [](V2) { return 1.0; });
            if (!(area > 0) || !std::isfinite(area)) return MP_ERR_ARG_WRONG;
            const double h = std::sqrt(area);
            const V2 c = corner_centre(target);
            t.geo[0 * N + cell] = c.x; t.geo[1 * N + cell] = c.y;
            t.geo[2 * N + cell] = h;   t.geo[3 * N + cell] = area;
            const int ci = i == 0 ? 0 : (i == nx - 1 ? 2 : 1), cj = j == 0 ? 0 : (j == ny - 1 ? 2 : 1);
            if (ci == 1 && cj == 1) {
                StencilBuild big;
                if (!big.build(m, i - 1, j - 1, 3, 2, h, -1, -1)) return MP_ERR_ARG_WRONG;
                const double dx = (c.x - big.center.x) / h, dy = (c.y - big.center.y) / h;
                for (int s = 1; s < 9; ++s) {
                    double e[9];
                    shift_q2(&big.coef[(size_t)s * 9], dx, dy, e);
                    for (int mm = 0; mm < 9; ++mm) t.G0[(size_t)((s - 1) * 9 + mm) * N + cell] = e[mm];
                }
                double f[kQS9];
                fold(big.sigma, 9, 1, f);
                for (int k = 0; k < kQS9; ++k) t.S9[(size_t)k * N + cell] = f[k];
            }
            for (int k = 0; k < 4; ++k) {
                const int oi = offi[k], oj = offj[k];
                const bool on = !((oi == 0 && ci == 2) || (oi == -1 && ci == 0) || (oj == 0 && cj == 2) || (oj == -1 && cj == 0));
                if (!on) continue;
                StencilBuild small;
                if (!small.build(m, i + oi, j + oj, 2, 1, h, -oi, -oj)) return MP_ERR_ARG_WRONG;
                const double dx = (c.x - small.center.x) / h, dy = (c.y - small.center.y) / h;
                for (int s = 1; s < 4; ++s) {
                    const double* a = &small.coef[(size_t)s * 4];
                    const double v[4] = {a[0] + a[1] * dx + a[2] * dy + a[3] * dx * dy, a[1] + a[3] * dy,
                                         a[2] + a[3] * dx, a[3]};
                    for (int mm = 0; mm < 4; ++mm) t.T4[(size_t)(k * 12 + (s - 1) * 4 + mm) * N + cell] = v[mm];
                }
                double f[6];
                fold(small.target, 4, 1, f);
                for (int q = 0; q < 6; ++q) t.S4[(size_t)(k * 6 + q) * N + cell] = f[q];
            }
        }
        return 0;
    });
    if (st) return st;
    // Edge spacing in the reference's face orientation (evolve.cpp:230-251):
    // the left cell has the oriented edge counter-clockwise; a wall edge
    // whose canonical left cell is missing is reversed.
    st = parallel_rows(rows + 1, threads, [&](int jl) -> int {
        const int j = row0 + jl;
        for (int i = 0; i < nx; ++i) {           // AlongI edge (i, j)
            const size_t e = (size_t)jl * nx + i;
            const V2 v0 = m.vert(i, j), v1 = m.vert(i + 1, j);
            double sp[5];
            if (j == ny) {
                edge_spacing(v1, v0, m.cell(i, ny - 1), nullptr, gp, sp);
                for (int q = 0; q < 5; ++q) t.spacing[e * 5 + (4 - q)] = sp[q];
            } else {
                const Quad r = j > 0 ? m.cell(i, j - 1) : Quad{};
                edge_spacing(v0, v1, m.cell(i, j), j > 0 ? &r : nullptr, gp, sp);
                for (int q = 0; q < 5; ++q) t.spacing[e * 5 + q] = sp[q];
            }
        }
        if (jl == rows) return 0;
        for (int i = 0; i <= nx; ++i) {          // AlongJ edge (i, j)
            const size_t e = NI + (size_t)jl * (nx + 1) + i;
            const V2 v0 = m.vert(i, j), v1 = m.vert(i, j + 1);
            double sp[5];
            if (i == 0) {
                edge_spacing(v1, v0, m.cell(0, j), nullptr, gp, sp);
                for (int q = 0; q < 5; ++q) t.spacing[e * 5 + (4 - q)] = sp[q];
            } else {
                const Quad r = i < nx ? m.cell(i, j) : Quad{};
                edge_spacing(v0, v1, m.cell(i - 1, j), i < nx ? &r : nullptr, gp, sp);
                for (int q = 0; q < 5; ++q) t.spacing[e * 5 + q] = sp[q];
            }
        }
        return 0;
    });
    return st;
}

}  // namespace mp

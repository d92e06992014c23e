// Device helpers of the general (logically rectangular) quad mesh kernels,
// shared by the transport stage and the preheat: vertex reads, the
// reference's edge and bilinear maps (src/core/integral.cpp:62-121), the
// cell frame, the normal-line diffusion samples, the table-driven
// reconstruction of one field, and the edge orientation of the flux loops.
#ifndef MP_QUAD_DEVICE_CUH
#define MP_QUAD_DEVICE_CUH

#include "common.hpp"
#include "quad_tables.hpp"
#include "stage_device.cuh"

namespace mp {
namespace {

struct P2 {
    double x, y;
};

__device__ __forceinline__ P2 vtx(const QuadDev& q, int nx, int I, int J) {
    const size_t k = (size_t)J * (nx + 1) + I;
    return P2{__ldg(q.xy + 2 * k), __ldg(q.xy + 2 * k + 1)};
}
// integral.cpp:91-121: edge interpolation, bilinear map, Jacobian on [-1,1]^2.
__device__ __forceinline__ P2 lerp_edge(double r, P2 a, P2 b) {
    const double s = 0.5 * (1.0 - r), t = 0.5 * (1.0 + r);
    return P2{s * a.x + t * b.x, s * a.y + t * b.y};
}
__device__ __forceinline__ P2 bilinear(double rx, double ry, const P2* c) {
    return lerp_edge(ry, lerp_edge(rx, c[0], c[1]), lerp_edge(rx, c[3], c[2]));
}
__device__ __forceinline__ double jacobian(double rx, double ry, const P2* c) {
    const double s = 0.5 * (1.0 + rx), t = 0.5 * (1.0 + ry);
    const double xi_x = 0.5 * ((1.0 - t) * (c[1].x - c[0].x) + t * (c[2].x - c[3].x));
    const double xi_y = 0.5 * ((1.0 - t) * (c[1].y - c[0].y) + t * (c[2].y - c[3].y));
    const double et_x = 0.5 * ((1.0 - s) * (c[3].x - c[0].x) + s * (c[2].x - c[1].x));
    const double et_y = 0.5 * ((1.0 - s) * (c[3].y - c[0].y) + s * (c[2].y - c[1].y));
    return xi_x * et_y - xi_y * et_x;
}
// integral.cpp:62-89: length and unit normal (dy, -dx)/length of a -> b.
__device__ __forceinline__ void edge_geometry(P2 a, P2 b, double& len, P2& n) {
    const double dx = b.x - a.x, dy = b.y - a.y;
    const double scale = fmax(fabs(dx), fabs(dy));
    const double ux = dx / scale, uy = dy / scale;
    const double norm = sqrt(ux * ux + uy * uy);
    len = scale * norm;
    n = P2{uy / norm, -ux / norm};
}
// Full Q2 form, monomial m = j*3 + i of xi^i eta^j.
__device__ __forceinline__ double q2v(const double* D, double x, double y) {
    const double r0 = D[0] + x * (D[1] + x * D[2]);
    const double r1 = D[3] + x * (D[4] + x * D[5]);
    const double r2 = D[6] + x * (D[7] + x * D[8]);
    return r0 + y * (r1 + y * r2);
}

// The cell's frame: centre, 1/h, and corners.
struct CellFrame {
    double cx, cy, inv_h, area;
    P2 c[4];
};
__device__ __forceinline__ CellFrame cell_frame(const QuadDev& q, int nx, size_t N, long long cell) {
    const int i = (int)(cell % nx), j = (int)(cell / nx);
    CellFrame f;
    f.cx = __ldg(q.geo + cell);
    f.cy = __ldg(q.geo + N + cell);
    f.inv_h = 1.0 / __ldg(q.geo + 2 * N + cell);
    f.area = __ldg(q.geo + 3 * N + cell);
    f.c[0] = vtx(q, nx, i, j); f.c[1] = vtx(q, nx, i + 1, j);
    f.c[2] = vtx(q, nx, i + 1, j + 1); f.c[3] = vtx(q, nx, i, j + 1);
    return f;
}

// Edge e of cell (i, j) in counter-clockwise order (0 bottom, 1 right, 2 top,
// 3 left): its local edge id, whether it is a wall, and whether the cell's
// point order runs against the canonical one. Local rows j of a mesh whose
// local row 0 is global row gj0 of gny global rows.
__device__ __forceinline__ void cell_edge(int nx, int ny, int i, int j, int gj0, int gny, int e, long long& id,
                                          bool& wall, bool& rev) {
    const long long nI = (long long)nx * (ny + 1);
    const int gj = gj0 + j;
    if (e == 0) { id = (long long)j * nx + i; wall = gj == 0; rev = false; }
    else if (e == 1) { id = nI + (long long)j * (nx + 1) + i + 1; wall = i == nx - 1; rev = false; }
    else if (e == 2) { id = (long long)(j + 1) * nx + i; wall = gj == gny - 1; rev = true; }
    else { id = nI + (long long)j * (nx + 1) + i; wall = i == 0; rev = true; }
}

// Visit every normal-line diffusion sample on this cell's side of its four
// edges (diffusiveflux.cpp:255-334, 4 samples; interior edges 2 on each side
// at offsets -1.5, -0.5 spacings from the edge, wall edges 4 at -4..-1).
template <class F>
__device__ __forceinline__ void visit_samples(const QuadDev& q, int nx, int ny, int gj0, int gny, int i, int j,
                                              const CellFrame& f, F&& visit) {
    for (int e = 0; e < 4; ++e) {
        long long id;
        bool wall, rev;
        cell_edge(nx, ny, i, j, gj0, gny, e, id, wall, rev);
        const P2 a = f.c[e], b = f.c[(e + 1) & 3];
        double len;
        P2 n;
        edge_geometry(a, b, len, n);
        for (int k = 0; k < kNQ; ++k) {
            const P2 p = lerp_edge(q.gq[k], a, b);
            const double sp = __ldg(q.sp + id * kNQ + (rev ? kNQ - 1 - k : k));
            const int ns = wall ? 4 : 2;
            for (int s = 0; s < ns; ++s) {
                const double d = (wall ? (double)(s - 4) : (double)s - 1.5) * sp;
                visit(P2{p.x + d * n.x, p.y + d * n.y});
            }
        }
    }
}

// Folded smoothness row offsets: entry (r, c >= r) of an n x n form.
__device__ __forceinline__ int fold_at(int n, int r, int c) { return r * n - (r * (r - 1)) / 2 + (c - r); }

// smoothness<>'s decision for a chain that failed its range test (roundoff
// at sigma ~ 0, or bad data), out of line: form n x n, folded entries at
// base[k * stride].
template <int NN>
__device__ __noinline__ double smoothness_out_of_line(const double* base, size_t stride, const double* diff) {
    auto SF = [&](int k) { return __ldg(base + (size_t)k * stride); };
    auto S = [&](int r, int c) { const double v = SF(fold_at(NN, r, c)); return r == c ? v : 0.5 * v; };
    return smoothness<double, NN>(SF, S, diff);
}

// The deviation polynomials D[f] of F fields from their 3x3 neighbourhoods
// u[f] with the cell's own tables (same candidate set, weights and clipping
// as reconstruct() of the uniform path). The fields share the cell's
// stencils and so its tables: every table entry is read once and applied to
// each field, and per field the operations run in the same order whatever F
// is, so a field's result does not depend on the fields reconstructed with
// it. For F > 1 smoothness<>'s FMA chains are formed here for all fields at
// once, and a chain that fails its range test is decided by smoothness<> out
// of line (it forms the same chain again, then the term-by-term sum), so
// that the rare path does not cost the multi-field form registers; F = 1
// calls smoothness<> inline. Returns the first failure in field order.
template <int F>
__device__ __forceinline__ int reconstruct_quad(const QuadDev& q, size_t N, long long cell, int ci, int cj,
                                                double eA, const double (&u)[F][3][3], double (&D)[F][9]) {
    double d[F][3][3];
#pragma unroll
    for (int f = 0; f < F; ++f)
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) d[f][a][b] = u[f][a][b] - u[f][1][1];
    const int offi[4] = {0, 0, -1, -1}, offj[4] = {-1, 0, -1, 0};
    bool on[5];
    on[0] = (ci == 1 && cj == 1);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        on[k + 1] = !((offi[k] == 0 && ci == 2) || (offi[k] == -1 && ci == 0) || (offj[k] == 0 && cj == 2) ||
                      (offj[k] == -1 && cj == 0));
    double sg[F][5];
    int st[F];
#pragma unroll
    for (int f = 0; f < F; ++f) st[f] = 0;
    auto fast_ok = [](double v) { return v >= 0.0 && v < INFINITY; };
    if (on[0]) {
        double fd[F][8];
#pragma unroll
        for (int f = 0; f < F; ++f)
#pragma unroll
            for (int c = 1; c < 9; ++c) fd[f][c - 1] = d[f][c / 3][c % 3] - d[f][0][0];
        auto SF = [&](int k) { return __ldg(q.S9 + (size_t)k * N + cell); };
        auto S = [&](int r, int c) { const double v = SF(fold_at(8, r, c)); return r == c ? v : 0.5 * v; };
        if constexpr (F == 1) {
            sg[0][0] = smoothness<double, 8>(SF, S, fd[0]);
        } else {
            double sum[F];
#pragma unroll
            for (int f = 0; f < F; ++f) sum[f] = 0;
            int k = 0;
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const double s0 = SF(k++);
                double t[F];
#pragma unroll
                for (int f = 0; f < F; ++f) t[f] = s0 * fd[f][r];
#pragma unroll
                for (int c = r + 1; c < 8; ++c) {
                    const double sv = SF(k++);
#pragma unroll
                    for (int f = 0; f < F; ++f) t[f] = fma(sv, fd[f][c], t[f]);
                }
#pragma unroll
                for (int f = 0; f < F; ++f) sum[f] = fma(fd[f][r], t[f], sum[f]);
            }
#pragma unroll
            for (int f = 0; f < F; ++f)
                sg[f][0] = fast_ok(sum[f]) ? sum[f] : smoothness_out_of_line<8>(q.S9 + cell, N, fd[f]);
        }
#pragma unroll
        for (int f = 0; f < F; ++f)
            if (sg[f][0] < 0.0) st[f] = MP_ERR_FP;
    } else {
#pragma unroll
        for (int f = 0; f < F; ++f) sg[f][0] = 0;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!on[k + 1]) {
#pragma unroll
            for (int f = 0; f < F; ++f) sg[f][k + 1] = 0;
            continue;
        }
        const int oi = offi[k], oj = offj[k];
        double fd[F][3];
#pragma unroll
        for (int f = 0; f < F; ++f) {
            const double a0 = d[f][1 + oj][1 + oi];
#pragma unroll
            for (int c = 1; c < 4; ++c) fd[f][c - 1] = d[f][1 + oj + c / 2][1 + oi + c % 2] - a0;
        }
        auto SF = [&](int m) { return __ldg(q.S4 + (size_t)(k * 6 + m) * N + cell); };
        auto S = [&](int r, int c) { const double v = SF(fold_at(3, r, c)); return r == c ? v : 0.5 * v; };
        if constexpr (F == 1) {
            sg[0][k + 1] = smoothness<double, 3>(SF, S, fd[0]);
        } else {
            double sum[F];
#pragma unroll
            for (int f = 0; f < F; ++f) sum[f] = 0;
            int m = 0;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const double s0 = SF(m++);
                double t[F];
#pragma unroll
                for (int f = 0; f < F; ++f) t[f] = s0 * fd[f][r];
#pragma unroll
                for (int c = r + 1; c < 3; ++c) {
                    const double sv = SF(m++);
#pragma unroll
                    for (int f = 0; f < F; ++f) t[f] = fma(sv, fd[f][c], t[f]);
                }
#pragma unroll
                for (int f = 0; f < F; ++f) sum[f] = fma(fd[f][r], t[f], sum[f]);
            }
#pragma unroll
            for (int f = 0; f < F; ++f)
                sg[f][k + 1] = fast_ok(sum[f]) ? sum[f]
                                               : smoothness_out_of_line<3>(q.S4 + (size_t)k * 6 * N + cell, N, fd[f]);
        }
#pragma unroll
        for (int f = 0; f < F; ++f)
            if (sg[f][k + 1] < 0.0) st[f] = MP_ERR_FP;
    }
    double w[F][5];
#pragma unroll
    for (int f = 0; f < F; ++f) weights(sg[f], on, eA, w[f]);
#pragma unroll
    for (int f = 0; f < F; ++f)
        if (!isfinite(w[f][0] + w[f][1] + w[f][2] + w[f][3] + w[f][4])) st[f] = MP_ERR_FP;
#pragma unroll
    for (int f = 0; f < F; ++f)
#pragma unroll
        for (int mm = 0; mm < 9; ++mm) D[f][mm] = 0;
    if (on[0]) {
        double fd[F][8];
#pragma unroll
        for (int f = 0; f < F; ++f)
#pragma unroll
            for (int c = 1; c < 9; ++c) fd[f][c - 1] = d[f][c / 3][c % 3] - d[f][0][0];
#pragma unroll
        for (int mm = 0; mm < 9; ++mm) {
            double v[F];
#pragma unroll
            for (int f = 0; f < F; ++f) v[f] = mm == 0 ? d[f][0][0] : 0.0;
#pragma unroll
            for (int c = 1; c < 9; ++c) {
                const double g = __ldg(q.G0 + (size_t)((c - 1) * 9 + mm) * N + cell);
#pragma unroll
                for (int f = 0; f < F; ++f) v[f] += fd[f][c - 1] * g;
            }
#pragma unroll
            for (int f = 0; f < F; ++f) D[f][mm] = w[f][0] * v[f];
        }
    }
    const int slot[4] = {0, 1, 3, 4};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!on[k + 1]) continue;
        const int oi = offi[k], oj = offj[k];
        double a0[F], fd[F][3];
#pragma unroll
        for (int f = 0; f < F; ++f) {
            a0[f] = d[f][1 + oj][1 + oi];
#pragma unroll
            for (int c = 1; c < 4; ++c) fd[f][c - 1] = d[f][1 + oj + c / 2][1 + oi + c % 2] - a0[f];
        }
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) {
            double v[F];
#pragma unroll
            for (int f = 0; f < F; ++f) v[f] = mm == 0 ? a0[f] : 0.0;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double tv = __ldg(q.T4 + (size_t)(k * 12 + c * 4 + mm) * N + cell);
#pragma unroll
                for (int f = 0; f < F; ++f) v[f] += fd[f][c] * tv;
            }
#pragma unroll
            for (int f = 0; f < F; ++f) D[f][slot[mm]] += w[f][k + 1] * v[f];
        }
    }
#pragma unroll
    for (int f = 0; f < F; ++f)
        if (st[f]) return st[f];
    return 0;
}

// Left/right cells and oriented vertices of edge e (evolve.cpp:230-251).
struct QuadEdge {
    bool horizontal, boundary, reverse;
    long long L, R;
    int wall;
    P2 a, b;
};
__device__ __forceinline__ QuadEdge quad_edge(const QuadDev& q, int nx, int ny, int gj0, int gny, long long e) {
    const long long nI = (long long)nx * (ny + 1);
    QuadEdge g;
    g.R = -1;
    g.wall = -1;
    P2 v0, v1;
    if (e < nI) {
        const int i = (int)(e % nx), j = (int)(e / nx);
        const int gj = gj0 + j;
        g.horizontal = true;
        g.boundary = gj == 0 || gj == gny;
        g.reverse = gj == gny;
        g.L = g.reverse ? (long long)(j - 1) * nx + i : (long long)j * nx + i;
        if (!g.boundary) g.R = (long long)(j - 1) * nx + i;
        else g.wall = gj == 0 ? 0 : 1;
        v0 = vtx(q, nx, i, j); v1 = vtx(q, nx, i + 1, j);
    } else {
        const long long k = e - nI;
        const int i = (int)(k % (nx + 1)), j = (int)(k / (nx + 1));
        g.horizontal = false;
        g.boundary = i == 0 || i == nx;
        g.reverse = i == 0;
        g.L = g.reverse ? (long long)j * nx : (long long)j * nx + (i - 1);
        if (!g.boundary) g.R = (long long)j * nx + i;
        else g.wall = i == 0 ? 2 : 3;
        v0 = vtx(q, nx, i, j); v1 = vtx(q, nx, i, j + 1);
    }
    g.a = g.reverse ? v1 : v0;
    g.b = g.reverse ? v0 : v1;
    return g;
}

}  // namespace
}  // namespace mp

#endif

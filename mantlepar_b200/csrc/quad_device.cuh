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

// One field's deviation polynomial D from the 3x3 neighbourhood with the
// cell's own tables (same candidate set, weights and clipping as
// reconstruct() of the uniform path).
__device__ __forceinline__ int reconstruct_quad(const QuadDev& q, size_t N, long long cell, int ci, int cj,
                                                double eA, const double (&u)[3][3], double (&D)[9]) {
    double d[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) d[a][b] = u[a][b] - u[1][1];
    const int offi[4] = {0, 0, -1, -1}, offj[4] = {-1, 0, -1, 0};
    bool on[5];
    on[0] = (ci == 1 && cj == 1);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        on[k + 1] = !((offi[k] == 0 && ci == 2) || (offi[k] == -1 && ci == 0) || (offj[k] == 0 && cj == 2) ||
                      (offj[k] == -1 && cj == 0));
    double sig[5];
    int st = 0;
    if (on[0]) {
        double diff[8];
#pragma unroll
        for (int c = 1; c < 9; ++c) diff[c - 1] = d[c / 3][c % 3] - d[0][0];
        auto SF = [&](int k) { return __ldg(q.S9 + (size_t)k * N + cell); };
        auto S = [&](int r, int c) { const double v = SF(fold_at(8, r, c)); return r == c ? v : 0.5 * v; };
        sig[0] = smoothness<double, 8>(SF, S, diff);
        if (sig[0] < 0.0) st = MP_ERR_FP;
    } else {
        sig[0] = 0;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!on[k + 1]) { sig[k + 1] = 0; continue; }
        const int oi = offi[k], oj = offj[k];
        const double a0 = d[1 + oj][1 + oi];
        double diff[3];
#pragma unroll
        for (int c = 1; c < 4; ++c) diff[c - 1] = d[1 + oj + c / 2][1 + oi + c % 2] - a0;
        auto SF = [&](int m) { return __ldg(q.S4 + (size_t)(k * 6 + m) * N + cell); };
        auto S = [&](int r, int c) { const double v = SF(fold_at(3, r, c)); return r == c ? v : 0.5 * v; };
        sig[k + 1] = smoothness<double, 3>(SF, S, diff);
        if (sig[k + 1] < 0.0) st = MP_ERR_FP;
    }
    double w[5];
    weights<double>(sig, on, eA, w);
    if (!isfinite(w[0] + w[1] + w[2] + w[3] + w[4])) st = MP_ERR_FP;
#pragma unroll
    for (int m = 0; m < 9; ++m) D[m] = 0;
    if (on[0]) {
        double diff[8];
#pragma unroll
        for (int c = 1; c < 9; ++c) diff[c - 1] = d[c / 3][c % 3] - d[0][0];
#pragma unroll
        for (int m = 0; m < 9; ++m) {
            double v = m == 0 ? d[0][0] : 0.0;
#pragma unroll
            for (int c = 1; c < 9; ++c) v += diff[c - 1] * __ldg(q.G0 + (size_t)((c - 1) * 9 + m) * N + cell);
            D[m] = w[0] * v;
        }
    }
    const int slot[4] = {0, 1, 3, 4};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!on[k + 1]) continue;
        const int oi = offi[k], oj = offj[k];
        const double a0 = d[1 + oj][1 + oi];
        double diff[3];
#pragma unroll
        for (int c = 1; c < 4; ++c) diff[c - 1] = d[1 + oj + c / 2][1 + oi + c % 2] - a0;
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) {
            double v = mm == 0 ? a0 : 0.0;
#pragma unroll
            for (int c = 0; c < 3; ++c) v += diff[c] * __ldg(q.T4 + (size_t)(k * 12 + c * 4 + mm) * N + cell);
            D[slot[mm]] += w[k + 1] * v;
        }
    }
    return st;
}

// Both fields' deviation polynomials (H and C share the cell's stencils,
// so they share its tables) with one read of every table entry: per field
// the operations and their order are those of reconstruct_quad, so DH and DC
// equal two reconstruct_quad calls bit for bit. Returns the first failure
// in field order (H, then C).
__device__ __forceinline__ int reconstruct_quad2(const QuadDev& q, size_t N, long long cell, int ci, int cj,
                                                 double eA, const double (&uH)[3][3], const double (&uC)[3][3],
                                                 double (&DH)[9], double (&DC)[9]) {
    double dH[3][3], dC[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            dH[a][b] = uH[a][b] - uH[1][1];
            dC[a][b] = uC[a][b] - uC[1][1];
        }
    const int offi[4] = {0, 0, -1, -1}, offj[4] = {-1, 0, -1, 0};
    bool on[5];
    on[0] = (ci == 1 && cj == 1);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        on[k + 1] = !((offi[k] == 0 && ci == 2) || (offi[k] == -1 && ci == 0) || (offj[k] == 0 && cj == 2) ||
                      (offj[k] == -1 && cj == 0));
    double sgH[5], sgC[5];
    int stH = 0, stC = 0;
    auto fast_ok = [](double v) { return v >= 0.0 && v < INFINITY; };
    if (on[0]) {
        double fH[8], fC[8];
#pragma unroll
        for (int c = 1; c < 9; ++c) {
            fH[c - 1] = dH[c / 3][c % 3] - dH[0][0];
            fC[c - 1] = dC[c / 3][c % 3] - dC[0][0];
        }
        auto SF = [&](int k) { return __ldg(q.S9 + (size_t)k * N + cell); };
        auto S = [&](int r, int c) { const double v = SF(fold_at(8, r, c)); return r == c ? v : 0.5 * v; };
        // The FMA chains of smoothness<double, 8> for both fields.
        double sumH = 0, sumC = 0;
        int k = 0;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const double s0 = SF(k++);
            double tH = s0 * fH[r], tC = s0 * fC[r];
#pragma unroll
            for (int c = r + 1; c < 8; ++c) {
                const double sv = SF(k++);
                tH = fma(sv, fH[c], tH);
                tC = fma(sv, fC[c], tC);
            }
            sumH = fma(fH[r], tH, sumH);
            sumC = fma(fC[r], tC, sumC);
        }
        sgH[0] = fast_ok(sumH) ? sumH : smoothness<double, 8>(SF, S, fH);
        sgC[0] = fast_ok(sumC) ? sumC : smoothness<double, 8>(SF, S, fC);
        if (sgH[0] < 0.0) stH = MP_ERR_FP;
        if (sgC[0] < 0.0) stC = MP_ERR_FP;
    } else {
        sgH[0] = 0;
        sgC[0] = 0;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!on[k + 1]) { sgH[k + 1] = 0; sgC[k + 1] = 0; continue; }
        const int oi = offi[k], oj = offj[k];
        const double aH = dH[1 + oj][1 + oi], aC = dC[1 + oj][1 + oi];
        double fH[3], fC[3];
#pragma unroll
        for (int c = 1; c < 4; ++c) {
            fH[c - 1] = dH[1 + oj + c / 2][1 + oi + c % 2] - aH;
            fC[c - 1] = dC[1 + oj + c / 2][1 + oi + c % 2] - aC;
        }
        auto SF = [&](int m) { return __ldg(q.S4 + (size_t)(k * 6 + m) * N + cell); };
        auto S = [&](int r, int c) { const double v = SF(fold_at(3, r, c)); return r == c ? v : 0.5 * v; };
        double sumH = 0, sumC = 0;
        int m = 0;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const double s0 = SF(m++);
            double tH = s0 * fH[r], tC = s0 * fC[r];
#pragma unroll
            for (int c = r + 1; c < 3; ++c) {
                const double sv = SF(m++);
                tH = fma(sv, fH[c], tH);
                tC = fma(sv, fC[c], tC);
            }
            sumH = fma(fH[r], tH, sumH);
            sumC = fma(fC[r], tC, sumC);
        }
        sgH[k + 1] = fast_ok(sumH) ? sumH : smoothness<double, 3>(SF, S, fH);
        sgC[k + 1] = fast_ok(sumC) ? sumC : smoothness<double, 3>(SF, S, fC);
        if (sgH[k + 1] < 0.0) stH = MP_ERR_FP;
        if (sgC[k + 1] < 0.0) stC = MP_ERR_FP;
    }
    double wH[5], wC[5];
    weights<double>(sgH, on, eA, wH);
    weights<double>(sgC, on, eA, wC);
    if (!isfinite(wH[0] + wH[1] + wH[2] + wH[3] + wH[4])) stH = MP_ERR_FP;
    if (!isfinite(wC[0] + wC[1] + wC[2] + wC[3] + wC[4])) stC = MP_ERR_FP;
#pragma unroll
    for (int m = 0; m < 9; ++m) { DH[m] = 0; DC[m] = 0; }
    if (on[0]) {
        double fH[8], fC[8];
#pragma unroll
        for (int c = 1; c < 9; ++c) {
            fH[c - 1] = dH[c / 3][c % 3] - dH[0][0];
            fC[c - 1] = dC[c / 3][c % 3] - dC[0][0];
        }
#pragma unroll
        for (int m = 0; m < 9; ++m) {
            double vH = m == 0 ? dH[0][0] : 0.0, vC = m == 0 ? dC[0][0] : 0.0;
#pragma unroll
            for (int c = 1; c < 9; ++c) {
                const double g = __ldg(q.G0 + (size_t)((c - 1) * 9 + m) * N + cell);
                vH += fH[c - 1] * g;
                vC += fC[c - 1] * g;
            }
            DH[m] = wH[0] * vH;
            DC[m] = wC[0] * vC;
        }
    }
    const int slot[4] = {0, 1, 3, 4};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!on[k + 1]) continue;
        const int oi = offi[k], oj = offj[k];
        const double aH = dH[1 + oj][1 + oi], aC = dC[1 + oj][1 + oi];
        double fH[3], fC[3];
#pragma unroll
        for (int c = 1; c < 4; ++c) {
            fH[c - 1] = dH[1 + oj + c / 2][1 + oi + c % 2] - aH;
            fC[c - 1] = dC[1 + oj + c / 2][1 + oi + c % 2] - aC;
        }
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) {
            double vH = mm == 0 ? aH : 0.0, vC = mm == 0 ? aC : 0.0;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double t = __ldg(q.T4 + (size_t)(k * 12 + c * 4 + mm) * N + cell);
                vH += fH[c] * t;
                vC += fC[c] * t;
            }
            DH[slot[mm]] += wH[k + 1] * vH;
            DC[slot[mm]] += wC[k + 1] * vC;
        }
    }
    return stH ? stH : stC;
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

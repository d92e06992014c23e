// Per-cell stage tables of a general quad mesh, built on the GPU: one thread
// per cell runs the host builder's arithmetic (geometry.hpp: stencil centre,
// Gauss moments of the monomials, the inverse by partial-pivoting
// elimination, the reference-square and target-cell smoothness forms;
// TensorStencilPoly::Initialize / SetTargetSmoothness,
// src/mlweno/tensorstencilpoly.cpp:146-231,318-398) for the cell's 3x3 and
// 2x2 candidates, re-expands them into the cell's frame and writes the
// tables of quad_tables.hpp. This file is compiled without FMA contraction,
// so every table entry is rounded as the host code rounds it.
#include "quad_tables.hpp"

#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "../../include/mantlepar/mp.h"

namespace mp {
namespace {

struct DV2 {
    double x, y;
};

// The Gauss rules the builder uses: 3 points (moments, smoothness) and 1 (areas).
struct Rules {
    double p3[3], w3[3];
    double p1, w1;
};

__device__ __forceinline__ DV2 vtx(const double* xy, int nx, int I, int J) {
    const size_t k = (size_t)J * (nx + 1) + I;
    return DV2{xy[2 * k], xy[2 * k + 1]};
}
__device__ __forceinline__ void cell_quad(const double* xy, int nx, int I, int J, DV2* q) {
    q[0] = vtx(xy, nx, I, J); q[1] = vtx(xy, nx, I + 1, J);
    q[2] = vtx(xy, nx, I + 1, J + 1); q[3] = vtx(xy, nx, I, J + 1);
}
__device__ __forceinline__ DV2 lerp_edge(double r, DV2 a, DV2 b) {
    const double s = 0.5 * (1.0 - r), t = 0.5 * (1.0 + r);
    return DV2{s * a.x + t * b.x, s * a.y + t * b.y};
}
__device__ __forceinline__ DV2 bilinear(double rx, double ry, const DV2* c) {
    return lerp_edge(ry, lerp_edge(rx, c[0], c[1]), lerp_edge(rx, c[3], c[2]));
}
__device__ __forceinline__ double jacobian(double rx, double ry, const DV2* c) {
    const double s = 0.5 * (1.0 + rx), t = 0.5 * (1.0 + ry);
    const double xi_x = 0.5 * ((1.0 - t) * (c[1].x - c[0].x) + t * (c[2].x - c[3].x));
    const double xi_y = 0.5 * ((1.0 - t) * (c[1].y - c[0].y) + t * (c[2].y - c[3].y));
    const double et_x = 0.5 * ((1.0 - s) * (c[3].x - c[0].x) + s * (c[2].x - c[1].x));
    const double et_y = 0.5 * ((1.0 - s) * (c[3].y - c[0].y) + s * (c[2].y - c[1].y));
    return xi_x * et_y - xi_y * et_x;
}
__device__ __forceinline__ double power(double x, int k) {
    double r = 1;
    for (int i = 0; i < k; ++i) r *= x;
    return r;
}
__device__ __forceinline__ double falling(int degree, int d) {
    double r = 1;
    for (int k = 0; k < d; ++k) r *= (double)(degree - k);
    return r;
}
__device__ double horner_derivative(const double* c, int si, int sj, double x, double y, int dx, int dy) {
    if (dx >= si || dy >= sj) return 0;
    double result = 0;
    for (int j = sj; j-- > dy;) {
        double row = 0;
        for (int i = si; i-- > dx;) row = row * x + c[j * si + i] * falling(i, dx);
        result = result * y + row * falling(j, dy);
    }
    return result;
}
// sum_q w_a w_b J f(x): f = x^i y^j (i, j >= 0), or 1 with i = j = 0.
__device__ double cell_moment(const DV2* c, const double* p, const double* w, int n, int i, int j) {
    double sum = 0.0;
    for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) {
            const DV2 x = bilinear(p[a], p[b], c);
            sum += w[a] * w[b] * jacobian(p[a], p[b], c) * (power(x.x, i) * power(x.y, j));
        }
    return sum;
}
__device__ double cell_area(const DV2* c, const double* p, const double* w, int n) {
    double sum = 0.0;
    for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) sum += w[a] * w[b] * jacobian(p[a], p[b], c) * 1.0;
    return sum;
}
// X = A^-1 by elimination with partial pivoting (A is overwritten).
__device__ bool solve_identity(int n, double* A, double* X) {
    for (int k = 0; k < n * n; ++k) X[k] = 0.0;
    for (int k = 0; k < n; ++k) X[k * n + k] = 1.0;
    for (int k = 0; k < n; ++k) {
        int piv = k;
        for (int r = k + 1; r < n; ++r) if (fabs(A[r * n + k]) > fabs(A[piv * n + k])) piv = r;
        if (A[piv * n + k] == 0.0) return false;
        if (piv != k)
            for (int c = 0; c < n; ++c) {
                const double a = A[k * n + c], x = X[k * n + c];
                A[k * n + c] = A[piv * n + c]; X[k * n + c] = X[piv * n + c];
                A[piv * n + c] = a; X[piv * n + c] = x;
            }
        for (int r = k + 1; r < n; ++r) {
            const double f = A[r * n + k] / A[k * n + k];
            for (int c = k + 1; c < n; ++c) A[r * n + c] -= f * A[k * n + c];
            for (int c = 0; c < n; ++c) X[r * n + c] -= f * X[k * n + c];
        }
    }
    for (int k = n - 1; k >= 0; --k)
        for (int c = 0; c < n; ++c) {
            double s = X[k * n + c];
            for (int j = k + 1; j < n; ++j) s -= A[k * n + j] * X[j * n + c];
            X[k * n + c] = s / A[k * n + k];
        }
    return true;
}

// Smoothness form of the basis coef (n = S*S) over the quad nc with a
// 3-point rule: sum_q w w (J/area) sum_{0 < dx+dy <= order} d_c d_r.
template <int S>
__device__ void smoothness(const DV2* nc, const Rules& R, int order, const double* coef, double* m) {
    constexpr int n = S * S;
    const double area = cell_area(nc, R.p3, R.w3, 3);
    for (int k = 0; k < n * n; ++k) m[k] = 0.0;
    double der[n];
    for (int qy = 0; qy < 3; ++qy)
        for (int qx = 0; qx < 3; ++qx) {
            const DV2 x = bilinear(R.p3[qx], R.p3[qy], nc);
            const double weight = R.w3[qx] * R.w3[qy] * (jacobian(R.p3[qx], R.p3[qy], nc) / area);
            for (int dy = 0; dy < S; ++dy)
                for (int dx = 0; dx < S; ++dx) {
                    if (dx + dy == 0 || dx + dy > order) continue;
                    for (int c = 0; c < n; ++c) der[c] = horner_derivative(coef + c * n, S, S, x.x, x.y, dx, dy);
                    for (int r2 = 0; r2 < n; ++r2)
                        for (int c = 0; c <= r2; ++c) m[r2 * n + c] += weight * der[r2] * der[c];
                }
        }
    for (int r2 = 0; r2 < n; ++r2)
        for (int c = 0; c <= r2; ++c) m[c * n + r2] = m[r2 * n + c];
}

// Basis coefficients coef[cell*n + m] of the S x S stencil with lower-left
// cell (I0, J0), normalised by h, its centre, and (ti >= 0) the smoothness
// form on its cell (ti, tj); without a target cell, on the reference square.
template <int S>
__device__ bool stencil(const double* xy, int nx, int I0, int J0, int order, double h, int ti, int tj, const Rules& R,
                        double* coef, double* form, DV2& center) {
    constexpr int n = S * S;
    DV2 cells[n][4];
    for (int j = 0; j < S; ++j)
        for (int i = 0; i < S; ++i) cell_quad(xy, nx, I0 + i, J0 + j, cells[j * S + i]);
    const DV2 anchor = cells[0][0];
    const DV2 outer[4] = {anchor, cells[S - 1][1], cells[n - 1][2], cells[(S - 1) * S][3]};
    double off[2] = {0, 0};
    for (int k = 0; k < 4; ++k) { off[0] += (outer[k].x - anchor.x) / 4; off[1] += (outer[k].y - anchor.y) / 4; }
    center = DV2{anchor.x + off[0], anchor.y + off[1]};
    for (int c = 0; c < n; ++c)
        for (int k = 0; k < 4; ++k) cells[c][k] = DV2{(cells[c][k].x - center.x) / h, (cells[c][k].y - center.y) / h};
    double M[n * n], X[n * n];
    for (int c = 0; c < n; ++c) {
        const double area = cell_area(cells[c], R.p3, R.w3, 3);
        for (int j = 0; j < S; ++j)
            for (int i = 0; i < S; ++i) M[c * n + j * S + i] = cell_moment(cells[c], R.p3, R.w3, 3, i, j) / area;
    }
    if (!solve_identity(n, M, X)) return false;
    for (int c = 0; c < n; ++c)
        for (int m = 0; m < n; ++m) coef[c * n + m] = X[m * n + c];
    if (ti < 0) {
        const DV2 ref[4] = {DV2{-0.5, -0.5}, DV2{0.5, -0.5}, DV2{0.5, 0.5}, DV2{-0.5, 0.5}};
        smoothness<S>(ref, R, order, coef, form);
    } else {
        smoothness<S>(cells[tj * S + ti], R, order, coef, form);
    }
    return true;
}

__global__ void __launch_bounds__(64) quad_table_kernel(int nx, int ny, const double* __restrict__ xy, int row0,
                                                        int rows, Rules R, double* G0, double* S9, double* T4,
                                                        double* S4, double* geo, int* failed) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t N = (size_t)nx * rows;
    if (k >= (long long)N) return;
    const int i = (int)(k % nx), jl = (int)(k / nx), j = row0 + jl;
    const size_t cell = (size_t)k;
    DV2 target[4];
    cell_quad(xy, nx, i, j, target);
    double area = 0.0;
    {
        const double p[1] = {R.p1}, w[1] = {R.w1};
        area = cell_area(target, p, w, 1);
    }
    if (!(area > 0) || !isfinite(area)) { atomicExch(failed, 1); return; }
    const double h = sqrt(area);
    double off[2] = {0, 0};
    for (int v = 0; v < 4; ++v) { off[0] += (target[v].x - target[0].x) / 4; off[1] += (target[v].y - target[0].y) / 4; }
    const DV2 c{target[0].x + off[0], target[0].y + off[1]};
    geo[cell] = c.x; geo[N + cell] = c.y; geo[2 * N + cell] = h; geo[3 * N + cell] = area;
    const int ci = i == 0 ? 0 : (i == nx - 1 ? 2 : 1), cj = j == 0 ? 0 : (j == ny - 1 ? 2 : 1);
    if (ci == 1 && cj == 1) {
        double coef[81], sigma[81];
        DV2 center;
        if (!stencil<3>(xy, nx, i - 1, j - 1, 2, h, -1, -1, R, coef, sigma, center)) { atomicExch(failed, 1); return; }
        const double dx = (c.x - center.x) / h, dy = (c.y - center.y) / h;
        // Binomial re-expansion of each basis polynomial into the cell's frame.
        const double bin[3][3] = {{1, 0, 0}, {1, 1, 0}, {1, 2, 1}};
        const double px[3] = {1, dx, dx * dx}, py[3] = {1, dy, dy * dy};
        for (int s = 1; s < 9; ++s) {
            const double* a = coef + s * 9;
            for (int jn = 0; jn < 3; ++jn)
                for (int in = 0; in < 3; ++in) {
                    double v = 0;
                    for (int jj = jn; jj < 3; ++jj)
                        for (int ii = in; ii < 3; ++ii)
                            v += a[jj * 3 + ii] * bin[ii][in] * px[ii - in] * bin[jj][jn] * py[jj - jn];
                    G0[(size_t)((s - 1) * 9 + jn * 3 + in) * N + cell] = v;
                }
        }
        int q = 0;
        for (int r = 1; r < 9; ++r)
            for (int cc = r; cc < 9; ++cc) S9[(size_t)(q++) * N + cell] = cc == r ? sigma[r * 9 + r] : 2.0 * sigma[r * 9 + cc];
    }
    const int offi[4] = {0, 0, -1, -1}, offj[4] = {-1, 0, -1, 0};
    for (int kk = 0; kk < 4; ++kk) {
        const int oi = offi[kk], oj = offj[kk];
        const bool on = !((oi == 0 && ci == 2) || (oi == -1 && ci == 0) || (oj == 0 && cj == 2) || (oj == -1 && cj == 0));
        if (!on) continue;
        double coef[16], form[16];
        DV2 center;
        if (!stencil<2>(xy, nx, i + oi, j + oj, 1, h, -oi, -oj, R, coef, form, center)) { atomicExch(failed, 1); return; }
        const double dx = (c.x - center.x) / h, dy = (c.y - center.y) / h;
        for (int s = 1; s < 4; ++s) {
            const double* a = coef + s * 4;
            const double v[4] = {a[0] + a[1] * dx + a[2] * dy + a[3] * dx * dy, a[1] + a[3] * dy, a[2] + a[3] * dx, a[3]};
            for (int mm = 0; mm < 4; ++mm) T4[(size_t)(kk * 12 + (s - 1) * 4 + mm) * N + cell] = v[mm];
        }
        int q = 0;
        for (int r = 1; r < 4; ++r)
            for (int cc = r; cc < 4; ++cc) S4[(size_t)(kk * 6 + q++) * N + cell] = cc == r ? form[r * 4 + r] : 2.0 * form[r * 4 + cc];
    }
}

}  // namespace

int build_quad_cell_tables_gpu(int nx, int ny, const double* d_xy, int row0, int rows, const double* gq3,
                               const double* gw3, double gq1, double gw1, double* G0, double* S9, double* T4,
                               double* S4, double* geo, int* d_failed, cudaStream_t stream) {
    Rules R;
    for (int k = 0; k < 3; ++k) { R.p3[k] = gq3[k]; R.w3[k] = gw3[k]; }
    R.p1 = gq1; R.w1 = gw1;
    const size_t N = (size_t)nx * rows;
    const size_t counts[4] = {kQG0 * N, kQS9 * N, kQT4 * N, kQS4 * N};
    double* zero_ptrs[4] = {G0, S9, T4, S4};
    for (int k = 0; k < 4; ++k)
        if (cudaMemsetAsync(zero_ptrs[k], 0, counts[k] * sizeof(double), stream) != cudaSuccess) return MP_ERR_CUDA;
    if (cudaMemsetAsync(d_failed, 0, sizeof(int), stream) != cudaSuccess) return MP_ERR_CUDA;
    quad_table_kernel<<<(unsigned)((N + 63) / 64), 64, 0, stream>>>(nx, ny, d_xy, row0, rows, R, G0, S9, T4, S4, geo,
                                                                   d_failed);
    if (cudaGetLastError() != cudaSuccess) return MP_ERR_CUDA;
    int failed = 0;
    if (cudaMemcpyAsync(&failed, d_failed, sizeof(int), cudaMemcpyDeviceToHost, stream) != cudaSuccess) return MP_ERR_CUDA;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return MP_ERR_CUDA;
    return failed ? MP_ERR_ARG_WRONG : MP_OK;
}

int upload_quad_tables(int nx, int ny, const double* xy, const QuadTables& qt, int row0, int rows,
                       cudaStream_t stream, double** buf, QuadDev& q, cudaError_t* cuda_err) {
    cudaError_t e = cudaSuccess;
    *buf = nullptr;
    const size_t N = (size_t)nx * rows;
    const size_t V = qt.xy.size(), NEq = qt.spacing.size();
    const size_t total = V + (size_t)(kQG0 + kQS9 + kQT4 + kQS4 + kQGeo) * N + NEq;
    e = cudaMalloc((void**)buf, total * sizeof(double));
    if (e != cudaSuccess) *buf = nullptr;
    double* at = *buf;
    auto put = [&](const std::vector<double>* v, size_t n) -> double* {
        if (v && e == cudaSuccess) e = cudaMemcpyAsync(at, v->data(), n * sizeof(double), cudaMemcpyHostToDevice, stream);
        double* p = at;
        at += n;
        return p;
    };
    double *G0, *S9, *T4, *S4, *geo;
    q.xy = put(&qt.xy, V);
    q.G0 = G0 = put(nullptr, (size_t)kQG0 * N);
    q.S9 = S9 = put(nullptr, (size_t)kQS9 * N);
    q.T4 = T4 = put(nullptr, (size_t)kQT4 * N);
    q.S4 = S4 = put(nullptr, (size_t)kQS4 * N);
    q.geo = geo = put(nullptr, (size_t)kQGeo * N);
    q.sp = put(&qt.spacing, NEq);
    for (int k = 0; k < 5; ++k) { q.gq[k] = qt.gq[k]; q.gw[k] = qt.gw[k]; q.dif_c_bnd[k] = qt.dif_c_bnd[k]; }
    for (int k = 0; k < 4; ++k) q.dif_c_int[k] = qt.dif_c_int[k];
    // The whole mesh's vertices and the failure flag, for the builder only.
    double* d_all = nullptr;
    int* d_failed = nullptr;
    const size_t VA = 2 * (size_t)(nx + 1) * (ny + 1);
    if (e == cudaSuccess) {
        e = cudaMalloc((void**)&d_all, VA * sizeof(double) + sizeof(int));
        if (e != cudaSuccess) d_all = nullptr;
    }
    if (e == cudaSuccess) {
        d_failed = reinterpret_cast<int*>(d_all + VA);
        e = cudaMemcpyAsync(d_all, xy, VA * sizeof(double), cudaMemcpyHostToDevice, stream);
    }
    int gs = MP_OK;
    if (e == cudaSuccess)
        gs = build_quad_cell_tables_gpu(nx, ny, d_all, row0, rows, qt.gq3, qt.gw3, qt.gq1, qt.gw1, G0, S9, T4, S4, geo,
                                        d_failed, stream);
    if (gs == MP_ERR_CUDA) {
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaErrorUnknown;
    }
    if (d_all) cudaFree(d_all);
    if (e != cudaSuccess) {
        if (cuda_err) *cuda_err = e;
        return MP_ERR_CUDA;
    }
    return gs;
}

}  // namespace mp

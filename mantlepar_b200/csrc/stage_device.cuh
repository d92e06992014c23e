// Device building blocks of the ML-WENO H/C transport stage.
//
// Per cell, the reference's reconstruction (Reconstruction::Update +
// TensorStencilPoly::Smoothness, src/mlweno/reconstruction.cpp:275-355 and
// tensorstencilpoly.cpp:400-459) is collapsed into one Q2 "deviation"
// polynomial D(xi, eta) in the target cell's normalised frame:
//   R(x) = u_t + sum_k w_k P_k(x)  ==  u_t + D(xi, eta),
// the 2x2 candidates being re-expanded about the target centre. The limiter
// (state_reconstruction.cpp:136-192) then scales D by theta, so each limited
// evaluation at a point is one 9-term polynomial. Smoothness indicators,
// weights and coefficients are FP64 in every form: the weights are
// (sigma + epsA)^-7 ratios, so an FP32 sigma moves them by several FP32 ulps,
// and the limited values handed to the phase inversion would carry that
// error (about 3e-9 absolute on a deviation of 0.05, more than the porosity
// of a cell near the solidus tolerates at 1e-6 relative).
#ifndef MP_STAGE_DEVICE_CUH
#define MP_STAGE_DEVICE_CUH

#include <cmath>

#include "phase_math.cuh"
#include "tables.hpp"

namespace mp {

// The tables a single-instance launch passes by value (__grid_constant__).
struct ParamTables {
    StageHot d;
};

inline void make_param_tables(const StageTables& t, ParamTables& p) { p.d = static_cast<const StageHot&>(t); }

template <class R> struct Tab;
// Tab pointing at the parameter-space copy (inside a kernel taking a
// __grid_constant__ ParamTables).
template <class R> __device__ __forceinline__ Tab<R> param_tab(const ParamTables& p);
template <> struct Tab<double> {
    const StageHot* t;
    __device__ double C9(int c, int m) const { return t->C9[c][m]; }
    __device__ double S9(int r, int c) const { return t->S9[r][c]; }
    __device__ double C4(int c, int m) const { return t->C4[c][m]; }
    __device__ double S4(int k, int r, int c) const { return t->S4[k][r][c]; }
    __device__ double SF9(int k) const { return t->SF9[k]; }
    __device__ double SF4(int p, int k) const { return t->SF4[p][k]; }
    __device__ double X() const { return t->X; }
    __device__ double Y() const { return t->Y; }
    __device__ double epsA() const { return t->epsA; }
    __device__ double gx(int q) const { return t->gx[q]; }
    __device__ double gy(int q) const { return t->gy[q]; }
    __device__ double line_c(int l) const { return t->line_c[l]; }
};

template <> __device__ __forceinline__ Tab<double> param_tab<double>(const ParamTables& p) { return Tab<double>{&p.d}; }

template <class R> __device__ __forceinline__ R eps_of();
template <> __device__ __forceinline__ double eps_of<double>() { return 2.220446049250313e-16; }

// Row / column coefficients of a Q2 polynomial (coefficient m = j*3 + i of
// xi^i eta^j): along the row eta = y, p(xi) = a0 + xi*(a1 + xi*a2).
template <class R>
__device__ __forceinline__ void q2_row(const R* D, R y, R& a0, R& a1, R& a2) {
    a0 = D[0] + y * (D[3] + y * D[6]);
    a1 = D[1] + y * (D[4] + y * D[7]);
    a2 = D[2] + y * (D[5] + y * D[8]);
}
// Along the column xi = x, p(eta) = b0 + eta*(b1 + eta*b2).
template <class R>
__device__ __forceinline__ void q2_col(const R* D, R x, R& b0, R& b1, R& b2) {
    b0 = D[0] + x * (D[1] + x * D[2]);
    b1 = D[3] + x * (D[4] + x * D[5]);
    b2 = D[6] + x * (D[7] + x * D[8]);
}
template <class R>
__device__ __forceinline__ R quad(R c0, R c1, R c2, R s) { return c0 + s * (c1 + s * c2); }

// sigma = d^T S d on differences to stencil cell 0, formed as one FMA chain
// per row of the folded upper triangle SF. A negative or non-finite chain
// (roundoff at sigma ~ 0, or bad data) is decided as the reference does:
// the term-by-term sum with its roundoff clip (tensorstencilpoly.cpp:424-430).
// Returns -1 on failure.
template <class R, int N, class GF, class G>
__device__ __forceinline__ R smoothness(GF&& SF, G&& S, const R* diff) {
    R sum = 0;
    int k = 0;
#pragma unroll
    for (int r = 0; r < N; ++r) {
        R tr = SF(k++) * diff[r];
#pragma unroll
        for (int c = r + 1; c < N; ++c) tr = fma(SF(k++), diff[c], tr);
        sum = fma(diff[r], tr, sum);
    }
    if (sum >= R(0) && sum < R(INFINITY)) return sum;
    R exact = 0, mag = 0;
#pragma unroll
    for (int r = 0; r < N; ++r) {
        const R sr = S(r, r) * diff[r] * diff[r];
        exact += sr; mag += fabs(sr);
#pragma unroll
        for (int c = r + 1; c < N; ++c) {
            const R term = R(2) * (S(r, c) * diff[r]) * diff[c];
            exact += term; mag += fabs(term);
        }
    }
    if (!isfinite(exact) || exact < -R(64) * eps_of<R>() * mag) return R(-1);
    return exact > R(0) ? exact : R(0);
}

// Nonlinear weights alpha_k = (sigma_k + eps*A)^-(s*r_k + eta(r_k)): 7 for
// the 3x3 order-2 candidate, 5 for the 2x2 order-1 candidates
// (reconstruction.cpp:43-54,212-265). Written as ratios r = epsA/(sigma+epsA)
// in (0,1] with the common factor (epsA)^-7 divided out, so nothing
// overflows; normalised to sum 1.
__device__ __forceinline__ void weights(const double* sig, const bool* on, double eA, double* w) {
    // The five reciprocals 1/(sigma_k + epsA) from one division: prefix
    // and suffix products of s_k = sigma_k + epsA (s_k >= epsA > 0).
    double sk[5], pre[5], suf[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) sk[k] = sig[k] + eA;
    pre[0] = 1.0;
#pragma unroll
    for (int k = 1; k < 5; ++k) pre[k] = pre[k - 1] * sk[k - 1];
    suf[4] = 1.0;
#pragma unroll
    for (int k = 3; k >= 0; --k) suf[k] = suf[k + 1] * sk[k + 1];
    const double P = pre[4] * sk[4];
    double inv_s[5];
    if (P > 1e-290 && P < 1e290) {
        const double invP = 1.0 / P;
#pragma unroll
        for (int k = 0; k < 5; ++k) inv_s[k] = (pre[k] * suf[k]) * invP;
    } else {
#pragma unroll
        for (int k = 0; k < 5; ++k) inv_s[k] = 1.0 / sk[k];
    }
    double alpha[5];
    const double scale = on[0] ? eA * eA : 1.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const double r = eA * inv_s[k];
        const double r2 = r * r;
        alpha[k] = !on[k] ? 0.0 : (k == 0 ? r2 * r2 * r2 * r : scale * (r2 * r2 * r));
    }
    double sum = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) sum += alpha[k];
    const double inv = 1.0 / sum;
#pragma unroll
    for (int k = 0; k < 5; ++k) w[k] = alpha[k] * inv;
}

// Build D (9 coefficients, FP64) for one field from the 3x3 neighbourhood
// u[dj][di] (index 1,1 = target). Candidate mask by boundary class (ci, cj):
// stencils that leave the domain are dropped (reconstruction.cpp:150-153).
// Returns a nonzero PETSC_ERR_FP-class status when a smoothness form is
// negative beyond roundoff or the weights cannot be normalised.
__device__ __forceinline__ int reconstruct(const StageHot& td, int ci, int cj, const double (&u)[3][3],
                                           double (&D)[9]) {
    using R = double;
    const Tab<double> t{&td};
    double d[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) d[a][b] = u[a][b] - u[1][1];
    // Candidate order: 3x3 at (-1,-1); 2x2 at (0,-1), (0,0), (-1,-1), (-1,0).
    const int offi[4] = {0, 0, -1, -1}, offj[4] = {-1, 0, -1, 0};
    bool on[5];
    on[0] = (ci == 1 && cj == 1);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        on[k + 1] = !((offi[k] == 0 && ci == 2) || (offi[k] == -1 && ci == 0) || (offj[k] == 0 && cj == 2) ||
                      (offj[k] == -1 && cj == 0));
    R sig[5];
    int st = 0;
    // Pass 1: smoothness of every active candidate.
    if (on[0]) {
        R diff[8];
#pragma unroll
        for (int c = 1; c < 9; ++c) diff[c - 1] = (R)(d[c / 3][c % 3] - d[0][0]);
        sig[0] = smoothness<R, 8>([&](int k) { return t.SF9(k); }, [&](int r, int c) { return t.S9(r, c); }, diff);
        if (sig[0] < R(0)) st = MP_ERR_FP;
    } else {
        sig[0] = 0;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!on[k + 1]) { sig[k + 1] = 0; continue; }
        const int oi = offi[k], oj = offj[k];
        const double a0 = d[1 + oj][1 + oi];
        R diff[3];
#pragma unroll
        for (int c = 1; c < 4; ++c) diff[c - 1] = (R)(d[1 + oj + c / 2][1 + oi + c % 2] - a0);
        const int tpos = (-oj) * 2 + (-oi);
        sig[k + 1] = smoothness<R, 3>([&](int q) { return t.SF4(tpos, q); }, [&](int r, int c) { return t.S4(tpos, r, c); },
                                      diff);
        if (sig[k + 1] < R(0)) st = MP_ERR_FP;
    }
    double w[5];
    weights(sig, on, t.epsA(), w);
    if (!isfinite(w[0] + w[1] + w[2] + w[3] + w[4])) st = MP_ERR_FP;
    // Pass 2: weighted coefficients accumulated into D (FP64).
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
            for (int c = 1; c < 9; ++c) v += diff[c - 1] * td.C9[c][m];
            D[m] = w[0] * v;
        }
    }
    const double X = td.X, Y = td.Y;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!on[k + 1]) continue;
        const int oi = offi[k], oj = offj[k];
        const double a0 = d[1 + oj][1 + oi];
        double diff[3];
#pragma unroll
        for (int c = 1; c < 4; ++c) diff[c - 1] = d[1 + oj + c / 2][1 + oi + c % 2] - a0;
        double b[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            double v = m == 0 ? a0 : 0.0;
#pragma unroll
            for (int c = 1; c < 4; ++c) v += diff[c - 1] * td.C4[c][m];
            b[m] = v;
        }
        // Re-expand about the target centre: zeta = xi - delta, delta = ((2oi+1)X, (2oj+1)Y).
        const double dx = (double)(2 * oi + 1) * X, dy = (double)(2 * oj + 1) * Y;
        const double wk = w[k + 1];
        D[0] += wk * (b[0] - b[1] * dx - b[2] * dy + b[3] * dx * dy);
        D[1] += wk * (b[1] - b[3] * dy);
        D[3] += wk * (b[2] - b[3] * dx);
        D[4] += wk * b[3];
    }
    return st;
}

}  // namespace mp

#endif

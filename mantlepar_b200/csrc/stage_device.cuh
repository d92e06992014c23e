// Device building blocks of the ML-WENO H/C transport stage (FP64).
//
// Per cell, the reference's reconstruction (Reconstruction::Update +
// TensorStencilPoly::Smoothness, src/mlweno/reconstruction.cpp:275-355 and
// tensorstencilpoly.cpp:400-459) is collapsed into one Q2 "deviation"
// polynomial D(xi, eta) in the target cell's normalised frame:
//   R(x) = u_t + sum_k w_k P_k(x)  ==  u_t + D(xi, eta),
// the 2x2 candidates being re-expanded about the target centre. The limiter
// (state_reconstruction.cpp:136-192) then scales D by theta, so each limited
// evaluation at a point is one 9-term Horner form.
#ifndef MP_STAGE_DEVICE_CUH
#define MP_STAGE_DEVICE_CUH

#include "phase_math.cuh"
#include "tables.hpp"

namespace mp {

// Evaluate a Q2 polynomial, coefficient m = j*3 + i of xi^i eta^j.
template <class R>
__device__ __forceinline__ R q2(const R* D, R x, R y) {
    const R r0 = D[0] + x * (D[1] + x * D[2]);
    const R r1 = D[3] + x * (D[4] + x * D[5]);
    const R r2 = D[6] + x * (D[7] + x * D[8]);
    return r0 + y * (r1 + y * r2);
}

// sigma = d^T S d on differences to stencil cell 0 with the reference's
// roundoff clip (tensorstencilpoly.cpp:424-430). S excludes row/col 0.
template <int N>
__device__ __forceinline__ double smoothness(const double (*S)[N], const double* diff, int& st) {
    double sum = 0.0, mag = 0.0;
#pragma unroll
    for (int r = 0; r < N; ++r) {
        const double sr = S[r][r] * diff[r] * diff[r];
        sum += sr; mag += fabs(sr);
#pragma unroll
        for (int c = r + 1; c < N; ++c) {
            const double term = 2.0 * (S[r][c] * diff[r]) * diff[c];
            sum += term; mag += fabs(term);
        }
    }
    if (!isfinite(sum)) { st = 72; return 0.0; }
    if (sum < -64.0 * 2.220446049250313e-16 * mag) { st = 72; return 0.0; }
    return fmax(0.0, sum);
}

// Build D (9 coefficients) for one field from the 3x3 neighbourhood u[dj][di]
// (index 1,1 = target). Candidate mask by boundary class (ci, cj):
// reconstruction.cpp:150-153 drops stencils that leave the domain.
__device__ __forceinline__ void reconstruct(const StageTables& t, int ci, int cj, const double (&u)[3][3],
                                            double (&D)[9], int& st) {
    const double ut = u[1][1];
    double d[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) d[a][b] = u[a][b] - ut;
#pragma unroll
    for (int m = 0; m < 9; ++m) D[m] = 0.0;
    const double eA = t.epsA;
    double alpha[5];
    double coef[5][9];
    bool on[5];
    // Large 3x3 candidate, offset (-1,-1), order 2 (weight exponent s*r+eta = 3+4 = 7).
    on[0] = (ci == 1 && cj == 1);
    if (on[0]) {
        double diff[8];
#pragma unroll
        for (int c = 1; c < 9; ++c) diff[c - 1] = d[c / 3][c % 3] - d[0][0];
        const double sig = smoothness<8>(t.S9, diff, st);
#pragma unroll
        for (int m = 0; m < 9; ++m) {
            double v = m == 0 ? d[0][0] : 0.0;
#pragma unroll
            for (int c = 1; c < 9; ++c) v += diff[c - 1] * t.C9[c][m];
            coef[0][m] = v;
        }
        const double r = eA / (sig + eA);
        const double r2 = r * r, r3 = r2 * r;
        alpha[0] = r3 * r3 * r;
    } else {
        alpha[0] = 0.0;
    }
    // Small 2x2 candidates, order 1 (exponent 2+3 = 5), offsets (0,-1),(0,0),(-1,-1),(-1,0);
    // target position in the stencil t = tj*2+ti with (ti,tj) = -offset.
    const int offi[4] = {0, 0, -1, -1}, offj[4] = {-1, 0, -1, 0};
    const double scale = on[0] ? eA * eA : 1.0;  // alpha_k * (eps A)^7 keeps all terms in range
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int oi = offi[k], oj = offj[k];
        on[k + 1] = !((oi == 0 && ci == 2) || (oi == -1 && ci == 0) || (oj == 0 && cj == 2) || (oj == -1 && cj == 0));
        if (!on[k + 1]) { alpha[k + 1] = 0.0; continue; }
        double a4[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) a4[s] = d[1 + oj + s / 2][1 + oi + s % 2];
        double diff[3];
#pragma unroll
        for (int c = 1; c < 4; ++c) diff[c - 1] = a4[c] - a4[0];
        const int tpos = (-oj) * 2 + (-oi);
        const double sig = smoothness<3>(t.S4[tpos], diff, st);
        double b[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            double v = m == 0 ? a4[0] : 0.0;
#pragma unroll
            for (int c = 1; c < 4; ++c) v += diff[c - 1] * t.C4[c][m];
            b[m] = v;
        }
        // Re-expand about the target centre: zeta = xi - delta, delta = ((2oi+1)X, (2oj+1)Y).
        const double dx = (2 * oi + 1) * t.X, dy = (2 * oj + 1) * t.Y;
        coef[k + 1][0] = b[0] - b[1] * dx - b[2] * dy + b[3] * dx * dy;
        coef[k + 1][1] = b[1] - b[3] * dy;
        coef[k + 1][3] = b[2] - b[3] * dx;
        coef[k + 1][4] = b[3];
        const double r = eA / (sig + eA);
        const double r2 = r * r;
        alpha[k + 1] = scale * (r2 * r2 * r);
    }
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) sum += alpha[k];
    if (!(sum > 0.0) || !isfinite(sum)) { st = 72; return; }
    const double inv = 1.0 / sum;
    if (on[0]) {
        const double w = alpha[0] * inv;
#pragma unroll
        for (int m = 0; m < 9; ++m) D[m] = w * coef[0][m];
    }
#pragma unroll
    for (int k = 1; k < 5; ++k) {
        if (!on[k]) continue;
        const double w = alpha[k] * inv;
        D[0] += w * coef[k][0];
        D[1] += w * coef[k][1];
        D[3] += w * coef[k][3];
        D[4] += w * coef[k][4];
    }
}

}  // namespace mp

#endif

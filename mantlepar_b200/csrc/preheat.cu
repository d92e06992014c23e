// Legacy dry preheat on B200 (mantle::couple::AdvanceLegacyPreheat,
// src/couple/preheat.cpp:65-287): H_t + div(us H - kappa grad H) = 0 with C
// fixed and the Stokes velocity frozen, forward Euler.
//
// One step is three kernels:
//   pre_recon_kernel   per cell: the unlimited deviation polynomial of H
//                      (StateReconstruction::Update(s, false): limiter 1);
//   pre_face_kernel    per edge: traces of both sides at the 5 Gauss points,
//                      linear-law Lax-Friedrichs flux or the boundary policy,
//                      plus the diffusion of the cell averages;
//   pre_update_kernel  per cell: the face fluxes summed in the reference's
//                      face order, H + dt*rhs into the other state buffer,
//                      block partials; the last block to finish folds them in
//                      a fixed order and applies the step's checks (finite
//                      candidate, heat balance), accepting or stopping.
// The step sizes do not depend on the state (the rate is fixed at Build), so
// the host plans a batch of steps and issues them without waiting; a failed
// step sets the status word and every kernel queued after it returns at once.
//
// On a general quad mesh (mp_preheat_create_quads; the reference's preheat
// runs on any mesh family, preheat.cpp:86-117) the reconstruction, face,
// rate and diagnostics kernels have quad forms that read the per-cell
// tables, map every point from the cell's corners and use physical edge
// lengths, normal-line spacing per edge point and per-cell areas.
#include "common.hpp"
#include "phase_math.cuh"
#include "stage_device.cuh"
#include "stage_kernels.cuh"
#include "quad_device.cuh"
#include "quad_tables.hpp"
#include "tables.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

namespace mp {

PhaseConst phase_const(const mp_material& p, const mp_derived& d);
mp_status derive_checked(const mp_material& p, mp_derived& d);

namespace {

// Boundary and flux constants of the preheat kernels.
struct PreheatPhys {
    double kappa;
    int diffusion;         // kappa > 0 or a wall prescribes a flux
    int wall_type[4];      // MP_THERMAL_* per wall: bottom, top, left, right
    double wall_value[4];
    int Hpol;              // MP_BC_* of H
    double inflowH;
    int lf_global;
    double lf_speed;
};

// Block partial of the preheat reductions.
struct PrePartial {
    double integral, minimum, maximum, bflux, nonfinite;
};
__device__ __forceinline__ PrePartial pre_identity() { return PrePartial{0.0, INFINITY, -INFINITY, 0.0, 0.0}; }

// Device record of one step (the host adds step, time, dt and courant).
struct PreRow {
    double integral, minimum, maximum, bflux, balance;
};

// Device control block of a preheat instance.
struct PreCtl {
    double prev_integral;      // integral of the latest accepted state
    unsigned int ticket;       // blocks finished in the running launch
    unsigned int accepted;     // steps accepted (running count)
    PrePartial last;           // totals of the latest rhs / measure / rate launch
};

enum PreMode : int { PRE_STEP = 0, PRE_RHS = 1, PRE_MEASURE = 2 };

constexpr int kPreBlock = 256;
constexpr int kPrePer = 4;                      // cells per thread in the update kernel
constexpr int kPreCells = kPreBlock * kPrePer;

__device__ __forceinline__ bool halted(const unsigned long long* status) {
    return *(volatile const unsigned long long*)status != ~0ULL;
}

// Fixed-tree block reduction; the result is valid in thread 0.
__device__ PrePartial pre_block_reduce(PrePartial v) {
    __shared__ double sh[kPreBlock / 32][5];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double r[5] = {warp_sum(v.integral), warp_min(v.minimum), warp_max(v.maximum), warp_sum(v.bflux),
                   warp_max(v.nonfinite)};
    if (lane == 0)
        for (int k = 0; k < 5; ++k) sh[warp][k] = r[k];
    __syncthreads();
    PrePartial out = pre_identity();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        double s[5] = {0.0, INFINITY, -INFINITY, 0.0, 0.0};
        if (lane < nw) for (int k = 0; k < 5; ++k) s[k] = sh[lane][k];
        out = PrePartial{warp_sum(s[0]), warp_min(s[1]), warp_max(s[2]), warp_sum(s[3]), warp_max(s[4])};
    }
    __syncthreads();
    return out;
}

__device__ __forceinline__ void pre_fold(PrePartial& a, const PrePartial* p) {
    a.integral += __ldcg(&p->integral);
    a.minimum = fmin(a.minimum, __ldcg(&p->minimum));
    a.maximum = fmax(a.maximum, __ldcg(&p->maximum));
    a.bflux += __ldcg(&p->bflux);
    a.nonfinite = fmax(a.nonfinite, __ldcg(&p->nonfinite));
}

// Write this block's partial; the last block of the launch folds all of them
// in block order (the same sums whichever block finishes last) and returns
// true in every thread with the totals in `tot` (valid in thread 0).
__device__ bool pre_finish_blocks(PrePartial v, PrePartial* partial, PreCtl* ctl, PrePartial& tot) {
    __shared__ bool last;
    const PrePartial b = pre_block_reduce(v);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(&ctl->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    PrePartial a = pre_identity();
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) pre_fold(a, partial + k);
    tot = pre_block_reduce(a);
    if (threadIdx.x == 0) ctl->ticket = 0;
    return true;
}

// Orientation of edge e as the reference's Build (preheat.cpp:86-95):
// left cell L (the wall cell on a boundary, whose edge is then reversed when
// the canonical normal points into it), right cell R, the edge's fixed
// normalised coordinate in each cell's frame, and the wall.
struct EdgeGeo {
    bool horizontal, boundary, reverse;
    long long L, R;
    double lfix, rfix;
    int wall;
};

__device__ __forceinline__ EdgeGeo edge_geo(const StageHot& t, int nx, int ny, long long e) {
    const long long nI = (long long)nx * (ny + 1);
    EdgeGeo g;
    g.R = -1;
    g.wall = -1;
    if (e < nI) {
        const unsigned ue = (unsigned)e;
        const int i = (int)(ue % (unsigned)nx), j = (int)(ue / (unsigned)nx);
        g.horizontal = true;
        g.boundary = j == 0 || j == ny;
        g.reverse = j == ny;
        g.L = g.reverse ? (long long)(j - 1) * nx + i : (long long)j * nx + i;
        if (!g.boundary) g.R = (long long)(j - 1) * nx + i;
        else g.wall = j == 0 ? 0 : 1;
        g.lfix = g.reverse ? t.Y : -t.Y;
        g.rfix = t.Y;
    } else {
        const unsigned k = (unsigned)(e - nI);
        const int i = (int)(k % (unsigned)(nx + 1)), j = (int)(k / (unsigned)(nx + 1));
        g.horizontal = false;
        g.boundary = i == 0 || i == nx;
        g.reverse = i == 0;
        g.L = g.reverse ? (long long)j * nx : (long long)j * nx + (i - 1);
        if (!g.boundary) g.R = (long long)j * nx + i;
        else g.wall = i == 0 ? 2 : 3;
        g.lfix = g.reverse ? -t.X : t.X;
        g.rfix = -t.X;
    }
    return g;
}

// Relative roundoff allowance of a speed bound (advectiveflux.cpp:82-87).
__device__ __forceinline__ bool speed_bounds(double bound, double required) {
    return bound >= required || required - bound <= 64.0 * 2.220446049250313e-16 * fmax(bound, required);
}

// ------------------------------------------------------------------ kernels

// H-only reconstruction without the limiter.
__global__ void __launch_bounds__(128) pre_recon_kernel(int nx, int ny, const double* __restrict__ H,
                                                        double* __restrict__ rec, unsigned long long* status,
                                                        const __grid_constant__ ParamTables p) {
    if (halted(status)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    const StageHot& t = p.d;
    const long long cell = (long long)j * nx + i;
    const size_t N = (size_t)nx * ny;
    double u[3][3];
#pragma unroll
    for (int dj = 0; dj < 3; ++dj)
#pragma unroll
        for (int di = 0; di < 3; ++di) {
            const int ii = min(max(i + di - 1, 0), nx - 1), jj = min(max(j + dj - 1, 0), ny - 1);
            u[dj][di] = __ldg(H + (size_t)jj * nx + ii);
        }
    const int ci = i == 0 ? 0 : (i == nx - 1 ? 2 : 1), cj = j == 0 ? 0 : (j == ny - 1 ? 2 : 1);
    double D[9];
    const int st = reconstruct(t, ci, cj, u, D);
#pragma unroll
    for (int m = 0; m < 9; ++m) rec[(size_t)m * N + cell] = D[m];
    if (st) record_error(status, PART_UPDATE, cell, st);
}

// Edge flux of preheat.cpp:166-196: advection + diffusion of H.
__global__ void __launch_bounds__(128, 8) pre_face_kernel(int nx, int ny, const double* __restrict__ H,
                                                       const double* __restrict__ rec, const double* __restrict__ vn,
                                                       double* __restrict__ flux, unsigned long long* status,
                                                       const __grid_constant__ PreheatPhys pp,
                                                       const __grid_constant__ ParamTables p) {
    if (halted(status)) return;
    const long long nE = (long long)nx * (ny + 1) + (long long)(nx + 1) * ny;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nE) return;
    const StageHot& t = p.d;
    const size_t N = (size_t)nx * ny;
    const EdgeGeo g = edge_geo(t, nx, ny, e);
    const int o = g.horizontal ? 0 : 1;
    double DL[9], DR[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) {
        DL[m] = __ldg(rec + (size_t)m * N + g.L);
        DR[m] = g.boundary ? 0.0 : __ldg(rec + (size_t)m * N + g.R);
    }
    const double mL = __ldg(H + g.L), mR = g.boundary ? mL : __ldg(H + g.R);
    double l0, l1, l2, r0, r1, r2;
    if (g.horizontal) { q2_row(DL, g.lfix, l0, l1, l2); q2_row(DR, g.rfix, r0, r1, r2); }
    else { q2_col(DL, g.lfix, l0, l1, l2); q2_col(DR, g.rfix, r0, r1, r2); }
    const double sgn = g.reverse ? -1.0 : 1.0;
    int st = 0;
    double sum = 0.0;
#pragma unroll
    for (int q = 0; q < kNQ; ++q) {
        const int cq = g.reverse ? kNQ - 1 - q : q;
        const double at = g.horizontal ? t.gx[cq] : t.gy[cq];
        const double v = sgn * __ldg(vn + e * kNQ + cq);
        const double uL = mL + quad(l0, l1, l2, at);
        if (!isfinite(v) || !isfinite(uL)) st = st ? st : E_OUTOFRANGE;
        double f;
        if (g.boundary) {
            // EvaluateAdvectionBoundary (initialization.cpp:469-489) and the
            // physical boundary flux (advectiveflux.cpp:229-271).
            if (pp.Hpol == MP_BC_ZERO_FLUX || v == 0.0) f = 0.0;
            else if (v < 0.0) {
                if (pp.Hpol != MP_BC_INFLOW_OUTFLOW) st = st ? st : E_OUTOFRANGE;
                f = v * pp.inflowH;
            } else f = v * uL;
        } else {
            const double uR = mR + quad(r0, r1, r2, at);
            if (!isfinite(uR)) st = st ? st : E_OUTOFRANGE;
            const double a = pp.lf_global ? pp.lf_speed : fabs(v);
            if (!speed_bounds(a, fabs(v))) st = st ? st : E_OUTOFRANGE;
            f = 0.5 * (v * uL + v * uR - a * (uR - uL));
        }
        if (!isfinite(f)) st = st ? st : E_FP;
        sum += t.dif_w[o][q] * f;
    }
    if (pp.diffusion) {
        // Diffusion of H on constant cell-average samples (preheat.cpp:183-194
        // with diffusiveflux.cpp:105-200): interior samples [L, L, R, R],
        // wall samples [L, L, L, L, wall value]; gradient sum_k c_k (v_k -
        // v_last) / ds.
        const int type = g.boundary ? pp.wall_type[g.wall] : MP_THERMAL_TEMPERATURE;
        const double wv = g.boundary ? pp.wall_value[g.wall] : 0.0;
        if (type == MP_THERMAL_FLUX) {
#pragma unroll
            for (int q = 0; q < kNQ; ++q) sum += t.dif_w[o][q] * wv;
        } else if (type == MP_THERMAL_TEMPERATURE) {
            double grad = 0.0;
            if (g.boundary) {
#pragma unroll
                for (int k = 0; k < 4; ++k) grad += t.dif_c_bnd[k] * (mL - wv);
            } else {
#pragma unroll
                for (int k = 0; k < 3; ++k) grad += t.dif_c_int[k] * ((k < 2 ? mL : mR) - mR);
            }
            grad /= t.dif_ds[o][g.boundary ? 1 : 0];
            if (!isfinite(grad)) st = st ? st : E_FP;
            double integral = 0.0;
#pragma unroll
            for (int q = 0; q < kNQ; ++q) integral -= t.dif_w[o][q] * pp.kappa * grad;
            sum += integral;
        }
    }
    flux[e] = sum;
    if (st) record_error(status, PART_FACES, e, st);
}

// Per-cell sum of the face fluxes (faces bottom, top, left, right in id order,
// each with its side's sign, preheat.cpp:195-197), the forward-Euler
// candidate and the step's checks (preheat.cpp:267-273).
// kQuad: per-cell areas (general quad mesh) instead of the uniform one.
template <bool kQuad>
__global__ void __launch_bounds__(kPreBlock) pre_update_kernel(int nx, int ny, double area, double inv_area,
                                                                const double* __restrict__ cell_area,
                                                                const double* __restrict__ H, const double* __restrict__ flux,
                                                                double* __restrict__ Hout, double* __restrict__ rhs,
                                                                int mode, double dt, int row, PreRow* rows,
                                                                PrePartial* partial, PreCtl* ctl,
                                                                unsigned long long* status) {
    if (halted(status)) return;
    const long long N = (long long)nx * ny;
    const long long nI = (long long)nx * (ny + 1);
    PrePartial v = pre_identity();
#pragma unroll
    for (int k = 0; k < kPrePer; ++k) {
        const long long cell = (long long)blockIdx.x * kPreCells + k * kPreBlock + threadIdx.x;
        if (cell >= N) continue;
        const double h = __ldg(H + cell);
        double cand = h;
        double a = area;
        if constexpr (kQuad) a = __ldg(cell_area + cell);
        if (mode != PRE_MEASURE) {
            const int i = (int)(cell % nx), j = (int)(cell / nx);
            const long long eb = (long long)j * nx + i, et = eb + nx;
            const long long el = nI + (long long)j * (nx + 1) + i, er = el + 1;
            const double fb = __ldg(flux + eb), ft = __ldg(flux + et), fl = __ldg(flux + el), fr = __ldg(flux + er);
            const double sum = ((-fb) + (j == ny - 1 ? -ft : ft)) + (i == 0 ? -fl : fl) - fr;
            double r;
            if constexpr (kQuad) r = sum / a;
            else r = sum * inv_area;
            double b = 0.0;
            if (j == 0) b += fb;
            if (j == ny - 1) b += ft;
            if (i == 0) b += fl;
            if (i == nx - 1) b += fr;
            v.bflux += b;
            if (mode == PRE_RHS) rhs[cell] = r;
            else {
                cand = __dadd_rn(h, __dmul_rn(dt, r));
                Hout[cell] = cand;
            }
        }
        v.integral += cand * a;
        v.minimum = fmin(v.minimum, cand);
        v.maximum = fmax(v.maximum, cand);
        v.nonfinite = fmax(v.nonfinite, isfinite(cand) ? 0.0 : 1.0);
    }
    PrePartial tot;
    if (!pre_finish_blocks(v, partial, ctl, tot) || threadIdx.x != 0) return;
    if (mode != PRE_STEP) { ctl->last = tot; return; }
    if (tot.nonfinite != 0.0) { record_error(status, PART_CELLS, 0, E_FP); return; }
    const double prev = ctl->prev_integral;
    const double bal = tot.integral - prev + dt * tot.bflux;
    const double tol = 1e-10 * (1.0 + fabs(tot.integral) + fabs(prev) + fabs(dt * tot.bflux));
    if (!(fabs(bal) <= tol)) { record_error(status, PART_CELLS, 0, MP_ERR_PLIB); return; }
    rows[row] = PreRow{tot.integral, tot.minimum, tot.maximum, tot.bflux, bal};
    ctl->prev_integral = tot.integral;
    ctl->accepted += 1;
}

// Build (preheat.cpp:130-156), per edge: LF speed sum_q L w_q alpha / 2 and
// the diffusion derivatives at zero samples summed per side; writes
// (speed + |derivative|) / area for the left [e] and right [NE + e] cell.
__global__ void __launch_bounds__(128) pre_rate_edge_kernel(int nx, int ny, double area, const double* __restrict__ vn,
                                                            double* __restrict__ rr, unsigned long long* status,
                                                            const __grid_constant__ PreheatPhys pp,
                                                            const __grid_constant__ ParamTables p) {
    const long long nE = (long long)nx * (ny + 1) + (long long)(nx + 1) * ny;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nE) return;
    const StageHot& t = p.d;
    const EdgeGeo g = edge_geo(t, nx, ny, e);
    const int o = g.horizontal ? 0 : 1;
    const double len = g.horizontal ? t.len_h : t.len_v;
    int st = 0;
    double speed = 0.0;
#pragma unroll
    for (int q = 0; q < kNQ; ++q) {
        const int cq = g.reverse ? kNQ - 1 - q : q;
        const double v = __ldg(vn + e * kNQ + cq);
        const double ns = fabs(v);
        if (!isfinite(v)) st = E_OUTOFRANGE;
        const double a = pp.lf_global ? pp.lf_speed : ns;
        if (!(a + 1e-14 >= ns)) st = E_OUTOFRANGE;
        // .5 * length * w_q * alpha, rounded as the reference writes it.
        speed = __dadd_rn(speed, __dmul_rn(__dmul_rn(__dmul_rn(0.5, len), t.gw[q]), a));
    }
    // d flux / d sample = -w kappa c_k / ds per sample (the last sample gets
    // -sum of the others' coefficients); interior samples k < 2 are the
    // left cell's, wall samples k < 4 all the wall cell's.
    double d0 = 0.0, d1 = 0.0;
    const int type = g.boundary ? pp.wall_type[g.wall] : MP_THERMAL_TEMPERATURE;
    if (type == MP_THERMAL_TEMPERATURE) {
        const double ds = t.dif_ds[o][g.boundary ? 1 : 0];
        double clast = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) clast -= t.dif_c_int[k];
#pragma unroll
        for (int q = 0; q < kNQ; ++q) {
            const double scale = -t.dif_w[o][q] * pp.kappa / ds;
            if (g.boundary) {
#pragma unroll
                for (int k = 0; k < 4; ++k) d0 += scale * t.dif_c_bnd[k];   // k = 4: the wall value
            } else {
                d0 += scale * t.dif_c_int[0];
                d0 += scale * t.dif_c_int[1];
                d1 += scale * t.dif_c_int[2];
                d1 += scale * clast;
            }
        }
    }
    const double d[2] = {d0, d1};
    rr[e] = (speed + fabs(d[0])) / area;
    rr[nE + e] = (speed + fabs(d[1])) / area;
    if (st) record_error(status, PART_FACES, e, st);
}

// Per-cell rate: the faces' shares in id order (bottom, top, left, right),
// the side of each face that this cell is; the last block keeps the maximum.
__global__ void __launch_bounds__(kPreBlock) pre_rate_cell_kernel(int nx, int ny, const double* __restrict__ rr,
                                                                   double* __restrict__ rate, PrePartial* partial,
                                                                   PreCtl* ctl) {
    const long long N = (long long)nx * ny;
    const long long nI = (long long)nx * (ny + 1), nE = nI + (long long)(nx + 1) * ny;
    PrePartial v = pre_identity();
#pragma unroll
    for (int k = 0; k < kPrePer; ++k) {
        const long long cell = (long long)blockIdx.x * kPreCells + k * kPreBlock + threadIdx.x;
        if (cell >= N) continue;
        const int i = (int)(cell % nx), j = (int)(cell / nx);
        const long long eb = (long long)j * nx + i, et = eb + nx;
        const long long el = nI + (long long)j * (nx + 1) + i, er = el + 1;
        double r = 0.0;
        r = __dadd_rn(r, __ldg(rr + eb));
        r = __dadd_rn(r, __ldg(rr + (j == ny - 1 ? 0 : nE) + et));
        r = __dadd_rn(r, __ldg(rr + (i == 0 ? 0 : nE) + el));
        r = __dadd_rn(r, __ldg(rr + er));
        rate[cell] = r;
        v.maximum = fmax(v.maximum, r);
        v.nonfinite = fmax(v.nonfinite, isfinite(r) ? 0.0 : 1.0);
    }
    PrePartial tot;
    if (pre_finish_blocks(v, partial, ctl, tot) && threadIdx.x == 0) ctl->last = tot;
}

// Diagnostics (preheat.cpp:202-233): the unlimited reconstructions of H and C
// and the 5x5 quadrature of the phase's T and phi.
__global__ void __launch_bounds__(128) pre_diag_kernel(int nx, int ny, const double* __restrict__ H,
                                                       const double* __restrict__ C, double* __restrict__ T,
                                                       double* __restrict__ phi, unsigned long long* status, Physics ph,
                                                       const __grid_constant__ ParamTables p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    const StageHot& t = p.d;
    const long long cell = (long long)j * nx + i;
    const int ci = i == 0 ? 0 : (i == nx - 1 ? 2 : 1), cj = j == 0 ? 0 : (j == ny - 1 ? 2 : 1);
    double D[2][9];
    double m[2];
    int st = 0;
    for (int f = 0; f < 2; ++f) {
        const double* F = f ? C : H;
        double u[3][3];
        for (int dj = 0; dj < 3; ++dj)
            for (int di = 0; di < 3; ++di) {
                const int ii = min(max(i + di - 1, 0), nx - 1), jj = min(max(j + dj - 1, 0), ny - 1);
                u[dj][di] = __ldg(F + (size_t)jj * nx + ii);
            }
        m[f] = u[1][1];
        const int s = reconstruct(t, ci, cj, u, D[f]);
        st = st ? st : s;
    }
    if (st) { record_error(status, PART_UPDATE, cell, st); return; }
    double Ts = 0.0, Ps = 0.0;
    for (int b = 0; b < kNQ; ++b) {
        double h0, h1, h2, c0, c1, c2;
        const double y = t.gy[b];
        q2_row(D[0], y, h0, h1, h2);
        q2_row(D[1], y, c0, c1, c2);
        const double tep = tep_at(ph, height(t, j, y));
        for (int q = 0; q < kNQ; ++q) {
            const double x = t.gx[q];
            PhaseLean pl;
            const int s = phase_stage_lean(ph.sk, m[0] + quad(h0, h1, h2, x), m[1] + quad(c0, c1, c2, x), tep, pl);
            if (s) { st = st ? st : s; continue; }
            const double w = t.cw[b * kNQ + q];
            Ts += w * pl.T;
            Ps += w * pl.phil;
        }
    }
    if (st) record_error(status, PART_CELLS, cell, st);
    T[cell] = Ts;
    phi[cell] = Ps;
}

// ------------------------------------------------- general quad mesh forms

// H-only reconstruction with the cell's own tables, without the limiter.
__global__ void __launch_bounds__(128, 4) pre_quad_recon_kernel(int nx, int ny, const double* __restrict__ H,
                                                                double* __restrict__ rec, unsigned long long* status,
                                                                QuadDev q) {
    if (halted(status)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    const long long cell = (long long)j * nx + i;
    const size_t N = (size_t)nx * ny;
    const int ci = i == 0 ? 0 : (i == nx - 1 ? 2 : 1), cj = j == 0 ? 0 : (j == ny - 1 ? 2 : 1);
    const double eA = 1e-2 * __ldg(q.geo + 3 * N + cell);
    double u[1][3][3];
#pragma unroll
    for (int dj = 0; dj < 3; ++dj)
#pragma unroll
        for (int di = 0; di < 3; ++di) {
            const int ii = min(max(i + di - 1, 0), nx - 1), jj = min(max(j + dj - 1, 0), ny - 1);
            u[0][dj][di] = __ldg(H + (size_t)jj * nx + ii);
        }
    double D[1][9];
    const int st = reconstruct_quad<1>(q, N, cell, ci, cj, eA, u, D);
#pragma unroll
    for (int m = 0; m < 9; ++m) rec[(size_t)m * N + cell] = D[0][m];
    if (st) record_error(status, PART_UPDATE, cell, st);
}

// One side of an edge: the cell's frame and its H polynomial.
struct PreSide {
    double cx, cy, inv_h, m;
    double D[9];
};
__device__ __forceinline__ void pre_side(const QuadDev& q, size_t N, const double* H, const double* rec, long long cell,
                                         PreSide& s) {
    s.cx = __ldg(q.geo + cell);
    s.cy = __ldg(q.geo + N + cell);
    s.inv_h = 1.0 / __ldg(q.geo + 2 * N + cell);
    s.m = __ldg(H + cell);
#pragma unroll
    for (int k = 0; k < 9; ++k) s.D[k] = __ldg(rec + (size_t)k * N + cell);
}
__device__ __forceinline__ double pre_trace(const PreSide& s, P2 p) {
    return s.m + q2v(s.D, (p.x - s.cx) * s.inv_h, (p.y - s.cy) * s.inv_h);
}

// Edge flux of preheat.cpp:166-196 on a general quad mesh: the traces at the
// edge's Gauss points in each side's frame, the linear-law Lax-Friedrichs
// flux or the boundary policy with weights L w_q / 2, and the diffusion of
// the cell averages with the normal-line spacing of each edge point.
__global__ void __launch_bounds__(128) pre_quad_face_kernel(int nx, int ny, const double* __restrict__ H,
                                                            const double* __restrict__ rec,
                                                            const double* __restrict__ vn, double* __restrict__ flux,
                                                            unsigned long long* status,
                                                            const __grid_constant__ PreheatPhys pp, QuadDev q) {
    if (halted(status)) return;
    const long long nE = (long long)nx * (ny + 1) + (long long)(nx + 1) * ny;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nE) return;
    const size_t N = (size_t)nx * ny;
    const QuadEdge g = quad_edge(q, nx, ny, 0, ny, e);
    double len;
    P2 nrm;
    edge_geometry(g.a, g.b, len, nrm);
    PreSide sl, sr;
    pre_side(q, N, H, rec, g.L, sl);
    if (!g.boundary) pre_side(q, N, H, rec, g.R, sr);
    const double mL = sl.m, mR = g.boundary ? mL : sr.m;
    const double sgn = g.reverse ? -1.0 : 1.0;
    int st = 0;
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < kNQ; ++k) {
        const int cq = g.reverse ? kNQ - 1 - k : k;
        const P2 p = lerp_edge(q.gq[k], g.a, g.b);
        const double v = sgn * __ldg(vn + e * kNQ + cq);
        const double uL = pre_trace(sl, p);
        if (!isfinite(v) || !isfinite(uL)) st = st ? st : E_OUTOFRANGE;
        double f;
        if (g.boundary) {
            if (pp.Hpol == MP_BC_ZERO_FLUX || v == 0.0) f = 0.0;
            else if (v < 0.0) {
                if (pp.Hpol != MP_BC_INFLOW_OUTFLOW) st = st ? st : E_OUTOFRANGE;
                f = v * pp.inflowH;
            } else f = v * uL;
        } else {
            const double uR = pre_trace(sr, p);
            if (!isfinite(uR)) st = st ? st : E_OUTOFRANGE;
            const double a = pp.lf_global ? pp.lf_speed : fabs(v);
            if (!speed_bounds(a, fabs(v))) st = st ? st : E_OUTOFRANGE;
            f = 0.5 * (v * uL + v * uR - a * (uR - uL));
        }
        if (!isfinite(f)) st = st ? st : E_FP;
        sum += 0.5 * len * q.gw[k] * f;
    }
    if (pp.diffusion) {
        // Interior samples [L, L, R, R], wall samples [L, L, L, L, wall
        // value]; gradient sum_k c_k (v_k - v_last) / spacing at each point.
        const int type = g.boundary ? pp.wall_type[g.wall] : MP_THERMAL_TEMPERATURE;
        const double wv = g.boundary ? pp.wall_value[g.wall] : 0.0;
        if (type == MP_THERMAL_FLUX) {
#pragma unroll
            for (int k = 0; k < kNQ; ++k) sum += len * q.gw[k] / 2 * wv;
        } else if (type == MP_THERMAL_TEMPERATURE) {
            double integral = 0.0;
#pragma unroll
            for (int k = 0; k < kNQ; ++k) {
                const int cq = g.reverse ? kNQ - 1 - k : k;
                const double sp = __ldg(q.sp + e * kNQ + cq);
                double grad = 0.0;
                if (g.boundary) {
#pragma unroll
                    for (int c = 0; c < 4; ++c) grad += q.dif_c_bnd[c] * (mL - wv);
                } else {
#pragma unroll
                    for (int c = 0; c < 3; ++c) grad += q.dif_c_int[c] * ((c < 2 ? mL : mR) - mR);
                }
                grad /= sp;
                if (!isfinite(grad)) st = st ? st : E_FP;
                integral -= len * q.gw[k] / 2 * pp.kappa * grad;
            }
            sum += integral;
        }
    }
    flux[e] = sum;
    if (st) record_error(status, PART_FACES, e, st);
}

// Build (preheat.cpp:130-156) on a general quad mesh: per edge the LF speed
// sum_q L w_q alpha / 2 and the diffusion derivatives at zero samples per
// side; (speed + |derivative|) / area of the left [e] and right [NE + e] cell.
__global__ void __launch_bounds__(128) pre_quad_rate_edge_kernel(int nx, int ny, const double* __restrict__ vn,
                                                                 double* __restrict__ rr, unsigned long long* status,
                                                                 const __grid_constant__ PreheatPhys pp, QuadDev q) {
    const long long nE = (long long)nx * (ny + 1) + (long long)(nx + 1) * ny;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nE) return;
    const size_t N = (size_t)nx * ny;
    const QuadEdge g = quad_edge(q, nx, ny, 0, ny, e);
    double len;
    P2 nrm;
    edge_geometry(g.a, g.b, len, nrm);
    int st = 0;
    double speed = 0.0;
#pragma unroll
    for (int k = 0; k < kNQ; ++k) {
        const int cq = g.reverse ? kNQ - 1 - k : k;
        const double v = __ldg(vn + e * kNQ + cq);
        const double ns = fabs(v);
        if (!isfinite(v)) st = E_OUTOFRANGE;
        const double a = pp.lf_global ? pp.lf_speed : ns;
        if (!(a + 1e-14 >= ns)) st = E_OUTOFRANGE;
        speed = __dadd_rn(speed, __dmul_rn(__dmul_rn(__dmul_rn(0.5, len), q.gw[k]), a));
    }
    double d0 = 0.0, d1 = 0.0;
    const int type = g.boundary ? pp.wall_type[g.wall] : MP_THERMAL_TEMPERATURE;
    if (type == MP_THERMAL_TEMPERATURE) {
        double clast = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) clast -= q.dif_c_int[c];
#pragma unroll
        for (int k = 0; k < kNQ; ++k) {
            const int cq = g.reverse ? kNQ - 1 - k : k;
            const double sp = __ldg(q.sp + e * kNQ + cq);
            const double scale = -(len * q.gw[k] / 2) * pp.kappa / sp;
            if (g.boundary) {
#pragma unroll
                for (int c = 0; c < 4; ++c) d0 += scale * q.dif_c_bnd[c];
            } else {
                d0 += scale * q.dif_c_int[0];
                d0 += scale * q.dif_c_int[1];
                d1 += scale * q.dif_c_int[2];
                d1 += scale * clast;
            }
        }
    }
    const double aL = __ldg(q.geo + 3 * N + g.L), aR = g.boundary ? aL : __ldg(q.geo + 3 * N + g.R);
    rr[e] = (speed + fabs(d0)) / aL;
    rr[nE + e] = (speed + fabs(d1)) / aR;
    if (st) record_error(status, PART_FACES, e, st);
}

// Diagnostics (preheat.cpp:202-233) on a general quad mesh: the unlimited
// reconstructions of H and C and the 5x5 quadrature of T and phi on the
// bilinear map, weights w_a w_b J / area.
__global__ void __launch_bounds__(128) pre_quad_diag_kernel(int nx, int ny, const double* __restrict__ H,
                                                            const double* __restrict__ C, double* __restrict__ T,
                                                            double* __restrict__ phi, unsigned long long* status,
                                                            Physics ph, QuadDev q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    const long long cell = (long long)j * nx + i;
    const size_t N = (size_t)nx * ny;
    const int ci = i == 0 ? 0 : (i == nx - 1 ? 2 : 1), cj = j == 0 ? 0 : (j == ny - 1 ? 2 : 1);
    const CellFrame f = cell_frame(q, nx, N, cell);
    const double eA = 1e-2 * f.area;
    double u[2][3][3];
    for (int dj = 0; dj < 3; ++dj)
        for (int di = 0; di < 3; ++di) {
            const int ii = min(max(i + di - 1, 0), nx - 1), jj = min(max(j + dj - 1, 0), ny - 1);
            u[0][dj][di] = __ldg(H + (size_t)jj * nx + ii);
            u[1][dj][di] = __ldg(C + (size_t)jj * nx + ii);
        }
    const double m[2] = {u[0][1][1], u[1][1][1]};
    double D[2][9];
    int st = reconstruct_quad<2>(q, N, cell, ci, cj, eA, u, D);
    if (st) { record_error(status, PART_UPDATE, cell, st); return; }
    double Ts = 0.0, Ps = 0.0;
    for (int b = 0; b < kNQ; ++b)
        for (int a = 0; a < kNQ; ++a) {
            const P2 p = bilinear(q.gq[a], q.gq[b], f.c);
            const double x = (p.x - f.cx) * f.inv_h, y = (p.y - f.cy) * f.inv_h;
            const double tep = ph.litho ? tep_at(ph, p.y) : ph.Tep;
            PhaseLean pl;
            const int s = phase_stage_lean(ph.sk, m[0] + q2v(D[0], x, y), m[1] + q2v(D[1], x, y), tep, pl);
            if (s) { st = st ? st : s; continue; }
            const double w = q.gw[a] * q.gw[b] * jacobian(q.gq[a], q.gq[b], f.c) / f.area;
            Ts += w * pl.T;
            Ps += w * pl.phil;
        }
    if (st) record_error(status, PART_CELLS, cell, st);
    T[cell] = Ts;
    phi[cell] = Ps;
}

}  // namespace
}  // namespace mp

// -------------------------------------------------------------------- handle

struct mp_preheat {
    mp_mesh_desc mesh;
    mp_preheat_opts opts;
    mp_derived der;
    mp::Physics ph;                 // phase constants and pressure model (diagnostics)
    mp::PreheatPhys pp;
    cudaStream_t stream = nullptr;
    int nx = 0, ny = 0;
    size_t N = 0, NE = 0;
    mp::StageTables host_tab;
    mp::ParamTables ptab;
    double* Hb[2] = {nullptr, nullptr};   // state ping-pong; Hb[cur] is accepted
    int cur = 0;
    double *C = nullptr, *rec = nullptr, *vn = nullptr, *flux = nullptr, *rr = nullptr, *rate = nullptr;
    double *rhs = nullptr, *T = nullptr, *phi = nullptr;
    mp::PrePartial* partial = nullptr;
    mp::PreCtl* ctl = nullptr;
    mp::PreRow* rows = nullptr;     // kBatch rows
    mp::PreCtl* h_ctl = nullptr;    // pinned mirrors
    mp::PreRow* h_rows = nullptr;
    unsigned long long* d_status = nullptr;
    unsigned long long* h_status = nullptr;
    int blocks = 0;
    double time = 0.0;
    long long accepted = 0;
    long long steps = 0;            // steps of the current run
    bool ready = false;             // begin() done for the current state
    double rate_max = 0.0, limit = 0.0;
    unsigned int acc_seen = 0;      // ctl->accepted after the last batch
    // General quad mesh (mp_preheat_create_quads): per-cell tables in HBM.
    bool quad = false;
    mp::QuadDev qdev{};
    double* qbuf = nullptr;         // one allocation holding every table
};

namespace mp {
namespace {

constexpr int kBatch = 512;         // steps issued per host round trip

void pre_free(mp_preheat* p) {
    void* bufs[] = {p->Hb[0], p->Hb[1], p->C, p->rec, p->vn, p->flux, p->rr, p->rate, p->rhs, p->T, p->phi,
                    p->partial, p->ctl, p->rows, p->d_status, p->qbuf};
    for (void* b : bufs) if (b) cudaFree(b);
    if (p->h_ctl) cudaFreeHost(p->h_ctl);
    if (p->h_rows) cudaFreeHost(p->h_rows);
    if (p->h_status) cudaFreeHost(p->h_status);
}

mp_status pre_status(mp_preheat* p, const char* where) {
    const unsigned long long v = *p->h_status;
    if (v == ~0ULL) return MP_OK;
    const int part = (int)(v >> 56);
    const long long at = (long long)((v >> 8) & ((1ULL << 48) - 1));
    const int code = (int)(v & 0xff);
    const char* what = code == MP_ERR_PLIB ? "Preheat heat balance failed; candidate rejected"
                     : code == MP_ERR_FP ? (part == PART_CELLS ? "Nonfinite preheat candidate rejected"
                                                               : "non-finite reconstruction or flux")
                     : code == MP_ERR_ARG_OUTOFRANGE ? "non-finite trace or velocity, backflow on an outflow-only "
                                                       "wall, or a global LF speed below a normal speed"
                     : "phase evaluation failed";
    set_error("%s: %s %lld: %s", where, part == PART_FACES ? "edge" : "cell", at, what);
    return (mp_status)code;
}

mp_status reset_status(mp_preheat* p) {
    MP_CUDA(cudaMemsetAsync(p->d_status, 0xff, sizeof(unsigned long long), p->stream));
    return MP_OK;
}

mp_status read_status(mp_preheat* p) {
    MP_CUDA(cudaMemcpyAsync(p->h_status, p->d_status, sizeof(unsigned long long), cudaMemcpyDeviceToHost, p->stream));
    MP_CUDA(cudaMemcpyAsync(p->h_ctl, p->ctl, sizeof(PreCtl), cudaMemcpyDeviceToHost, p->stream));
    MP_CUDA(cudaStreamSynchronize(p->stream));
    return MP_OK;
}

// The three kernels of one RHS evaluation / step on state Hb[src].
void launch_rhs_kernels(mp_preheat* p, const double* H) {
    const int nx = p->nx, ny = p->ny;
    if (p->quad) {
        dim3 blk(32, 4), grd((nx + 31) / 32, (ny + 3) / 4);
        pre_quad_recon_kernel<<<grd, blk, 0, p->stream>>>(nx, ny, H, p->rec, p->d_status, p->qdev);
        pre_quad_face_kernel<<<(unsigned)((p->NE + 127) / 128), 128, 0, p->stream>>>(nx, ny, H, p->rec, p->vn, p->flux,
                                                                                     p->d_status, p->pp, p->qdev);
        count_launch(2);
        return;
    }
    {
        dim3 blk(32, 4), grd((nx + 31) / 32, (ny + 3) / 4);
        pre_recon_kernel<<<grd, blk, 0, p->stream>>>(nx, ny, H, p->rec, p->d_status, p->ptab);
    }
    pre_face_kernel<<<(unsigned)((p->NE + 127) / 128), 128, 0, p->stream>>>(nx, ny, H, p->rec, p->vn, p->flux,
                                                                            p->d_status, p->pp, p->ptab);
    count_launch(2);
}

void launch_update(mp_preheat* p, const double* H, double* Hout, int mode, double dt, int row) {
    if (p->quad)
        pre_update_kernel<true><<<p->blocks, kPreBlock, 0, p->stream>>>(p->nx, p->ny, 0.0, 0.0, p->qdev.geo + 3 * p->N,
                                                                       H, p->flux, Hout, p->rhs, mode, dt, row,
                                                                       p->rows, p->partial, p->ctl, p->d_status);
    else
        pre_update_kernel<false><<<p->blocks, kPreBlock, 0, p->stream>>>(p->nx, p->ny, p->host_tab.area,
                                                                        1.0 / p->host_tab.area, nullptr, H, p->flux,
                                                                        Hout, p->rhs, mode, dt, row, p->rows,
                                                                        p->partial, p->ctl, p->d_status);
    count_launch();
}

// Step plan of Run (preheat.cpp:256-265): dt of the next step from the
// controls, or a failure status.
mp_status plan_step(const mp_preheat* p, double time, long long steps, double& dt, double& next) {
    const mp_preheat_opts& o = p->opts;
    if (steps >= o.max_steps) { set_error("maximum_steps reached before time.end"); return MP_ERR_NOT_CONVERGED; }
    const double remaining = o.end - time;
    dt = o.control == MP_TIME_FIXED ? o.dt_initial : std::min(o.dt_max, p->limit);
    if (o.control == MP_TIME_CFL && steps == 0) dt = std::min(dt, o.dt_initial);
    dt = std::min(dt, remaining);
    const double roundoff = 8 * std::numeric_limits<double>::epsilon() *
                            std::max({std::fabs(o.end), std::fabs(time), dt});
    if (remaining - dt <= roundoff) dt = remaining;
    if (!(dt <= p->limit * (1 + 1e-12))) {
        set_error("Requested step %g exceeds advection/diffusion limit %g; reduce step or use control: cfl", dt, p->limit);
        return MP_ERR_ARG_OUTOFRANGE;
    }
    if (!(dt >= o.dt_min || dt == remaining)) { set_error("Stable step is below time.step.minimum"); return MP_ERR_ARG_OUTOFRANGE; }
    if (!(time + dt > time && std::isfinite(dt))) { set_error("Time step does not advance finite time"); return MP_ERR_FP; }
    next = dt == remaining ? o.end : time + dt;
    return MP_OK;
}

}  // namespace
}  // namespace mp

// -------------------------------------------------------------------- C ABI

namespace {
mp_status preheat_create_impl(const mp_mesh_desc* mesh, const double* xy, const mp_preheat_opts* opts,
                              mp_stream_t stream, mp_preheat** out) {
    using namespace mp;
    if (!mesh || !opts || !out) { set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (mesh->nx < 2 || mesh->ny < 2) { set_error("Preheat requires at least 2x2 cells"); return MP_ERR_ARG_SIZ; }
    if (mesh_too_large(mesh->nx, mesh->ny)) { set_error("mesh has 2^31 edges or more"); return MP_ERR_ARG_SIZ; }
    if (!(opts->cfl > 0 && opts->cfl <= 1)) { set_error("Explicit preheat requires time.step.cfl <= 1"); return MP_ERR_ARG_OUTOFRANGE; }
    if (opts->control != MP_TIME_CFL && opts->control != MP_TIME_FIXED) { set_error("unknown time control"); return MP_ERR_ARG_OUTOFRANGE; }
    if (!(std::isfinite(opts->end) && opts->dt_initial > 0 && opts->dt_max > 0 && opts->dt_min >= 0 && opts->max_steps >= 0)) {
        set_error("time controls must be finite and positive");
        return MP_ERR_ARG_OUTOFRANGE;
    }
    if (!(std::isfinite(opts->diffusivity) && opts->diffusivity >= 0.0)) { set_error("Diffusivity must be finite and nonnegative"); return MP_ERR_ARG_OUTOFRANGE; }
    if (opts->H_policy < 0 || opts->H_policy > 2 || !std::isfinite(opts->inflow_H)) { set_error("unknown boundary policy"); return MP_ERR_ARG_OUTOFRANGE; }
    if (opts->lf_global && !(std::isfinite(opts->lf_global_speed) && opts->lf_global_speed >= 0)) {
        set_error("Global LF speed must be finite and nonnegative");
        return MP_ERR_ARG_OUTOFRANGE;
    }
    for (int w = 0; w < 4; ++w)
        if (opts->thermal_type[w] < 0 || opts->thermal_type[w] > 2 || !std::isfinite(opts->thermal_value[w])) {
            set_error("thermal condition of wall %d: unknown type or non-finite value", w);
            return MP_ERR_ARG_OUTOFRANGE;
        }
    mp_derived der;
    MP_TRY(derive_checked(opts->material, der));
    QuadTables qt;
    if (xy) {
        long long bad = -1;
        if (validate_quads(mesh->nx, mesh->ny, xy, &bad)) {
            set_error("Mesh has non-real/non-finite coordinates or an inverted, degenerate, or nearly singular "
                      "quadrilateral (cell %lld)", bad);
            return MP_ERR_ARG_WRONG;
        }
        // Vertices and edge spacing on the host; the per-cell tables are
        // built on the GPU below.
        const int qs = build_quad_tables(mesh->nx, mesh->ny, xy, 0, qt, 0, mesh->ny, false);
        if (qs) { set_error("per-cell stencil table construction failed"); return (mp_status)qs; }
    }
    mp_preheat* p = new mp_preheat;
    p->mesh = *mesh; p->opts = *opts; p->der = der;
    p->stream = (cudaStream_t)stream;
    p->nx = mesh->nx; p->ny = mesh->ny;
    p->N = (size_t)p->nx * p->ny;
    p->NE = (size_t)p->nx * (p->ny + 1) + (size_t)(p->nx + 1) * p->ny;
    Physics& ph = p->ph;
    ph = Physics{};
    ph.k = phase_const(opts->material, der);
    ph.sk = stage_const(ph.k);
    if (opts->pressure_model == MP_PRESSURE_CONSTANT) {
        double Tep;
        if (!(opts->pressure >= 0) || eutectic_temperature(ph.k, opts->pressure, Tep)) {
            delete p; set_error("pressure must be finite and nonnegative"); return MP_ERR_ARG_OUTOFRANGE;
        }
        ph.Tep = Tep;
        ph.litho = 0;
    } else if (opts->pressure_model == MP_PRESSURE_LITHOSTATIC) {
        if (!(std::isfinite(opts->pressure) && opts->pressure >= mesh->y1)) {
            delete p; set_error("surface_y must be at or above the mesh top"); return MP_ERR_ARG_OUTOFRANGE;
        }
        const long double b = (long double)opts->material.rho * opts->material.g * der.l0 / opts->material.nu / der.dT;
        ph.litho = 1; ph.tep_a = der.TDe0; ph.tep_b = (double)b; ph.surface = opts->pressure;
    } else {
        delete p; set_error("unknown pressure model"); return MP_ERR_ARG_OUTOFRANGE;
    }
    PreheatPhys& pp = p->pp;
    pp.kappa = opts->diffusivity;
    pp.diffusion = opts->diffusivity > 0.0;
    for (int w = 0; w < 4; ++w) {
        pp.wall_type[w] = opts->thermal_type[w];
        pp.wall_value[w] = opts->thermal_type[w] == MP_THERMAL_ZERO_FLUX ? 0.0 : opts->thermal_value[w];
        if (opts->thermal_type[w] == MP_THERMAL_FLUX) pp.diffusion = 1;
    }
    pp.Hpol = opts->H_policy; pp.inflowH = opts->inflow_H;
    pp.lf_global = opts->lf_global; pp.lf_speed = opts->lf_global_speed;
    if (!xy) {
        const int tb = build_stage_tables(mesh->nx, mesh->ny, mesh->x0, mesh->x1, mesh->y0, mesh->y1, p->host_tab);
        if (tb) { delete p; set_error("stencil table construction failed"); return (mp_status)tb; }
        make_param_tables(p->host_tab, p->ptab);
    }
    p->blocks = (int)((p->N + kPreCells - 1) / kPreCells);
    const size_t N = p->N, NE = p->NE;
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void** q, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(q, bytes); };
    for (double** q : {&p->Hb[0], &p->Hb[1], &p->C, &p->rate, &p->rhs, &p->T, &p->phi}) alloc((void**)q, N * sizeof(double));
    alloc((void**)&p->rec, 9 * N * sizeof(double));
    alloc((void**)&p->vn, NE * kNQ * sizeof(double));
    alloc((void**)&p->flux, NE * sizeof(double));
    alloc((void**)&p->rr, 2 * NE * sizeof(double));
    alloc((void**)&p->partial, (size_t)p->blocks * sizeof(PrePartial));
    alloc((void**)&p->ctl, sizeof(PreCtl));
    alloc((void**)&p->rows, kBatch * sizeof(PreRow));
    alloc((void**)&p->d_status, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&p->h_ctl, sizeof(PreCtl));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&p->h_rows, kBatch * sizeof(PreRow));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&p->h_status, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(p->vn, 0, NE * kNQ * sizeof(double), p->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->ctl, 0, sizeof(PreCtl), p->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->d_status, 0xff, sizeof(unsigned long long), p->stream);
    if (xy && e == cudaSuccess) {
        const int gs = upload_quad_tables(p->nx, p->ny, xy, qt, 0, p->ny, p->stream, &p->qbuf, p->qdev, &e);
        p->quad = true;
        if (gs == MP_ERR_ARG_WRONG) {
            pre_free(p); delete p;
            set_error("per-cell stencil table construction failed (singular stencil or degenerate cell)");
            return (mp_status)gs;
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) { pre_free(p); delete p; return cuda_status(e, "mp_preheat_create"); }
    *out = p;
    return MP_OK;
}
}  // namespace

extern "C" mp_status mp_preheat_create(const mp_mesh_desc* mesh, const mp_preheat_opts* opts, mp_stream_t stream,
                                       mp_preheat** out) {
    return preheat_create_impl(mesh, nullptr, opts, stream, out);
}

extern "C" mp_status mp_preheat_create_quads(const mp_mesh_desc* mesh, const double* xy, const mp_preheat_opts* opts,
                                             mp_stream_t stream, mp_preheat** out) {
    if (!xy) { mp::set_error("null vertex array"); return MP_ERR_ARG_WRONG; }
    return preheat_create_impl(mesh, xy, opts, stream, out);
}

extern "C" void mp_preheat_destroy(mp_preheat* p) {
    if (!p) return;
    cudaStreamSynchronize(p->stream);
    mp::pre_free(p);
    delete p;
}

extern "C" mp_status mp_preheat_set_velocity(mp_preheat* p, const double* vn) {
    if (!p || !vn) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    MP_CUDA(cudaMemcpyAsync(p->vn, vn, p->NE * mp::kNQ * sizeof(double), cudaMemcpyDefault, p->stream));
    MP_CUDA(cudaStreamSynchronize(p->stream));
    p->ready = false;
    return MP_OK;
}

extern "C" mp_status mp_preheat_set_state(mp_preheat* p, const double* H, const double* C, double time,
                                          long long accepted) {
    if (!p || !H || !C) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (!std::isfinite(time)) { mp::set_error("Nonfinite source time"); return MP_ERR_ARG_OUTOFRANGE; }
    MP_CUDA(cudaMemcpyAsync(p->Hb[0], H, p->N * sizeof(double), cudaMemcpyDefault, p->stream));
    MP_CUDA(cudaMemcpyAsync(p->C, C, p->N * sizeof(double), cudaMemcpyDefault, p->stream));
    MP_CUDA(cudaStreamSynchronize(p->stream));
    p->cur = 0;
    p->time = time;
    p->accepted = accepted;
    p->steps = 0;
    p->ready = false;
    return MP_OK;
}

extern "C" mp_status mp_preheat_get_state(mp_preheat* p, double* H, double* time, long long* accepted) {
    if (!p) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (H) {
        MP_CUDA(cudaMemcpyAsync(H, p->Hb[p->cur], p->N * sizeof(double), cudaMemcpyDefault, p->stream));
        MP_CUDA(cudaStreamSynchronize(p->stream));
    }
    if (time) *time = p->time;
    if (accepted) *accepted = p->accepted;
    return MP_OK;
}

extern "C" mp_status mp_preheat_begin(mp_preheat* p, double* rate, double* limit, mp_preheat_step* first) {
    using namespace mp;
    if (!p) { set_error("null argument"); return MP_ERR_ARG_WRONG; }
    p->ready = false;
    if (!(p->time <= p->opts.end)) { set_error("State time exceeds time.end"); return MP_ERR_ARG_OUTOFRANGE; }
    MP_TRY(reset_status(p));
    if (p->quad)
        pre_quad_rate_edge_kernel<<<(unsigned)((p->NE + 127) / 128), 128, 0, p->stream>>>(p->nx, p->ny, p->vn, p->rr,
                                                                                          p->d_status, p->pp, p->qdev);
    else
        pre_rate_edge_kernel<<<(unsigned)((p->NE + 127) / 128), 128, 0, p->stream>>>(p->nx, p->ny, p->host_tab.area,
                                                                                     p->vn, p->rr, p->d_status, p->pp,
                                                                                     p->ptab);
    pre_rate_cell_kernel<<<p->blocks, kPreBlock, 0, p->stream>>>(p->nx, p->ny, p->rr, p->rate, p->partial, p->ctl);
    count_launch(2);
    MP_CUDA(cudaGetLastError());
    MP_TRY(read_status(p));
    MP_TRY(pre_status(p, "mp_preheat_begin"));
    const PrePartial rt = p->h_ctl->last;
    if (rt.nonfinite != 0.0) { set_error("Nonfinite preheat rate"); return MP_ERR_FP; }
    p->rate_max = rt.maximum;
    p->limit = p->rate_max > 0 ? p->opts.cfl / p->rate_max : p->opts.dt_max;
    // Integral, minimum and maximum of the initial H (preheat.cpp:245-249).
    launch_update(p, p->Hb[p->cur], nullptr, PRE_MEASURE, 0.0, 0);
    MP_CUDA(cudaGetLastError());
    MP_TRY(read_status(p));
    const PrePartial m = p->h_ctl->last;
    MP_CUDA(cudaMemcpyAsync(&p->ctl->prev_integral, &m.integral, sizeof(double), cudaMemcpyHostToDevice, p->stream));
    if (rate) MP_CUDA(cudaMemcpyAsync(rate, p->rate, p->N * sizeof(double), cudaMemcpyDefault, p->stream));
    MP_CUDA(cudaStreamSynchronize(p->stream));
    p->acc_seen = p->h_ctl->accepted;
    p->steps = 0;
    p->ready = true;
    if (limit) *limit = p->limit;
    if (first) {
        *first = mp_preheat_step{};
        first->step = p->accepted; first->time = p->time; first->integral = m.integral;
        first->minimum = m.minimum; first->maximum = m.maximum;
    }
    return MP_OK;
}

extern "C" mp_status mp_preheat_rhs(mp_preheat* p, double* rhs, double* boundary_flux) {
    using namespace mp;
    if (!p) { set_error("null argument"); return MP_ERR_ARG_WRONG; }
    MP_TRY(reset_status(p));
    const double* H = p->Hb[p->cur];
    launch_rhs_kernels(p, H);
    launch_update(p, H, nullptr, PRE_RHS, 0.0, 0);
    MP_CUDA(cudaGetLastError());
    MP_TRY(read_status(p));
    MP_TRY(pre_status(p, "mp_preheat_rhs"));
    if (rhs) {
        MP_CUDA(cudaMemcpyAsync(rhs, p->rhs, p->N * sizeof(double), cudaMemcpyDefault, p->stream));
        MP_CUDA(cudaStreamSynchronize(p->stream));
    }
    if (boundary_flux) *boundary_flux = p->h_ctl->last.bflux;
    return MP_OK;
}

extern "C" mp_status mp_preheat_advance(mp_preheat* p, long long nsteps, mp_preheat_step* rows, long long* taken) {
    mp::NvtxRange range("mp_preheat advance");
    using namespace mp;
    if (taken) *taken = 0;
    if (!p) { set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (!p->ready) { set_error("call mp_preheat_begin after setting the state and velocity"); return MP_ERR_ARG_WRONGSTATE; }
    long long done = 0;
    while (done < nsteps && p->time < p->opts.end) {
        // Plan a batch: dt and the time after each step.
        double dts[kBatch], times[kBatch];
        int n = 0;
        mp_status plan = MP_OK;
        double t = p->time;
        while (n < kBatch && done + n < nsteps && t < p->opts.end) {
            double dt, next;
            plan = plan_step(p, t, p->steps + n, dt, next);
            if (plan != MP_OK) break;
            dts[n] = dt; times[n] = next; t = next; ++n;
        }
        if (n > 0) {
            MP_TRY(reset_status(p));
            for (int k = 0; k < n; ++k) {
                const double* H = p->Hb[(p->cur + k) & 1];
                double* Hn = p->Hb[(p->cur + k + 1) & 1];
                launch_rhs_kernels(p, H);
                launch_update(p, H, Hn, PRE_STEP, dts[k], k);
            }
            MP_CUDA(cudaGetLastError());
            MP_CUDA(cudaMemcpyAsync(p->h_rows, p->rows, (size_t)n * sizeof(PreRow), cudaMemcpyDeviceToHost, p->stream));
            MP_TRY(read_status(p));
            const int m = (int)(p->h_ctl->accepted - p->acc_seen);
            p->acc_seen = p->h_ctl->accepted;
            for (int k = 0; k < m; ++k) {
                const PreRow& r = p->h_rows[k];
                ++p->accepted; ++p->steps;
                p->time = times[k];
                if (rows) {
                    mp_preheat_step& o = rows[done + k];
                    o.step = p->accepted; o.time = times[k]; o.dt = dts[k]; o.courant = dts[k] * p->rate_max;
                    o.integral = r.integral; o.minimum = r.minimum; o.maximum = r.maximum;
                    o.boundaryFlux = r.bflux; o.balanceError = r.balance;
                }
            }
            p->cur = (p->cur + m) & 1;
            done += m;
            if (taken) *taken = done;
            if (m < n) {
                const mp_status s = pre_status(p, "mp_preheat_advance");
                if (s != MP_OK) return s;
                set_error("mp_preheat_advance: step %lld was not accepted", p->accepted + 1);
                return MP_ERR_PLIB;
            }
        }
        if (plan != MP_OK) return plan;
    }
    if (taken) *taken = done;
    return MP_OK;
}

extern "C" mp_status mp_preheat_diagnostics(mp_preheat* p, double* T, double* phi) {
    using namespace mp;
    if (!p) { set_error("null argument"); return MP_ERR_ARG_WRONG; }
    MP_TRY(reset_status(p));
    dim3 blk(32, 4), grd((p->nx + 31) / 32, (p->ny + 3) / 4);
    if (p->quad)
        pre_quad_diag_kernel<<<grd, blk, 0, p->stream>>>(p->nx, p->ny, p->Hb[p->cur], p->C, p->T, p->phi, p->d_status,
                                                         p->ph, p->qdev);
    else
        pre_diag_kernel<<<grd, blk, 0, p->stream>>>(p->nx, p->ny, p->Hb[p->cur], p->C, p->T, p->phi, p->d_status,
                                                    p->ph, p->ptab);
    count_launch();
    MP_CUDA(cudaGetLastError());
    MP_TRY(read_status(p));
    MP_TRY(pre_status(p, "mp_preheat_diagnostics"));
    if (T) MP_CUDA(cudaMemcpyAsync(T, p->T, p->N * sizeof(double), cudaMemcpyDefault, p->stream));
    if (phi) MP_CUDA(cudaMemcpyAsync(phi, p->phi, p->N * sizeof(double), cudaMemcpyDefault, p->stream));
    MP_CUDA(cudaStreamSynchronize(p->stream));
    return MP_OK;
}

extern "C" mp_status mp_preheat_run(mp_preheat* p, mp_preheat_report* report, mp_preheat_step* history,
                                    long long capacity, long long* rows, double* T, double* phi) {
    if (rows) *rows = 0;
    if (!p) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    mp_preheat_step first;
    double limit;
    MP_TRY(mp_preheat_begin(p, nullptr, &limit, &first));
    mp_preheat_report rep{};
    rep.initialTime = rep.finalTime = p->time;
    rep.stepLimit = limit;
    rep.initialIntegral = rep.finalIntegral = first.integral;
    long long count = 0;
    if (history && capacity > 0) history[0] = first;
    count = 1;
    std::vector<mp_preheat_step> chunk(mp::kBatch);
    mp_status s = MP_OK;
    while (p->time < p->opts.end) {
        long long got = 0;
        s = mp_preheat_advance(p, mp::kBatch, chunk.data(), &got);
        for (long long k = 0; k < got; ++k) {
            if (history && count < capacity) history[count] = chunk[k];
            ++count;
            rep.finalIntegral = chunk[k].integral;
            rep.boundaryIntegral += chunk[k].dt * chunk[k].boundaryFlux;
        }
        rep.finalTime = p->time;
        if (s != MP_OK || got == 0) break;
    }
    if (rows) *rows = count;
    if (report) *report = rep;
    if (s != MP_OK) return s;
    return mp_preheat_diagnostics(p, T, phi);
}

// Transport stage kernels of a general (logically rectangular) quad mesh:
// perturbed-quadrilateral and stretched meshes, where every cell has its own
// stencil geometry (src/core/mesh.cpp:27-55; src/mlweno/reconstruction.cpp:
// 109-210). Same stage as the uniform kernels (src/couple/evolve.cpp:279-384),
// with
//   * per-cell candidate matrices and smoothness forms read from HBM
//     (quad_tables.hpp) instead of one table set in the kernel parameters;
//   * every evaluation point mapped from the cell's corners (bilinear map,
//     edge interpolation, normal-line samples with per-edge spacing) into the
//     cell's frame, and the limited polynomial evaluated as a full Q2 form;
//   * physical edge lengths, normals and cell areas of each cell and edge.
// The per-point physics (phase, porosity, velocities, fluxes, rate) is the
// uniform kernels' own device code.
#ifndef MP_QUAD_KERNELS_CUH
#define MP_QUAD_KERNELS_CUH

#include "common.hpp"
#include "phase_math.cuh"
#include "stage_device.cuh"
#include "stage_kernels.cuh"
#include "quad_device.cuh"

namespace mp {
namespace {

// Adiabatic-source inputs and per-cell outputs (null when alpha0 = 0).
struct SourcePtrs {
    const double* cvs_y = nullptr;
    const double* cud_y = nullptr;
    double* srcH = nullptr;
    double* srcR = nullptr;
    double* srcS = nullptr;
};

// Everything one stage of one quad mesh reads and writes (the single-mesh
// launch passes it by value; the batched launch reads one per instance).
struct QuadStageArgs {
    int nx = 0, ny = 0, gj0 = 0, gny = 0;   // local rows; local row 0 is global row gj0 of gny
    const double* H = nullptr;              // stage input
    const double* C = nullptr;
    double* rec = nullptr;                  // 18 * ncell deviation coefficients
    unsigned char* flags = nullptr;
    double* T = nullptr;
    double* phi = nullptr;
    const double* vsn = nullptr;            // [edge*5 + q], canonical
    const double* udn = nullptr;
    double* face = nullptr;                 // 4 * nedge: fluxH, fluxC, rate, fluxMixture
    unsigned long long* status = nullptr;
    double* theta = nullptr;                // optional limiter factors (2 * ncell)
    QuadDev q{};
    SourcePtrs src{};
};

// ------------------------------------------------------------------ kernels

// Reconstruction (Reconstruction::Update, src/mlweno/reconstruction.cpp:
// 275-355) of H and C with the cell's own tables, each table entry read once
// for both fields: the unlimited deviation polynomials into rec. The limiter runs in the next kernel, so that neither
// kernel holds both the table-driven weights and the point scan in
// registers (the table reads need many warps in flight).
__device__ __forceinline__ void quad_weno_cell(const QuadStageArgs& a, int i, int j) {
    const int nx = a.nx, ny = a.ny, gj0 = a.gj0, gny = a.gny;
    const double* __restrict__ H = a.H;
    const double* __restrict__ C = a.C;
    unsigned long long* status = a.status;
    const QuadDev& q = a.q;
    double* __restrict__ rec = a.rec;
    const long long cell = (long long)j * nx + i;
    const size_t N = (size_t)nx * ny;
    MP_CHECK_INDEX(status, cell, N);
    const int gj = gj0 + j;
    const int ci = i == 0 ? 0 : (i == nx - 1 ? 2 : 1), cj = gj == 0 ? 0 : (gj == gny - 1 ? 2 : 1);
    const double eA = 1e-2 * __ldg(q.geo + 3 * N + cell);
    double u[2][3][3];
#pragma unroll
    for (int dj = 0; dj < 3; ++dj)
#pragma unroll
        for (int di = 0; di < 3; ++di) {
            const int ii = min(max(i + di - 1, 0), nx - 1), jj = min(max(j + dj - 1, 0), ny - 1);
            MP_CHECK_INDEX(status, (long long)jj * nx + ii, N);
            u[0][dj][di] = __ldg(H + (size_t)jj * nx + ii);
            u[1][dj][di] = __ldg(C + (size_t)jj * nx + ii);
        }
    double D[2][9];
    const int st = reconstruct_quad<2>(q, N, cell, ci, cj, eA, u, D);
#pragma unroll
    for (int m = 0; m < 9; ++m) {
        rec[(size_t)m * N + cell] = D[0][m];
        rec[(size_t)(m + 9) * N + cell] = D[1][m];
    }
    if (st) record_error(status, PART_UPDATE, cell + (long long)gj0 * nx, st);
}
__global__ void __launch_bounds__(128, 3) quad_weno_kernel(const __grid_constant__ QuadStageArgs a, int jlo, int jhi,
                                                           const int* gate) {
    if (gated_off(gate)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = jlo + (int)(blockIdx.y * blockDim.y + threadIdx.y);
    if (i >= a.nx || j >= jhi) return;
    quad_weno_cell(a, i, j);
}

// Limiter over the cell's own limiter points (state_reconstruction.cpp:
// 136-192): theta of H and C from the unlimited polynomials in rec, which
// are scaled in place.
__device__ __forceinline__ void quad_limit_cell(const QuadStageArgs& a, const Physics& ph, int i, int j) {
    const int nx = a.nx, ny = a.ny, gj0 = a.gj0, gny = a.gny;
    const double* __restrict__ H = a.H;
    const double* __restrict__ C = a.C;
    unsigned long long* status = a.status;
    const QuadDev& q = a.q;
    double* __restrict__ rec = a.rec;
    unsigned char* __restrict__ flags = a.flags;
    double* theta = a.theta;
    const long long cell = (long long)j * nx + i;
    const size_t N = (size_t)nx * ny;
    MP_CHECK_INDEX(status, cell, N);
    const CellFrame f = cell_frame(q, nx, N, cell);
    double DH[9], DC[9];
    load_rec(rec, N, cell, DH, DC);
    // 3x3 neighbour bounds of the averages (state_reconstruction.cpp:189-196).
    double lo[2], hi[2], m[2];
#pragma unroll
    for (int fi = 0; fi < 2; ++fi) {
        const double* F = fi ? C : H;
        m[fi] = __ldg(F + cell);
        lo[fi] = m[fi]; hi[fi] = m[fi];
#pragma unroll
        for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
            for (int di = -1; di <= 1; ++di) {
                const int ii = min(max(i + di, 0), nx - 1), jj = min(max(j + dj, 0), ny - 1);
                MP_CHECK_INDEX(status, (long long)jj * nx + ii, N);
                const double v = __ldg(F + (size_t)jj * nx + ii);
                lo[fi] = fmin(lo[fi], v); hi[fi] = fmax(hi[fi], v);
            }
    }
    const double mH = m[0], mC = m[1];
    const double loH = fmax(0.0, lo[0]), hiH = hi[0], loC = fmax(0.0, lo[1]), hiC = fmin(ph.k.Xe, hi[1]);
    int st_lim = 0;
    if (!(isfinite(mH) && mH >= 0.0 && isfinite(mC) && mC >= 0.0 && mC <= ph.k.Xe)) st_lim = E_OUTOFRANGE;
    double hmx = -INFINITY, hmn = INFINITY, cmx = -INFINITY, cmn = INFINITY;
    bool bad = false;
    auto visit = [&](P2 p) {
        const double x = (p.x - f.cx) * f.inv_h, y = (p.y - f.cy) * f.inv_h;
        const double vh = q2v(DH, x, y), vc = q2v(DC, x, y);
        bad = bad || !isfinite(vh) || !isfinite(vc);
        hmx = fmax(hmx, vh); hmn = fmin(hmn, vh);
        cmx = fmax(cmx, vc); cmn = fmin(cmn, vc);
    };
    // Limiter points (state_reconstruction.cpp:152-168): centre, 5x5 Gauss
    // points, 5 points per edge, the normal-line samples on this side.
    visit(bilinear(0.0, 0.0, f.c));
    for (int a = 0; a < kNQ; ++a)
        for (int b = 0; b < kNQ; ++b) visit(bilinear(q.gq[a], q.gq[b], f.c));
    for (int e = 0; e < 4; ++e)
        for (int k = 0; k < kNQ; ++k) visit(lerp_edge(q.gq[k], f.c[e], f.c[(e + 1) & 3]));
    visit_samples(q, nx, ny, gj0, gny, i, j, f, visit);
    if (bad) st_lim = st_lim ? st_lim : E_FP;
    const double thH = theta_of(mH, loH, hiH, hmx, hmn);
    const double thC = theta_of(mC, loC, hiC, cmx, cmn);
    if (theta) { theta[cell] = thH; theta[N + cell] = thC; }
    // Diffusion-sample admissibility as the uniform path: provably safe when
    // the largest neighbour average is below the liquidus at the lowest
    // eutectic temperature over the cell's height range.
    double ylo = f.c[0].y, yhi = f.c[0].y;
    for (int k = 1; k < 4; ++k) { ylo = fmin(ylo, f.c[k].y); yhi = fmax(yhi, f.c[k].y); }
    const double tep = ph.litho ? fmin(tep_at(ph, ylo), tep_at(ph, yhi)) : ph.Tep;
    const double Hliq = tep + (1.0 - hiC / ph.k.Xe) + ph.k.LD;
    const bool safe = tep >= 0.0 && hiH + 1e-12 * (1.0 + fabs(hiH)) < Hliq;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        rec[(size_t)k * N + cell] = DH[k] * thH;
        rec[(size_t)(k + 9) * N + cell] = DC[k] * thC;
    }
    flags[cell] = safe ? 0 : FLAG_CHECK;
    if (st_lim) record_error(status, PART_LIMIT, cell + (long long)gj0 * nx, st_lim);
}
__global__ void __launch_bounds__(128, 4) quad_limit_kernel(const __grid_constant__ QuadStageArgs a, Physics ph, int jlo,
                                                         int jhi, const int* gate) {
    if (gated_off(gate)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = jlo + (int)(blockIdx.y * blockDim.y + threadIdx.y);
    if (i >= a.nx || j >= jhi) return;
    quad_limit_cell(a, ph, i, j);
}


// 5x5 cell quadrature of T and phi on the bilinear map, wet flag, adiabatic
// source, and the exact check of the diffusion samples when flagged.
__device__ __forceinline__ void quad_cellphase_cell(const QuadStageArgs& a, const Physics& ph, long long cell) {
    const int nx = a.nx, ny = a.ny, gj0 = a.gj0, gny = a.gny;
    const double* __restrict__ H = a.H;
    const double* __restrict__ C = a.C;
    unsigned long long* status = a.status;
    const QuadDev& q = a.q;
    const double* __restrict__ rec = a.rec;
    unsigned char* __restrict__ flags = a.flags;
    double* __restrict__ T = a.T;
    double* __restrict__ phi = a.phi;
    const SourcePtrs& src = a.src;
    const long long N = (long long)nx * ny;
    MP_CHECK_INDEX(status, cell, N);
    const int i = (int)(cell % nx), j = (int)(cell / nx);
    const CellFrame f = cell_frame(q, nx, (size_t)N, cell);
    const double mH = __ldg(H + cell), mC = __ldg(C + cell);
    double DH[9], DC[9];
    load_rec(rec, (size_t)N, cell, DH, DC);
    int st_por = 0, st_cell = 0, st_face = 0;
    double Tsum = 0.0, Psum = 0.0, Ssum = 0.0, Rsum = 0.0, Wsum = 0.0;
    bool wet = false;
    for (int b = 0; b < kNQ; ++b)
        for (int a = 0; a < kNQ; ++a) {
            const P2 p = bilinear(q.gq[a], q.gq[b], f.c);
            const double wj = q.gw[a] * q.gw[b] * jacobian(q.gq[a], q.gq[b], f.c);
            const double x = (p.x - f.cx) * f.inv_h, y = (p.y - f.cy) * f.inv_h;
            const double tep = ph.litho ? tep_at(ph, p.y) : ph.Tep;
            PhaseLean pl;
            const int s = phase_stage_lean(ph.sk, mH + q2v(DH, x, y), mC + q2v(DC, x, y), tep, pl);
            if (s) { st_por = st_por ? st_por : s; continue; }
            if (!(pl.T >= 0.0 && pl.phil < 1.0)) st_cell = st_cell ? st_cell : E_OUTOFRANGE;
            const double w = wj / f.area;
            Tsum += w * pl.T;
            Psum += w * pl.phil;
            wet = wet || pl.phil > 0.0;
            if (ph.source) {
                const long long at = cell * (kNQ * kNQ) + b * kNQ + a;
                const double factor = pl.phil == 0.0 ? 0.0 : (ph.theta == 0.0 ? pl.phil : pow(pl.phil, 1.0 + ph.theta));
                const double vy = __ldg(src.cvs_y + at) + factor * __ldg(src.cud_y + at);
                const double s_ = -ph.cooling * pl.T * vy;
                Ssum += w * s_;
                Rsum += w * ph.cooling * fabs(vy);
                Wsum += wj * s_;
            }
        }
    const unsigned char fl = flags[cell];
    if (fl & FLAG_CHECK) {
        visit_samples(q, nx, ny, gj0, gny, i, j, f, [&](P2 p) {
            const double x = (p.x - f.cx) * f.inv_h, y = (p.y - f.cy) * f.inv_h;
            const double tep = ph.litho ? tep_at(ph, p.y) : ph.Tep;
            PhaseLean pl;
            const int s = phase_stage_lean(ph.sk, mH + q2v(DH, x, y), mC + q2v(DC, x, y), tep, pl);
            if (s) { st_face = st_face ? st_face : s; return; }
            if (!(pl.T >= 0.0 && pl.phil < 1.0)) st_face = st_face ? st_face : E_OUTOFRANGE;
        });
    }
    const long long key = cell + (long long)gj0 * nx;
    if (st_por) record_error(status, PART_POROSITY, key, st_por);
    if (st_face) record_error(status, PART_FACES, key, st_face);
    if (st_cell) record_error(status, PART_CELLS, key, st_cell);
    flags[cell] = (unsigned char)((fl & FLAG_CHECK) | (wet ? FLAG_WET : 0));
    T[cell] = Tsum;
    phi[cell] = Psum;
    if (ph.source) { src.srcH[cell] = Ssum; src.srcR[cell] = Rsum; src.srcS[cell] = Wsum; }
}
__global__ void __launch_bounds__(128, 4) quad_cellphase_kernel(const __grid_constant__ QuadStageArgs a, Physics ph,
                                                             long long c0, long long c1, const int* gate) {
    if (gated_off(gate)) return;
    const long long cell = c0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= c1) return;
    quad_cellphase_cell(a, ph, cell);
}


struct Side {
    double cx, cy, inv_h, mH, mC;
    double DH[9], DC[9];
};
__device__ __forceinline__ void load_side(const QuadDev& q, size_t N, const double* H, const double* C,
                                          const double* rec, long long cell, Side& s) {
    s.cx = __ldg(q.geo + cell);
    s.cy = __ldg(q.geo + N + cell);
    s.inv_h = 1.0 / __ldg(q.geo + 2 * N + cell);
    s.mH = __ldg(H + cell);
    s.mC = __ldg(C + cell);
    load_rec(rec, N, cell, s.DH, s.DC);
}
__device__ __forceinline__ void side_values(const Side& s, P2 p, double& h, double& c) {
    const double x = (p.x - s.cx) * s.inv_h, y = (p.y - s.cy) * s.inv_h;
    h = s.mH + q2v(s.DH, x, y);
    c = s.mC + q2v(s.DC, x, y);
}

// Face fluxes, edge porosity and rate of one edge at its 5 Gauss points.
__device__ __forceinline__ void quad_face_edge(const QuadStageArgs& a, const Physics& ph, long long e) {
    const int nx = a.nx, ny = a.ny, gj0 = a.gj0, gny = a.gny;
    const double* __restrict__ H = a.H;
    const double* __restrict__ C = a.C;
    unsigned long long* status = a.status;
    const QuadDev& q = a.q;
    const double* __restrict__ rec = a.rec;
    const unsigned char* __restrict__ flags = a.flags;
    const double* __restrict__ vsn = a.vsn;
    const double* __restrict__ udn = a.udn;
    double* __restrict__ face = a.face;
    const long long nE = (long long)nx * (ny + 1) + (long long)(nx + 1) * ny;
    const size_t N = (size_t)nx * ny;
    MP_CHECK_INDEX(status, e, nE);
    const QuadEdge g = quad_edge(q, nx, ny, gj0, gny, e);
    MP_CHECK_INDEX(status, g.L, N);
    if (!g.boundary) MP_CHECK_INDEX(status, g.R, N);
    double len;
    P2 nrm;
    edge_geometry(g.a, g.b, len, nrm);
    Side sl, sr;
    load_side(q, N, H, C, rec, g.L, sl);
    if (!g.boundary) load_side(q, N, H, C, rec, g.R, sr);
    const bool wetL = (flags[g.L] & FLAG_WET) != 0, wetR = g.boundary ? true : (flags[g.R] & FLAG_WET) != 0;
    const double sgn = g.reverse ? -1.0 : 1.0;
    double fluxH = 0.0, fluxC = 0.0, fluxMix = 0.0, rate = 0.0;
    int st = 0;
    for (int k = 0; k < kNQ; ++k) {
        const int cq = g.reverse ? kNQ - 1 - k : k;
        const P2 p = lerp_edge(q.gq[k], g.a, g.b);
        const double vs = sgn * __ldg(vsn + e * kNQ + cq);
        const double ud = sgn * __ldg(udn + e * kNQ + cq);
        const double tep = ph.litho ? tep_at(ph, p.y) : ph.Tep;
        double hL, cL, hR, cR;
        PhaseLean A, B;
        side_values(sl, p, hL, cL);
        int s = phase_stage(ph.sk, hL, cL, tep, A);
        if (!s && !(A.T >= 0.0 && A.phil < 1.0)) s = E_OUTOFRANGE;
        if (g.boundary) { B = A; hR = hL; cR = cL; }
        else {
            side_values(sr, p, hR, cR);
            int s2 = phase_stage(ph.sk, hR, cR, tep, B);
            if (!s2 && !(B.T >= 0.0 && B.phil < 1.0)) s2 = E_OUTOFRANGE;
            s = s ? s : s2;
        }
        if (s) { st = st ? st : s; continue; }
        const PointFlux pf = face_point(ph, A, B, cL, cR, wetL, wetR, g.boundary, vs, ud, tep, ph.k.LD, st);
        const double w = 0.5 * len * q.gw[k];
        fluxH += w * pf.fh;
        fluxC += w * pf.fc;
        fluxMix += w * pf.vn;
        rate += w * pf.speed;
    }
    if (st) record_error(status, PART_FACES, g.L + (long long)gj0 * nx, st);
    face[e] = fluxH;
    face[nE + e] = fluxC;
    face[2 * nE + e] = rate;
    face[3 * nE + e] = fluxMix;
}
__global__ void __launch_bounds__(128, 4) quad_face_kernel(const __grid_constant__ QuadStageArgs a, Physics ph,
                                                        long long h0, long long nh, long long v0, long long nv,
                                                        const int* gate) {
    if (gated_off(gate)) return;
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nh + nv) return;
    quad_face_edge(a, ph, k < nh ? h0 + k : v0 + (k - nh));
}


// Diffusive H flux and rate of one edge (diffusiveflux.cpp:105-200 through
// evolve.cpp:330-347): temperatures of the limited states at the normal-line
// samples, spacing per edge point.
__device__ __forceinline__ void quad_diffusion_edge(const QuadStageArgs& a, const Physics& ph, long long e) {
    const int nx = a.nx, ny = a.ny, gj0 = a.gj0, gny = a.gny;
    const double* __restrict__ H = a.H;
    const double* __restrict__ C = a.C;
    unsigned long long* status = a.status;
    const QuadDev& q = a.q;
    const double* __restrict__ rec = a.rec;
    double* __restrict__ face = a.face;
    const long long nE = (long long)nx * (ny + 1) + (long long)(nx + 1) * ny;
    const size_t N = (size_t)nx * ny;
    MP_CHECK_INDEX(status, e, nE);
    const QuadEdge g = quad_edge(q, nx, ny, gj0, gny, e);
    MP_CHECK_INDEX(status, g.L, N);
    if (!g.boundary) MP_CHECK_INDEX(status, g.R, N);
    const int type = g.boundary ? ph.wall_type[g.wall] : 1;
    if (g.boundary && type == 0) return;
    double len;
    P2 nrm;
    edge_geometry(g.a, g.b, len, nrm);
    Side sl, sr;
    if (type == 1) {
        load_side(q, N, H, C, rec, g.L, sl);
        if (!g.boundary) load_side(q, N, H, C, rec, g.R, sr);
    }
    double integral = 0.0, rate = face[2 * nE + e];
    const double kappa = ph.kappa;
    int st = 0;
    for (int k = 0; k < kNQ; ++k) {
        const double w = len * q.gw[k] / 2;
        if (g.boundary && type == 2) { integral += w * ph.wall_value[g.wall]; continue; }
        const int cq = g.reverse ? kNQ - 1 - k : k;
        const P2 p = lerp_edge(q.gq[k], g.a, g.b);
        const double sp = __ldg(q.sp + e * kNQ + cq);
        const int count = g.boundary ? 5 : 4;
        double v[5];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const bool left = g.boundary || s < 2;
            const double d = (g.boundary ? (double)(s - 4) : (double)s - 1.5) * sp;
            const P2 x = P2{p.x + d * nrm.x, p.y + d * nrm.y};
            double h, c;
            side_values(left ? sl : sr, x, h, c);
            const double tep = ph.litho ? tep_at(ph, x.y) : ph.Tep;
            PhaseLean pl;
            int s1 = phase_stage_lean(ph.sk, h, c, tep, pl);
            if (!s1 && !(pl.T >= 0.0 && pl.phil < 1.0)) s1 = E_OUTOFRANGE;
            if (s1) st = st ? st : s1;
            v[s] = s1 ? 0.0 : pl.T;
        }
        v[4] = g.boundary ? ph.wall_value[g.wall] : 0.0;
        const double* c = g.boundary ? q.dif_c_bnd : q.dif_c_int;
        const double last = v[count - 1];
        double grad = 0.0, clast = 0.0;
        for (int s = 0; s + 1 < count; ++s) { grad += c[s] * (v[s] - last); clast -= c[s]; }
        grad /= sp;
        if (!isfinite(grad)) st = st ? st : E_FP;
        integral -= w * kappa * grad;
        const double scale = -w * kappa / sp;
        for (int s = 0; s < count; ++s) {
            if (g.boundary && s + 1 == count) continue;
            rate += fabs(scale * (s + 1 == count ? clast : c[s]));
        }
    }
    if (st) record_error(status, PART_FACES, g.L + (long long)gj0 * nx, st);
    face[e] += integral;
    face[2 * nE + e] = rate;
}
__global__ void __launch_bounds__(128) quad_diffusion_kernel(const __grid_constant__ QuadStageArgs a, Physics ph,
                                                             long long h0, long long nh, long long v0, long long nv,
                                                             const int* gate) {
    if (gated_off(gate)) return;
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nh + nv) return;
    quad_diffusion_edge(a, ph, k < nh ? h0 + k : v0 + (k - nh));
}


// Reconstruction, limiter, cell phase, faces (+ diffusion) of state (H, C)
// on a general quad mesh; the accumulation is the shared sum kernel. Local
// rows [rec0, rec1) are reconstructed, the edges [h0, h0+nh) and [v0, v0+nv)
// (those of the advanced rows) get fluxes; local row 0 is global row gj0 of
// gny (a whole mesh: gj0 = 0, gny = ny). gate: device flag, every kernel
// returns at once while it is 0 (the device-resident step graph).
void launch_quad_stage(const QuadDev& q, int nx, int ny, int gj0, int gny, int rec0, int rec1, long long h0,
                       long long nh, long long v0, long long nv, const Physics& ph, const double* H, const double* C,
                       double* rec, unsigned char* flags, double* T, double* phi, const double* vsn, const double* udn,
                       double* face, unsigned long long* status, double* theta, const SourcePtrs& src,
                       cudaStream_t s, const int* gate = nullptr) {
    QuadStageArgs a;
    a.nx = nx; a.ny = ny; a.gj0 = gj0; a.gny = gny;
    a.H = H; a.C = C; a.rec = rec; a.flags = flags; a.T = T; a.phi = phi;
    a.vsn = vsn; a.udn = udn; a.face = face; a.status = status; a.theta = theta;
    a.q = q; a.src = src;
    dim3 blk(32, 4), grd((nx + 31) / 32, (rec1 - rec0 + 3) / 4);
    quad_weno_kernel<<<grd, blk, 0, s>>>(a, rec0, rec1, gate);
    quad_limit_kernel<<<grd, blk, 0, s>>>(a, ph, rec0, rec1, gate);
    const long long c0 = (long long)rec0 * nx, c1 = (long long)rec1 * nx;
    quad_cellphase_kernel<<<(unsigned)((c1 - c0 + 127) / 128), 128, 0, s>>>(a, ph, c0, c1, gate);
    const unsigned ge = (unsigned)((nh + nv + 127) / 128);
    quad_face_kernel<<<ge, 128, 0, s>>>(a, ph, h0, nh, v0, nv, gate);
    count_launch(4);
    if (ph.diffusion) {
        quad_diffusion_kernel<<<ge, 128, 0, s>>>(a, ph, h0, nh, v0, nv, gate);
        count_launch();
    }
}

}  // namespace
}  // namespace mp

#endif

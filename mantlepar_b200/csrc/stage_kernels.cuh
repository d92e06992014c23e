// Per-element device functions of the transport stage, shared by the
// single-instance kernels (transport.cu) and the batched kernels (batch.cu).
//
// recon_cell      reconstruction, weights, limiter theta (one cell)
// cellphase_cell  5x5 phase quadrature of T, phi and the wet flag (one cell)
// face_edge       limited values, phase, porosity, LF flux and rate (one edge)
// sum_cell        reference-ordered accumulation and RK combination (one cell)
#ifndef MP_STAGE_KERNELS_CUH
#define MP_STAGE_KERNELS_CUH

#include "common.hpp"
#include "phase_math.cuh"
#include "stage_device.cuh"
#include "tables.hpp"

namespace mp {
namespace {

constexpr int kRec = 18;          // limited deviation coefficients: 9 for H, 9 for C
constexpr int kRedBlock = 256;
// The accumulation and axpy kernels give each thread kSumPer cells (strided
// by the block size, so loads stay coalesced) before one block reduction.
constexpr int kSumPer = 4;
constexpr int kSumCells = kRedBlock * kSumPer;

enum : int {
    E_OUTOFRANGE = MP_ERR_ARG_OUTOFRANGE, E_FP = MP_ERR_FP, E_WRONG = MP_ERR_ARG_WRONG
};

struct Physics {
    PhaseConst k;
    StageConst sk;
    double Tep;            // pressure-corrected eutectic temperature (constant pressure)
    double theta;          // Darcy exponent
    double inflowH, inflowC;
    int Hpol, Cpol, lf_global;
    double lf_speed;
    // Thermal diffusion: on when kappa > 0 or a wall prescribes a flux.
    // Walls 0 bottom, 1 top, 2 left, 3 right: 0 zero flux, 1 prescribed
    // temperature, 2 prescribed outward flux (per unit length).
    int diffusion;
    double kappa;
    int wall_type[4];
    double wall_value[4];
    // Phase-law pressure: constant (litho = 0, Tep above), or lithostatic
    // rho g l0 (surface - y): Tep(y) = tep_a + tep_b (surface - y).
    int litho;
    double tep_a, tep_b, surface;
    // Adiabatic source -cooling T v_mix,y (evolve.cpp:359-369), cooling =
    // alpha0 l0 g / cp; on when alpha0 != 0.
    int source;
    double cooling;
};

// Pressure-corrected eutectic temperature at height y (one FMA for the
// lithostatic model; the constant model returns the stored value exactly).
__device__ __forceinline__ double tep_at(const Physics& ph, double y) {
    return ph.litho ? fma(ph.tep_b, ph.surface - y, ph.tep_a) : ph.Tep;
}

// Height of a point at normalised eta in the cell of global row gj.
__device__ __forceinline__ double height(const StageHot& t, int gj, double eta) {
    return t.y0 + (gj + 0.5) * t.dy + eta * t.hn;
}

// Block partials of one stage (sum_kernel) or state check (axpy_kernel).
struct Partial {
    double maxRate, divergence, bH, bC, HI, CI, Hmin, Cmin, Cmax;
    double nonfinite;
    double sH;             // adiabatic source integral
};

__device__ __forceinline__ Partial partial_identity() {
    return Partial{-INFINITY, 0.0, 0.0, 0.0, 0.0, 0.0, INFINITY, INFINITY, -INFINITY, 0.0, 0.0};
}

struct Totals {
    double maxRate, divergence, bH, bC, HI, CI, Hmin, Cmin, Cmax;
    double nonfinite;
    double sH;
};

// Fold one block partial into a running partial (fixed field rules).
__device__ __forceinline__ void fold_partial(Partial& v, const Partial& p) {
    v.maxRate = fmax(v.maxRate, p.maxRate); v.divergence = fmax(v.divergence, p.divergence);
    v.bH += p.bH; v.bC += p.bC; v.HI += p.HI; v.CI += p.CI;
    v.Hmin = fmin(v.Hmin, p.Hmin); v.Cmin = fmin(v.Cmin, p.Cmin); v.Cmax = fmax(v.Cmax, p.Cmax);
    v.nonfinite = fmax(v.nonfinite, p.nonfinite);
    v.sH += p.sH;
}

// Row slabs of a decomposed mesh: the local arrays hold rows gj0 .. of a
// global mesh of gny rows (gny = 0: the local mesh is the whole mesh).
// Physical-boundary tests and error keys use global rows.
template <class A>
__device__ __forceinline__ int global_ny(const A& a) { return a.gny > 0 ? a.gny : a.ny; }

// Status word: the smallest key wins. The key orders failures as the
// reference's RHS meets them (evolve.cpp:279-384): reconstruction update,
// limiter, porosity sampling, face loop, cell quadrature; then by cell/edge.
enum : int { PART_UPDATE = 0, PART_LIMIT = 1, PART_POROSITY = 2, PART_FACES = 3, PART_CELLS = 4, PART_CHECK = 7 };
__device__ __forceinline__ void record_error(unsigned long long* status, int part, long long where, int code) {
    atomicMin(status, ((unsigned long long)part << 56) | ((unsigned long long)where << 8) | (unsigned long long)(code & 0xff));
}

// Bounds-checked build (MP_CHECKED, libmantlepar_b200_checked.so): every
// cell and edge index a stage element derives is checked against its array
// before use; one outside [0, n) records MP_ERR_ARG_OUTOFRANGE with part
// PART_CHECK and the index in the status word, and the element returns
// without touching memory. In the default build the check compiles away.
#ifdef MP_CHECKED
#define MP_CHECK_INDEX(status, idx, n)                                                        \
    do {                                                                                      \
        const long long mp_i_ = (long long)(idx);                                            \
        if (!(mp_i_ >= 0 && mp_i_ < (long long)(n))) {                                       \
            if (status) record_error((status), PART_CHECK, mp_i_ < 0 ? 0 : mp_i_, MP_ERR_ARG_OUTOFRANGE); \
            return;                                                                           \
        }                                                                                     \
    } while (0)
#else
#define MP_CHECK_INDEX(status, idx, n) \
    do {                               \
    } while (0)
#endif


// ------------------------------------------------------- reconstruction kernel

// Cell flags byte: bit 0 wet (porosity sampling), bit 1 exact diffusion-sample
// check needed (the cheap bound could not prove admissibility).
enum : unsigned char { FLAG_WET = 1, FLAG_CHECK = 2 };

template <class R>
struct ReconArgs {
    int nx, ny;
    Tab<R> tab;
    const double* H;
    const double* C;
    double* rec;           // 18 * ncell, SoA: rec[m*N + cell], m < 9 for H
    unsigned char* flags;
    unsigned long long* status;
    double* theta;         // optional (2 * ncell): limiter factors for H, C
    int gj0 = 0, gny = 0;  // slab: global row of local row 0, global rows
    const int* gate = nullptr;   // device flag: the launch does nothing while it is 0
};

// Max/min of the deviation polynomial over the class's limiter points by
// exact per-point evaluation in FP64, with the finiteness check of every
// value. Used when the coefficients are too large for the fast scan's bound.
__device__ __noinline__ void scan_lines_exact(const StageHot& t, int l0, int l1, const double* D, double& mx,
                                              double& mn, bool& bad) {
    double rmx = D[0], rmn = D[0];
    bad = bad || !isfinite(D[0]);
    for (int l = l0; l < l1; ++l) {
        double a0, a1, a2;
        const bool row = t.line_dir[l] == 0;
        if (row) q2_row(D, t.line_c[l], a0, a1, a2);
        else q2_col(D, t.line_c[l], a0, a1, a2);
        for (int q = 0; q < kNQ; ++q) {
            const double v = quad(a0, a1, a2, row ? t.gx[q] : t.gy[q]);
            rmx = fmax(rmx, v); rmn = fmin(rmn, v);
            bad = bad || !isfinite(v);
        }
    }
    mx = rmx; mn = rmn;
}

// Candidates of one limiter line: its centre p0 = a0 and the larger (p1, p2)
// and smaller (m1, m2) value of each Gauss pair, v(+-s_k) = e_k +- a1 s_k.
template <class R>
__device__ __forceinline__ void line_candidates(const StageHot& t, const Tab<R>& tb, int l, const R* D, R sx1, R sx2,
                                                R sy1, R sy2, R qx1, R qx2, R qy1, R qy2, R& p0, R& p1, R& p2, R& m1,
                                                R& m2) {
    const R c = tb.line_c(l);
    R a0, a1, a2;
    const bool row = t.line_dir[l] == 0;
    if (row) q2_row(D, c, a0, a1, a2);
    else q2_col(D, c, a0, a1, a2);
    const R s1 = row ? sx1 : sy1, s2 = row ? sx2 : sy2;
    const R e1 = fma(a2, row ? qx1 : qy1, a0), e2 = fma(a2, row ? qx2 : qy2, a0);
    const R b = fabs(a1);
    const R d1 = b * s1, d2 = b * s2;
    p0 = a0; p1 = e1 + d1; p2 = e2 + d2; m1 = e1 - d1; m2 = e2 - d2;
}

// Max/min of the deviation polynomial over the class's limiter points. Each
// line holds its centre (s = 0) and the symmetric Gauss pairs s = +-s_k
// (g = 0, +-g1, +-g2), so along a line v(+-s_k) = (a0 + a2 s_k^2) +- a1 s_k
// and the larger of a pair is e_k + |a1| s_k: three candidates per line for
// the maximum and three for the minimum. With every |D_m| below scan_guard
// no value can overflow, so no per-point finiteness test is needed;
// otherwise the exact scan runs.
template <class R>
__device__ __forceinline__ void scan_lines(const StageHot& t, const Tab<R>& tb, int l0, int l1, const double* D,
                                           double& mx, double& mn, bool& bad) {
    bool small = true;
#pragma unroll
    for (int m = 0; m < 9; ++m) small = small && fabs(D[m]) < t.scan_guard;
    if (!small) { scan_lines_exact(t, l0, l1, D, mx, mn, bad); return; }
    const double sx1 = tb.gx(3), sx2 = tb.gx(4), sy1 = tb.gy(3), sy2 = tb.gy(4);
    const double qx1 = sx1 * sx1, qx2 = sx2 * sx2, qy1 = sy1 * sy1, qy2 = sy2 * sy2;
    double rmx = D[0], rmn = D[0];   // cell centre
    for (int l = l0; l < l1; ++l) {
        double p0, p1, p2, m1, m2;
        line_candidates<double>(t, tb, l, D, sx1, sx2, sy1, sy2, qx1, qx2, qy1, qy2, p0, p1, p2, m1, m2);
        rmx = p0 > rmx ? p0 : rmx; rmx = p1 > rmx ? p1 : rmx; rmx = p2 > rmx ? p2 : rmx;
        rmn = p0 < rmn ? p0 : rmn; rmn = m1 < rmn ? m1 : rmn; rmn = m2 < rmn ? m2 : rmn;
    }
    mx = rmx; mn = rmn;
}

// theta of one field: min over points of (bound - mean)/(v - mean) for v
// outside [lo, hi] (state_reconstruction.cpp:216-224). With v = mean + D and
// rounding monotone, the minimum is reached at the extreme D, so one
// division per bound gives the reference's value.
__device__ __forceinline__ double theta_of(double m, double lo, double hi, double dmax, double dmin) {
    double th = 1.0;
    const double vmax = m + dmax, vmin = m + dmin;
    if (vmax > hi) th = fmin(th, (hi - m) / (vmax - m));
    if (vmin < lo) th = fmin(th, (lo - m) / (vmin - m));
    return th < 1.0 ? fmax(0.0, th * (1.0 - 1e-13)) : 1.0;
}

template <class R>
__device__ __forceinline__ void recon_cell(const ReconArgs<R>& a, const Physics& ph, int i, int j) {
    if (i >= a.nx || j >= a.ny) return;
    const StageHot& t = *a.tab.t;
    const int nx = a.nx, ny = a.ny;
    const long long cell = (long long)j * nx + i;
    const size_t N = (size_t)nx * ny;
    MP_CHECK_INDEX(a.status, cell, N);
    const int ci = i == 0 ? 0 : (i == nx - 1 ? 2 : 1);
    const int gj = a.gj0 + j, gny = global_ny(a);
    const int cj = gj == 0 ? 0 : (gj == gny - 1 ? 2 : 1);
    const long long key = cell + (long long)a.gj0 * nx;
    int st_lim = 0;

    double u[3][3];
    double DH[9], DC[9];
    double mH, mC, loH, hiH, loC, hiC;
    int st = 0;
    // Enthalpy, then composition: one 3x3 gather at a time keeps registers low.
#pragma unroll
    for (int f = 0; f < 2; ++f) {
        const double* F = f ? a.C : a.H;
#pragma unroll
        for (int dj = 0; dj < 3; ++dj)
#pragma unroll
            for (int di = 0; di < 3; ++di) {
                const int ii = min(max(i + di - 1, 0), nx - 1), jj = min(max(j + dj - 1, 0), ny - 1);
                MP_CHECK_INDEX(a.status, (long long)jj * nx + ii, N);
                u[dj][di] = __ldg(F + (size_t)jj * nx + ii);
            }
        // 3x3 neighbour bounds (state_reconstruction.cpp:189-196); the clamped
        // gather repeats in-domain values, which leaves min/max unchanged.
        double lo = u[1][1], hi = u[1][1];
#pragma unroll
        for (int dj = 0; dj < 3; ++dj)
#pragma unroll
            for (int di = 0; di < 3; ++di) { lo = fmin(lo, u[dj][di]); hi = fmax(hi, u[dj][di]); }
        if (f == 0) {
            mH = u[1][1]; loH = fmax(0.0, lo); hiH = hi;
            const int s1 = reconstruct(t, ci, cj, u, DH);
            st = st ? st : s1;
        } else {
            mC = u[1][1]; loC = fmax(0.0, lo); hiC = fmin(ph.k.Xe, hi);
            const int s1 = reconstruct(t, ci, cj, u, DC);
            st = st ? st : s1;
        }
    }
    // state_reconstruction.cpp:187-188: admissible means.
    if (!(isfinite(mH) && mH >= 0.0 && isfinite(mC) && mC >= 0.0 && mC <= ph.k.Xe)) st_lim = E_OUTOFRANGE;

    // Limiter over the class's points, evaluated line by line.
    const int cls = cj * 3 + ci;
    const int l0 = t.line_off[cls], l1 = t.line_off[cls + 1];
    double hmx, hmn, cmx, cmn;
    bool bad = false;
    scan_lines<R>(t, a.tab, l0, l1, DH, hmx, hmn, bad);
    scan_lines<R>(t, a.tab, l0, l1, DC, cmx, cmn, bad);
    if (bad) st_lim = st_lim ? st_lim : E_FP;
    const double thH = theta_of(mH, loH, hiH, hmx, hmn);
    const double thC = theta_of(mC, loC, hiC, cmx, cmn);
    if (a.theta) { a.theta[cell] = thH; a.theta[N + cell] = thC; }
    // Diffusion samples (zero diffusivity: kept for their admissibility
    // check). Limited values at limiter points stay in [lo, hi], so the
    // samples are admissible when hi_H is below the liquidus at hi_C and
    // Tep >= 0; otherwise the phase kernel checks each sample exactly.
    // (With a lithostatic pressure the lower Tep over the cell's height bounds it.)
    const double tep = ph.litho ? fmin(tep_at(ph, t.y0 + gj * t.dy), tep_at(ph, t.y0 + (gj + 1) * t.dy)) : ph.Tep;
    const double Hliq = tep + (1.0 - hiC / ph.k.Xe) + ph.k.LD;
    const bool safe = tep >= 0.0 && hiH + 1e-12 * (1.0 + fabs(hiH)) < Hliq;
#pragma unroll
    for (int m = 0; m < 9; ++m) {
        a.rec[(size_t)m * N + cell] = DH[m] * thH;
        a.rec[(size_t)(m + 9) * N + cell] = DC[m] * thC;
    }
    a.flags[cell] = safe ? 0 : FLAG_CHECK;
    if (st) record_error(a.status, PART_UPDATE, key, st);
    if (st_lim) record_error(a.status, PART_LIMIT, key, st_lim);
}

// ---------------------------------------------------------- cell phase kernel

template <class R>
struct CellPhaseArgs {
    int nx, ny;
    Tab<R> tab;
    const double* H;
    const double* C;
    const double* rec;
    unsigned char* flags;
    double* T;
    double* phi;
    unsigned long long* status;
    int gj0 = 0, gny = 0;  // slab: global row of local row 0, global rows
    // Adiabatic source (when Physics::source): vertical solid and Darcy
    // velocities at the cell points [cell*25 + b*5 + a]; per cell the heat
    // sum w/A * source, the rate sum w/A * cooling |v_y| and sum w * source.
    const double* cvs_y = nullptr;
    const double* cud_y = nullptr;
    double* srcH = nullptr;
    double* srcR = nullptr;
    double* srcS = nullptr;
    const int* gate = nullptr;   // device flag: the launch does nothing while it is 0
};

__device__ __forceinline__ void load_rec(const double* rec, size_t N, long long cell, double* DH, double* DC) {
#pragma unroll
    for (int m = 0; m < 9; ++m) {
        DH[m] = __ldg(rec + (size_t)m * N + cell);
        DC[m] = __ldg(rec + (size_t)(m + 9) * N + cell);
    }
}

// Cell quadrature of T and phi (evolve.cpp:359-376) and the wet flag of the
// porosity sampling (initial_flow.cpp:56-67) on the same 5x5 points.
// kExt: the lithostatic pressure and the adiabatic source are compiled in
// (a launch picks the variant; the default path carries none of their code).
template <class R, bool kExt = false>
__device__ __forceinline__ void cellphase_cell(const CellPhaseArgs<R>& a, const Physics& ph, long long cell) {
    const long long N = (long long)a.nx * a.ny;
    if (cell >= N) return;
    MP_CHECK_INDEX(a.status, cell, N);
    const StageHot& t = *a.tab.t;
    const double mH = __ldg(a.H + cell), mC = __ldg(a.C + cell);
    double DH[9], DC[9];
    load_rec(a.rec, (size_t)N, cell, DH, DC);
    int st_por = 0, st_cell = 0, st_face = 0;
    double Tsum = 0.0, Psum = 0.0, Ssum = 0.0, Rsum = 0.0, Wsum = 0.0;
    bool wet = false;
    const int gjc = a.gj0 + (int)(cell / a.nx);
    for (int b = 0; b < kNQ; ++b) {
        double h0, h1, h2, c0, c1, c2;
        const double y = t.gy[b];
        q2_row(DH, y, h0, h1, h2);
        q2_row(DC, y, c0, c1, c2);
        const double tep = (kExt && ph.litho) ? tep_at(ph, height(t, gjc, y)) : ph.Tep;
#pragma unroll
        for (int q = 0; q < kNQ; ++q) {
            const double x = t.gx[q];
            const double h = mH + quad(h0, h1, h2, x);
            const double c = mC + quad(c0, c1, c2, x);
            PhaseLean pl;
            const int s = phase_stage_lean(ph.sk, h, c, tep, pl);
            if (s) { st_por = st_por ? st_por : s; continue; }
            if (!(pl.T >= 0.0 && pl.phil < 1.0)) st_cell = st_cell ? st_cell : E_OUTOFRANGE;
            const double w = t.cw[b * kNQ + q];
            Tsum += w * pl.T;
            Psum += w * pl.phil;
            wet = wet || pl.phil > 0.0;
            if (kExt && ph.source) {
                // evolve.cpp:359-369 with PhaseTransportVelocities at this point's porosity.
                const long long at = cell * (kNQ * kNQ) + b * kNQ + q;
                const double factor = pl.phil == 0.0 ? 0.0 : (ph.theta == 0.0 ? pl.phil : pow(pl.phil, 1.0 + ph.theta));
                const double vy = __ldg(a.cvs_y + at) + factor * __ldg(a.cud_y + at);
                const double src = -ph.cooling * pl.T * vy;
                Ssum += w * src;
                Rsum += w * ph.cooling * fabs(vy);
                Wsum += t.cwp[b * kNQ + q] * src;
            }
        }
    }
    const unsigned char fl = a.flags[cell];
    if (fl & FLAG_CHECK) {
        // Exact admissibility of the limited values at the diffusion samples.
        const int i = (int)(cell % a.nx), j = a.gj0 + (int)(cell / a.nx);
        const int ci = i == 0 ? 0 : (i == a.nx - 1 ? 2 : 1);
        const int cj = j == 0 ? 0 : (j == global_ny(a) - 1 ? 2 : 1);
        const int cls = cj * 3 + ci;
        for (int l = t.line_off[cls]; l < t.line_off[cls + 1]; ++l) {
            if (!t.line_kind[l]) continue;
            double h0, h1, h2, c0, c1, c2;
            const bool row = t.line_dir[l] == 0;
            const double lc = t.line_c[l];
            if (row) { q2_row(DH, lc, h0, h1, h2); q2_row(DC, lc, c0, c1, c2); }
            else { q2_col(DH, lc, h0, h1, h2); q2_col(DC, lc, c0, c1, c2); }
            for (int q = 0; q < kNQ; ++q) {
                const double s_ = row ? t.gx[q] : t.gy[q];
                const double h = mH + quad(h0, h1, h2, s_);
                const double c = mC + quad(c0, c1, c2, s_);
                const double tep = (kExt && ph.litho) ? tep_at(ph, height(t, j, row ? lc : t.gy[q])) : ph.Tep;
                PhaseLean pl;
                const int s = phase_stage_lean(ph.sk, h, c, tep, pl);
                if (s) { st_face = st_face ? st_face : s; continue; }
                if (!(pl.T >= 0.0 && pl.phil < 1.0)) st_face = st_face ? st_face : E_OUTOFRANGE;
            }
        }
    }
    const long long key = cell + (long long)a.gj0 * a.nx;
    if (st_por) record_error(a.status, PART_POROSITY, key, st_por);
    if (st_face) record_error(a.status, PART_FACES, key, st_face);
    if (st_cell) record_error(a.status, PART_CELLS, key, st_cell);
    a.flags[cell] = (unsigned char)((fl & FLAG_CHECK) | (wet ? FLAG_WET : 0));
    a.T[cell] = Tsum;
    a.phi[cell] = Psum;
    if (kExt && ph.source) { a.srcH[cell] = Ssum; a.srcR[cell] = Rsum; a.srcS[cell] = Wsum; }
}

// ---------------------------------------------------------------- face kernel

template <class R>
struct FaceArgs {
    int nx, ny;
    Tab<R> tab;
    const double* H;
    const double* C;
    const double* rec;
    const unsigned char* flags;
    const double* vsn;     // [edge*5 + q], canonical
    const double* udn;
    double* face;          // 4 * nedge SoA: fluxH, fluxC, rate, fluxMixture
    unsigned long long* status;
    int gj0 = 0, gny = 0;  // slab: global row of local row 0, global rows
    const int* gate = nullptr;   // device flag: the launch does nothing while it is 0
};

// Limited H and C of one side along the edge line: v(s) = m + c0 + s*(c1 + s*c2).
struct SideLine {
    double mH, mC;
    double h0, h1, h2, c0, c1, c2;
};

template <class R>
__device__ __forceinline__ void side_line(const FaceArgs<R>& a, size_t N, long long cell, bool row, double fixed,
                                          SideLine& s) {
    double DH[9], DC[9];
    load_rec(a.rec, N, cell, DH, DC);
    s.mH = __ldg(a.H + cell);
    s.mC = __ldg(a.C + cell);
    if (row) { q2_row(DH, fixed, s.h0, s.h1, s.h2); q2_row(DC, fixed, s.c0, s.c1, s.c2); }
    else { q2_col(DH, fixed, s.h0, s.h1, s.h2); q2_col(DC, fixed, s.c0, s.c1, s.c2); }
}

// Limited evaluation + phase + Phase()'s admissibility (evolve.cpp:270-277).
__device__ __forceinline__ int side_phase(const Physics& ph, const SideLine& s, double at, double tep, double& h,
                                          double& c, PhaseLean& pl) {
    h = s.mH + quad(s.h0, s.h1, s.h2, at);
    c = s.mC + quad(s.c0, s.c1, s.c2, at);
    int st = phase_stage(ph.sk, h, c, tep, pl);
    if (!st && !(pl.T >= 0.0 && pl.phil < 1.0)) st = E_OUTOFRANGE;
    return st;
}

// One edge Gauss point of the face fluxes from both sides' phase states:
// edge porosity, transport velocities, Lax-Friedrichs fluxes or the boundary
// policy (evolve.cpp:36-52,292-329; initial_flow.cpp:94-117), and the point's
// CFL rate term before its quadrature weight; st keeps the first failure.
// Used by the general-quad face kernel. face_edge below carries the same
// statements inline: called from there, this function changes the uniform
// face kernel's register allocation (12 more bytes of spills, 2% slower).
struct PointFlux {
    double fh, fc, vn, speed;   // speed: (aC + aH + 2 |vs|) * sens
};
__device__ __forceinline__ PointFlux face_point(const Physics& ph, const PhaseLean& A, const PhaseLean& B, double cL,
                                                double cR, bool wetL, bool wetR, bool boundary, double vs, double ud,
                                                double tep, double LD, int& st) {
    // Edge porosity: harmonic mean of both sides, zero next to a dry cell
    // (initial_flow.cpp:94-117). PhaseTransportVelocities (evolve.cpp:36-52)
    // on normal components: bulk = ephi cl + (1 - ephi) cs, and the
    // composition velocity adds cl/bulk times the Darcy flux. With
    // S = phil_A + phil_B and Q = S bulk, ephi = 2 phil_A phil_B / S and
    // cl/bulk = cl S / Q come from one division 1/(S Q) where it is in range.
    const double cl = 0.5 * (A.cl + B.cl), cs = 0.5 * (A.cs + B.cs);
    const double S = A.phil + B.phil;
    double ephi = 0.0, clb = 0.0;   // clb = cl/bulk where bulk > 0, else 0
    if (wetL && wetR && S > 0.0) {
        const double P2 = 2.0 * A.phil * B.phil;
        const double Q = P2 * (cl - cs) + cs * S;
        const double SQ = S * Q;
        if (SQ > 1e-290 && SQ < 1e290) {
            const double x = 1.0 / SQ;
            ephi = P2 * (Q * x);
            clb = cl * (S * (S * x));
        } else {
            ephi = P2 / S;
            const double bulk = ephi * cl + (1.0 - ephi) * cs;
            clb = bulk > 0.0 ? cl / bulk : 0.0;
        }
    }
    const double factor = ephi == 0.0 ? 0.0 : (ph.theta == 0.0 ? ephi : pow(ephi, 1.0 + ph.theta));
    const double flux = factor * ud;
    const double vn = vs + flux;
    const double ve = vs + clb * flux;
    const double aH = ph.lf_global ? ph.lf_speed : fabs(vn);
    const double aC = ph.lf_global ? ph.lf_speed : fabs(ve);
    if (ph.lf_global && !(aH + 1e-14 >= fabs(vn) && aC + 1e-14 >= fabs(ve))) st = st ? st : E_OUTOFRANGE;
    double fh = 0.5 * (vn * (A.T + B.T) - aH * (B.T - A.T)) - LD * (1.0 - ephi) * vs;
    double fc = 0.5 * (ve * (cL + cR) - aC * (cR - cL));
    if (boundary) {
        // EvaluateAdvectionBoundary (initialization.cpp:469-489) per field.
        const int kh = (ph.Hpol == MP_BC_ZERO_FLUX || vn == 0.0) ? 2 : (vn < 0.0 ? 0 : 1);
        const int kc = (ph.Cpol == MP_BC_ZERO_FLUX || ve == 0.0) ? 2 : (ve < 0.0 ? 0 : 1);
        if ((kh == 0 && ph.Hpol != MP_BC_INFLOW_OUTFLOW) || (kc == 0 && ph.Cpol != MP_BC_INFLOW_OUTFLOW))
            st = st ? st : E_OUTOFRANGE;
        const double inC = kc == 0 ? ph.inflowC : cL;
        double Tb = A.T;
        if (kh == 0) {
            PhaseLean pin;
            const int s3 = phase_stage(ph.sk, ph.inflowH, inC, tep, pin);
            if (s3) st = st ? st : s3;
            Tb = pin.T;
        }
        fh = kh == 2 ? 0.0 : vn * Tb - LD * (1.0 - ephi) * vs;
        fc = kc == 2 ? 0.0 : ve * (kc == 0 ? ph.inflowC : cL);
    }
    const double sens = 1.0 + fmax(fabs(A.dTdC), fabs(B.dTdC));
    if (!isfinite(sens)) st = st ? st : E_FP;
    return PointFlux{fh, fc, vn, (aC + aH + 2.0 * fabs(vs)) * sens};
}

// kExt: the lithostatic pressure is compiled in.
template <class R, bool kExt = false>
__device__ __forceinline__ void face_edge(const FaceArgs<R>& a, const Physics& ph, long long e) {
    const int nx = a.nx, ny = a.ny;
    const long long nI = (long long)nx * (ny + 1);
    const long long nE = nI + (long long)(nx + 1) * ny;
    if (e >= nE) return;
    const StageHot& t = *a.tab.t;
    const size_t N = (size_t)nx * ny;
    bool boundary, reverse, horizontal;
    int erow;                // local row of the edge (horizontal) or of its cells (vertical)
    long long L, Rc = -1;
    double len;
    double lfix, rfix;   // the edge's fixed normalised coordinate in the left / right cell frame
    // Left/right cells and orientation as the reference's Build (evolve.cpp:230-251).
    if (e < nI) {
        horizontal = true;
        const unsigned ue = (unsigned)e;   // edge counts stay below 2^31 (checked on create)
        const int i = (int)(ue % (unsigned)nx), j = (int)(ue / (unsigned)nx);
        const int gj = a.gj0 + j, gny = global_ny(a);
        erow = j;
        boundary = (gj == 0 || gj == gny);
        reverse = (gj == gny);
        L = reverse ? (long long)(j - 1) * nx + i : (long long)j * nx + i;
        if (!boundary) Rc = (long long)(j - 1) * nx + i;
        lfix = reverse ? t.Y : -t.Y;
        rfix = t.Y;
        len = t.len_h;
    } else {
        horizontal = false;
        const unsigned k = (unsigned)(e - nI);
        const int i = (int)(k % (unsigned)(nx + 1)), j = (int)(k / (unsigned)(nx + 1));
        erow = j;
        boundary = (i == 0 || i == nx);
        reverse = (i == 0);
        L = reverse ? (long long)j * nx : (long long)j * nx + (i - 1);
        if (!boundary) Rc = (long long)j * nx + i;
        lfix = reverse ? -t.X : t.X;
        rfix = -t.X;
        len = t.len_v;
    }
    MP_CHECK_INDEX(a.status, L, N);
    if (!boundary) MP_CHECK_INDEX(a.status, Rc, N);
    SideLine sl, sr;
    side_line(a, N, L, horizontal, lfix, sl);
    if (!boundary) side_line(a, N, Rc, horizontal, rfix, sr);
    const bool wetL = (a.flags[L] & FLAG_WET) != 0, wetR = boundary ? true : (a.flags[Rc] & FLAG_WET) != 0;
    const double sgn = reverse ? -1.0 : 1.0;
    const double LD = ph.k.LD;
    double fluxH = 0.0, fluxC = 0.0, fluxMix = 0.0, rate = 0.0;
    int st = 0;
    for (int q = 0; q < kNQ; ++q) {
        const int cq = reverse ? kNQ - 1 - q : q;
        const double at = horizontal ? t.gx[cq] : t.gy[cq];
        const double vs = sgn * __ldg(a.vsn + e * kNQ + cq);
        const double ud = sgn * __ldg(a.udn + e * kNQ + cq);
        double hL, cL, hR, cR;
        PhaseLean A, B;
        // Height of this Gauss point: the edge row for horizontal edges.
        const double tep = !(kExt && ph.litho) ? ph.Tep
                         : tep_at(ph, horizontal ? t.y0 + (a.gj0 + erow) * t.dy : height(t, a.gj0 + erow, at));
        int s = side_phase(ph, sl, at, tep, hL, cL, A);
        if (boundary) { B = A; hR = hL; cR = cL; }
        else {
            const int s2 = side_phase(ph, sr, at, tep, hR, cR, B);
            s = s ? s : s2;
        }
        if (s) { st = st ? st : s; continue; }
        // Edge porosity: harmonic mean of both sides, zero next to a dry cell
        // (initial_flow.cpp:94-117). PhaseTransportVelocities (evolve.cpp:36-52)
        // on normal components: bulk = ephi cl + (1 - ephi) cs, and the
        // composition velocity adds cl/bulk times the Darcy flux. With
        // S = phil_A + phil_B and Q = S bulk, ephi = 2 phil_A phil_B / S and
        // cl/bulk = cl S / Q come from one division 1/(S Q) where it is in range.
        const double cl = 0.5 * (A.cl + B.cl), cs = 0.5 * (A.cs + B.cs);
        const double S = A.phil + B.phil;
        double ephi = 0.0, clb = 0.0;   // clb = cl/bulk where bulk > 0, else 0
        if (wetL && wetR && S > 0.0) {
            const double P2 = 2.0 * A.phil * B.phil;
            const double Q = P2 * (cl - cs) + cs * S;
            const double SQ = S * Q;
            if (SQ > 1e-290 && SQ < 1e290) {
                const double x = 1.0 / SQ;
                ephi = P2 * (Q * x);
                clb = cl * (S * (S * x));
            } else {
                ephi = P2 / S;
                const double bulk = ephi * cl + (1.0 - ephi) * cs;
                clb = bulk > 0.0 ? cl / bulk : 0.0;
            }
        }
        const double factor = ephi == 0.0 ? 0.0 : (ph.theta == 0.0 ? ephi : pow(ephi, 1.0 + ph.theta));
        const double flux = factor * ud;
        const double vn = vs + flux;
        const double ve = vs + clb * flux;
        const double aH = ph.lf_global ? ph.lf_speed : fabs(vn);
        const double aC = ph.lf_global ? ph.lf_speed : fabs(ve);
        if (ph.lf_global && !(aH + 1e-14 >= fabs(vn) && aC + 1e-14 >= fabs(ve))) st = st ? st : E_OUTOFRANGE;
        double fh = 0.5 * (vn * (A.T + B.T) - aH * (B.T - A.T)) - LD * (1.0 - ephi) * vs;
        double fc = 0.5 * (ve * (cL + cR) - aC * (cR - cL));
        if (boundary) {
            // EvaluateAdvectionBoundary (initialization.cpp:469-489) per field.
            const int kh = (ph.Hpol == MP_BC_ZERO_FLUX || vn == 0.0) ? 2 : (vn < 0.0 ? 0 : 1);
            const int kc = (ph.Cpol == MP_BC_ZERO_FLUX || ve == 0.0) ? 2 : (ve < 0.0 ? 0 : 1);
            if ((kh == 0 && ph.Hpol != MP_BC_INFLOW_OUTFLOW) || (kc == 0 && ph.Cpol != MP_BC_INFLOW_OUTFLOW))
                st = st ? st : E_OUTOFRANGE;
            const double inC = kc == 0 ? ph.inflowC : cL;
            double Tb = A.T;
            if (kh == 0) {
                PhaseLean pin;
                const int s3 = phase_stage(ph.sk, ph.inflowH, inC, tep, pin);
                if (s3) st = st ? st : s3;
                Tb = pin.T;
            }
            fh = kh == 2 ? 0.0 : vn * Tb - LD * (1.0 - ephi) * vs;
            fc = kc == 2 ? 0.0 : ve * (kc == 0 ? ph.inflowC : cL);
        }
        const double w = 0.5 * len * t.gw[q];
        fluxH += w * fh;
        fluxC += w * fc;
        fluxMix += w * vn;
        const double sens = 1.0 + fmax(fabs(A.dTdC), fabs(B.dTdC));
        if (!isfinite(sens)) st = st ? st : E_FP;
        rate += w * (aC + aH + 2.0 * fabs(vs)) * sens;
    }
    if (st) record_error(a.status, PART_FACES, L + (long long)a.gj0 * nx, st);
    a.face[e] = fluxH;
    a.face[nE + e] = fluxC;
    a.face[2 * nE + e] = rate;
    a.face[3 * nE + e] = fluxMix;
}

// ------------------------------------------------------------- diffusion

// The diffusive part of one edge's H flux and rate (evolve.cpp:330-347 with
// IntegrateDiffusive(Boundary)FluxWithDerivatives, diffusiveflux.cpp:105-200,
// identity law): temperatures of the limited states at 4 samples per Gauss
// point on the line normal to the edge (2 per side; at a wall 4 inside and the
// wall value), gradient sum_k c_k (T_k - T_last) / ds, flux -= w kappa grad,
// and |d flux / d T_k| added to the rate sample by sample. Added to the face
// results after the advective part, as the reference adds them.
template <class R>
__device__ __forceinline__ void diffusion_edge(const FaceArgs<R>& a, const Physics& ph, long long e) {
    const int nx = a.nx, ny = a.ny;
    const long long nI = (long long)nx * (ny + 1);
    const long long nE = nI + (long long)(nx + 1) * ny;
    if (e >= nE) return;
    const StageHot& t = *a.tab.t;
    const size_t N = (size_t)nx * ny;
    bool boundary, reverse, horizontal;
    long long L, Rc = -1;
    int wall = -1;
    if (e < nI) {
        horizontal = true;
        const unsigned ue = (unsigned)e;
        const int i = (int)(ue % (unsigned)nx), j = (int)(ue / (unsigned)nx);
        const int gj = a.gj0 + j, gny = global_ny(a);
        boundary = (gj == 0 || gj == gny);
        reverse = (gj == gny);
        L = reverse ? (long long)(j - 1) * nx + i : (long long)j * nx + i;
        if (!boundary) Rc = (long long)(j - 1) * nx + i;
        else wall = gj == 0 ? 0 : 1;
    } else {
        horizontal = false;
        const unsigned k = (unsigned)(e - nI);
        const int i = (int)(k % (unsigned)(nx + 1)), j = (int)(k / (unsigned)(nx + 1));
        boundary = (i == 0 || i == nx);
        reverse = (i == 0);
        L = reverse ? (long long)j * nx : (long long)j * nx + (i - 1);
        if (!boundary) Rc = (long long)j * nx + i;
        else wall = i == 0 ? 2 : 3;
    }
    const int type = boundary ? ph.wall_type[wall] : 1;
    if (boundary && type == 0) return;             // zero flux: nothing added
    MP_CHECK_INDEX(a.status, L, N);
    if (!boundary) MP_CHECK_INDEX(a.status, Rc, N);
    const int o = horizontal ? 0 : 1;
    double DL[9], CL[9], DR[9], CR[9];
    double mHL = 0, mCL = 0, mHR = 0, mCR = 0;
    if (type == 1) {
        load_rec(a.rec, N, L, DL, CL);
        mHL = __ldg(a.H + L); mCL = __ldg(a.C + L);
        if (!boundary) {
            load_rec(a.rec, N, Rc, DR, CR);
            mHR = __ldg(a.H + Rc); mCR = __ldg(a.C + Rc);
        }
    }
    double integral = 0.0, rate = a.face[2 * nE + e];
    const double kappa = ph.kappa;
    int st = 0;
    for (int q = 0; q < kNQ; ++q) {
        const double w = t.dif_w[o][q];
        if (boundary && type == 2) { integral += w * ph.wall_value[wall]; continue; }
        const int cq = reverse ? kNQ - 1 - q : q;
        const double at = horizontal ? t.gx[cq] : t.gy[cq];
        const int count = boundary ? 5 : 4;
        double v[5];
        // Temperatures at the samples: limited H, C on the line across the edge
        // through this Gauss point, in the frame of the sample's cell.
        double lh0, lh1, lh2, lc0, lc1, lc2, rh0 = 0, rh1 = 0, rh2 = 0, rc0 = 0, rc1 = 0, rc2 = 0;
        if (horizontal) { q2_col(DL, at, lh0, lh1, lh2); q2_col(CL, at, lc0, lc1, lc2); }
        else { q2_row(DL, at, lh0, lh1, lh2); q2_row(CL, at, lc0, lc1, lc2); }
        if (!boundary) {
            if (horizontal) { q2_col(DR, at, rh0, rh1, rh2); q2_col(CR, at, rc0, rc1, rc2); }
            else { q2_row(DR, at, rh0, rh1, rh2); q2_row(CR, at, rc0, rc1, rc2); }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const bool left = boundary || k < 2;
            const double s = boundary ? t.dif_pos_bnd[wall][k] : t.dif_pos_int[o][k];
            const double h = left ? mHL + quad(lh0, lh1, lh2, s) : mHR + quad(rh0, rh1, rh2, s);
            const double c = left ? mCL + quad(lc0, lc1, lc2, s) : mCR + quad(rc0, rc1, rc2, s);
            const long long cellk = left ? L : Rc;
            const double tep = !ph.litho ? ph.Tep
                             : tep_at(ph, height(t, a.gj0 + (int)(cellk / nx), horizontal ? s : at));
            PhaseLean pl;
            int s1 = phase_stage_lean(ph.sk, h, c, tep, pl);
            if (!s1 && !(pl.T >= 0.0 && pl.phil < 1.0)) s1 = E_OUTOFRANGE;
            if (s1) st = st ? st : s1;
            v[k] = s1 ? 0.0 : pl.T;
        }
        if (boundary) v[4] = ph.wall_value[wall];
        const double* c = boundary ? t.dif_c_bnd : t.dif_c_int;
        const double last = v[count - 1];
        double grad = 0.0, clast = 0.0;
        for (int k = 0; k + 1 < count; ++k) { grad += c[k] * (v[k] - last); clast -= c[k]; }
        const double ds = t.dif_ds[o][boundary ? 1 : 0];
        grad /= ds;
        if (!isfinite(grad)) st = st ? st : E_FP;
        integral -= w * kappa * grad;
        const double scale = -w * kappa / ds;
        for (int k = 0; k < count; ++k) {
            if (boundary && k + 1 == count) continue;     // the wall value: not a sample
            rate += fabs(scale * (k + 1 == count ? clast : c[k]));
        }
    }
    if (st) record_error(a.status, PART_FACES, L + (long long)a.gj0 * nx, st);
    a.face[e] += integral;
    a.face[2 * nE + e] = rate;
}

// ----------------------------------------------------------------- sum kernel

enum SumMode : int { SUM_STORE_L = 0, SUM_RK = 1 };

struct SumArgs {
    int nx, ny;
    double area;           // cell area
    double inv_area;       // 1 / area
    const double* face;
    const double* H;       // stage state
    const double* C;
    const double* H0;      // U^n
    const double* C0;
    double* outH;          // RK: next state; STORE_L: rhs
    double* outC;
    double* rate;          // optional per-cell rate
    int mode;
    double a0, a1, dt;     // next = a0*U^n + a1*(U + dt*L)
    Partial* partial;
    const double* dtp;     // when set, dt is read from device memory (batched instances)
    int gj0 = 0, gny = 0;  // slab: global row of local row 0, global rows
    long long cbeg = 0;    // cells [cbeg, cend) are accumulated (cend < 0: all)
    long long cend = -1;
    // Adiabatic source per cell (cell phase kernel): heat, rate, integral.
    const double* srcH = nullptr;
    const double* srcR = nullptr;
    const double* srcS = nullptr;
    // General quad meshes: the area of every cell (else `area` for all).
    const double* cell_area = nullptr;
    const int* gate = nullptr;   // device flag: the launch does nothing while it is 0
    unsigned long long* status = nullptr;   // status word of the index checks (MP_CHECKED)
};

__device__ __forceinline__ bool gated_off(const int* gate) { return gate && *gate == 0; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Deterministic block reduction of a Partial (fixed shuffle tree per block).
__device__ void block_reduce_write(Partial v, Partial* out) {
    __shared__ double sh[32][11];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double r[11] = {v.maxRate, v.divergence, v.bH, v.bC, v.HI, v.CI, v.Hmin, v.Cmin, v.Cmax, v.nonfinite, v.sH};
    r[0] = warp_max(r[0]); r[1] = warp_max(r[1]);
    r[2] = warp_sum(r[2]); r[3] = warp_sum(r[3]); r[4] = warp_sum(r[4]); r[5] = warp_sum(r[5]);
    r[6] = warp_min(r[6]); r[7] = warp_min(r[7]); r[8] = warp_max(r[8]); r[9] = warp_max(r[9]);
    r[10] = warp_sum(r[10]);
    if (lane == 0)
        for (int k = 0; k < 11; ++k) sh[warp][k] = r[k];
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        const Partial id = partial_identity();
        double s[11] = {id.maxRate, id.divergence, 0, 0, 0, 0, id.Hmin, id.Cmin, id.Cmax, 0, 0};
        if (lane < nw) for (int k = 0; k < 11; ++k) s[k] = sh[lane][k];
        s[0] = warp_max(s[0]); s[1] = warp_max(s[1]);
        s[2] = warp_sum(s[2]); s[3] = warp_sum(s[3]); s[4] = warp_sum(s[4]); s[5] = warp_sum(s[5]);
        s[6] = warp_min(s[6]); s[7] = warp_min(s[7]); s[8] = warp_max(s[8]); s[9] = warp_max(s[9]);
        s[10] = warp_sum(s[10]);
        if (lane == 0) *out = Partial{s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7], s[8], s[9], s[10]};
    }
}

// Per-cell accumulation + RK combination; folds the cell's contribution to
// the stage reductions into v.
// kSrc: the adiabatic source terms are added. kArea: per-cell areas.
template <bool kSrc = false, bool kArea = false>
__device__ __forceinline__ void sum_cell(const SumArgs& a, unsigned cell, Partial& v) {
    const int nx = a.nx, ny = a.ny;
    const long long nI = (long long)nx * (ny + 1);
    const long long nE = nI + (long long)(nx + 1) * ny;
    const int i = (int)(cell % (unsigned)nx), j = (int)(cell / (unsigned)nx);
    MP_CHECK_INDEX(a.status, cell, (long long)nx * ny);
    const double A = kArea ? __ldg(a.cell_area + cell) : a.area, invA = kArea ? 1.0 / A : a.inv_area;
    // Faces of this cell in the reference's id order: bottom, top, left, right,
    // each with the sign of its side (evolve.cpp:350-354).
    const long long eb = (long long)j * nx + i, et = (long long)(j + 1) * nx + i;
    const long long el = nI + (long long)j * (nx + 1) + i, er = el + 1;
    MP_CHECK_INDEX(a.status, et, nI);
    MP_CHECK_INDEX(a.status, er, nE);
    const int gj = a.gj0 + j, gny = global_ny(a);
    const double sb = -1.0, stp = (gj == gny - 1) ? -1.0 : 1.0, sl = (i == 0) ? -1.0 : 1.0, sr = -1.0;
    const long long ids[4] = {eb, et, el, er};
    const double sg[4] = {sb, stp, sl, sr};
    // The reference divides each face term by the area; here the signed sums
    // are scaled once by 1/A (a few ulp apart).
    double rH = 0.0, rC = 0.0, rr = 0.0, dv = 0.0, bH = 0.0, bC = 0.0;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const double FH = __ldg(a.face + ids[f]), FC = __ldg(a.face + nE + ids[f]);
        const double FR = __ldg(a.face + 2 * nE + ids[f]), FM = __ldg(a.face + 3 * nE + ids[f]);
        rH += sg[f] * FH;
        rC += sg[f] * FC;
        rr += FR;
        dv -= sg[f] * FM;
    }
    rH *= invA; rC *= invA; rr *= invA; dv *= invA;
    double sH = 0.0;
    if (kSrc) {
        // The source terms follow the face terms, as the reference adds them.
        rH += __ldg(a.srcH + cell); rr += __ldg(a.srcR + cell); sH = __ldg(a.srcS + cell);
    }
    if (gj == 0) { bH += __ldg(a.face + eb); bC += __ldg(a.face + nE + eb); }
    if (gj == gny - 1) { bH += __ldg(a.face + et); bC += __ldg(a.face + nE + et); }
    if (i == 0) { bH += __ldg(a.face + el); bC += __ldg(a.face + nE + el); }
    if (i == nx - 1) { bH += __ldg(a.face + er); bC += __ldg(a.face + nE + er); }
    double nh, nc;
    if (a.mode == SUM_RK) {
        const double dt_ = a.dtp ? *a.dtp : a.dt;
        const double h = __ldg(a.H + cell), c = __ldg(a.C + cell);
        const double sh_ = __dadd_rn(h, __dmul_rn(dt_, rH));
        const double sc_ = __dadd_rn(c, __dmul_rn(dt_, rC));
        nh = __dadd_rn(__dmul_rn(a.a0, __ldg(a.H0 + cell)), __dmul_rn(a.a1, sh_));
        nc = __dadd_rn(__dmul_rn(a.a0, __ldg(a.C0 + cell)), __dmul_rn(a.a1, sc_));
    } else {
        nh = __ldg(a.H + cell); nc = __ldg(a.C + cell);
    }
    a.outH[cell] = a.mode == SUM_RK ? nh : rH;
    a.outC[cell] = a.mode == SUM_RK ? nc : rC;
    if (a.rate) a.rate[cell] = rr;
    v.maxRate = fmax(v.maxRate, rr);
    v.divergence = fmax(v.divergence, fabs(dv));
    v.bH += bH; v.bC += bC;
    v.HI += nh * A; v.CI += nc * A;
    v.Hmin = fmin(v.Hmin, nh); v.Cmin = fmin(v.Cmin, nc); v.Cmax = fmax(v.Cmax, nc);
    v.nonfinite = fmax(v.nonfinite, (isfinite(nh) && isfinite(nc) && isfinite(rr)) ? 0.0 : 1.0);
    v.sH += sH;
}

// The kSumPer cells of this thread in the sum block starting at first.
// `first` counts from the start of the accumulated range [cbeg, cend).
template <bool kSrc = false, bool kArea = false>
__device__ __forceinline__ Partial sum_cells(const SumArgs& a, long long first) {
    const long long end = a.cend >= 0 ? a.cend : (long long)a.nx * a.ny;
    Partial v = partial_identity();
#pragma unroll
    for (int k = 0; k < kSumPer; ++k) {
        const long long c = a.cbeg + first + k * kRedBlock + threadIdx.x;
        if (c < end) sum_cell<kSrc, kArea>(a, (unsigned)c, v);
    }
    return v;
}

// U1 = U^n + dt*L^n over the kSumPer cells of this thread, with the
// admissibility/integral partials of U1 (cell_area: per-cell areas, or null
// for `area` everywhere).
__device__ __forceinline__ Partial axpy_cells(long long n, const double* H0, const double* C0, const double* LH,
                                              const double* LC, double dt, double area, double* H1, double* C1,
                                              long long first, const double* cell_area = nullptr) {
    Partial v = partial_identity();
#pragma unroll
    for (int q = 0; q < kSumPer; ++q) {
        const long long k = first + q * kRedBlock + threadIdx.x;
        if (k >= n) continue;
        const double h = __dadd_rn(H0[k], __dmul_rn(dt, LH[k]));
        const double c = __dadd_rn(C0[k], __dmul_rn(dt, LC[k]));
        H1[k] = h; C1[k] = c;
        const double A = cell_area ? __ldg(cell_area + k) : area;
        v.HI += h * A; v.CI += c * A;
        v.Hmin = fmin(v.Hmin, h); v.Cmin = fmin(v.Cmin, c); v.Cmax = fmax(v.Cmax, c);
        v.nonfinite = fmax(v.nonfinite, (isfinite(h) && isfinite(c)) ? 0.0 : 1.0);
    }
    return v;
}


}  // namespace
}  // namespace mp

#endif

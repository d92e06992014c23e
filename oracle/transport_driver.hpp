// CPU oracle: the coupled H/C transport stage and time loop.
// TEST INFRASTRUCTURE ONLY -- the checker for the CUDA transport kernels.
//
// Restates, for one rank (no MPI), with the synthetic flow supplier:
//   src/couple/evolve.cpp:36-52     PhaseTransportVelocities
//   src/couple/evolve.cpp:221-268   Build (face table, diffusion sampling)
//   src/couple/evolve.cpp:270-277   Phase (limited evaluation + admissibility)
//   src/couple/evolve.cpp:279-384   RHS (faces, cell quadrature, totals)
//   src/couple/evolve.cpp:386-393   Admissible
//   src/couple/evolve.cpp:428-511   Run (SSPRK2 with CFL retry, balance check)
//   src/couple/state_reconstruction.cpp:101-192  Update, Evaluate, Limit
//   src/couple/initial_flow.cpp:94-117  edge porosity (harmonic mean, dry cells)
//   src/couple/preheat.cpp:65-287   legacy dry preheat (Build, RHS, Run,
//                                   Diagnostics)
// The flow supplier (Stokes-Darcy FEM, re-solved per stage in the reference)
// is replaced by face-normal velocity data: solid velocity and Darcy velocity
// normal components at each edge Gauss point, frozen for the run. The edge
// porosity is recomputed from the current stage exactly as the reference's
// porosity sampling does. Shu-Osher SSPRK3 is added beside SSPRK2.
//
// Backend B supplies the per-cell numerics: B::Recon (update/evaluate of one
// field's reconstruction of one cell), B::phase, and the geometry primitives.
#ifndef MP_ORACLE_TRANSPORT_DRIVER_HPP
#define MP_ORACLE_TRANSPORT_DRIVER_HPP

#include "oracle.h"
#include "restated.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <thread>
#include <limits>
#include <vector>

namespace orc {

// Static-chunked parallel loop over [0, n) on std::threads (the image has no
// OpenMP runtime). Records the first orc::Error by lowest index.
inline int& oracle_threads() { static int t = 0; return t; }
template <class F>
void parallel_for(int n, F&& f) {
    int nt = oracle_threads() > 0 ? oracle_threads() : (int)std::thread::hardware_concurrency();
    nt = std::max(1, std::min(nt, n));
    std::vector<int> codes(nt, 0);
    std::vector<int> where(nt, n);
    auto body = [&](int t) {
        const int lo = (int)((long long)n * t / nt), hi = (int)((long long)n * (t + 1) / nt);
        for (int k = lo; k < hi; ++k) {
            try { f(k); } catch (const Error& e) { codes[t] = e.code; where[t] = k; return; }
        }
    };
    if (nt == 1) body(0);
    else {
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t) pool.emplace_back(body, t);
        body(0);
        for (auto& th : pool) th.join();
    }
    for (int t = 0; t < nt; ++t) if (codes[t]) throw Error{codes[t], "parallel loop failed"};
}

struct Face {
    int left = 0, right = -1;        // cell ids (x fastest); right = -1 on a boundary
    int edge = 0;                    // canonical edge id
    bool boundary = false, reverse = false;
    Pt a, b;                         // oriented vertices (left cell CCW)
    double length = 0;
    Pt normal;
    double area[2] = {0, 0};
    Sampling diffusion;
};

template <class B>
struct Driver {
    orc_material mat{};
    orc_derived der{};
    orc_transport_opts o{};
    B backend;
    int nx = 0, ny = 0, ncell = 0, nIedge = 0, nedge = 0;
    std::vector<Pt> vert;                // (nx+1)*(ny+1)
    std::vector<double> area;            // per cell
    std::vector<double> gp, gw;          // 5-point Gauss rule (edges and cells)
    std::vector<Face> faces;
    std::vector<typename B::Recon> rh, rc;   // per-cell reconstructions of H and C
    std::vector<double> H, C, T, phi, oldH, oldC;
    std::vector<double> lim_h, lim_c;
    std::vector<double> vsn, udn;        // per edge, per canonical q
    std::vector<double> edge_phi;        // per edge, per canonical q
    std::vector<unsigned char> wet;
    std::vector<double> rhsH, rhsC, rate, divg;
    double time = 0;
    int accepted = 0;
    // Time controls (evolve.cpp:449-457,483): end time and the "fixed" control.
    double t_end = INFINITY;
    bool fixed = false;
    // Thermal diffusion (evolve.cpp:330-349): constant diffusivity and one
    // thermal condition per wall (0 bottom y0, 1 top y1, 2 left x0, 3 right x1).
    double kappa = 0;
    ThermalBC wall_bc[4];
    // Phase-law pressure (initialization.cpp:148-163): constant o.pressure, or
    // lithostatic rho*g*l0*(surface_y - y).
    bool lithostatic = false;
    double surface_y = 0;
    double pressure_at(Pt p) const { return lithostatic ? B::static_pressure(mat, der, surface_y - p.y) : o.pressure; }
    // Flow velocities at the cell quadrature points, vertical components
    // [cell*nq*nq + b*nq + a], for the adiabatic source (evolve.cpp:359-369).
    std::vector<double> cell_vs_y, cell_ud_y;
    bool diffusion_active() const {
        if (kappa > 0) return true;
        for (const auto& b : wall_bc) if (b.type == 2) return true;
        return false;
    }
    int wall_of(const Face& f) const {
        if (f.edge < nIedge) return f.edge / nx == 0 ? 0 : 1;
        return (f.edge - nIedge) % (nx + 1) == 0 ? 2 : 3;
    }
    int nq = 5;
    int samples_n = 4;
    double samples_frac = 0.9;

    struct Rates { double boundaryH = 0, boundaryC = 0, sourceH = 0, maximumRate = 0, divergence = 0; };
    Rates current;
    bool have_current = false;

    int cell_id(int i, int j) const { return j * nx + i; }
    Quad corners(int i, int j) const {
        const int M = nx + 1;
        return Quad{{vert[(size_t)j * M + i], vert[(size_t)j * M + i + 1], vert[(size_t)(j + 1) * M + i + 1], vert[(size_t)(j + 1) * M + i]}};
    }

    // mesh.cpp:27-55 (VertexAt: rectangular, perturbed, sine-stretched),
    // integral-based areas as MeshInfo::CacheAreas.
    void build_mesh() {
        const int M = nx + 1, N = ny + 1;
        const double L = o.x1 - o.x0, Hh = o.y1 - o.y0;
        const double hx = L / (double)(M - 1), hy = Hh / (double)(N - 1);
        require(o.mesh_family >= 0 && o.mesh_family <= 2, E_OUTOFRANGE, "Unknown mesh family");
        require(o.mesh_family != 1 || (std::isfinite(o.perturbation) && o.perturbation >= 0 && o.perturbation < 0.25),
                E_OUTOFRANGE, "Perturbation must satisfy 0 <= perturbation < 0.25");
        const double pi = 3.14159265358979323846;
        auto signed_noise = [](uint64_t key) { return 2.0 * unit_noise(key) - 1.0; };
        vert.resize((size_t)M * N);
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < M; ++i) {
                Pt p{o.x0 + (double)i * hx, o.y0 + (double)j * hy};
                if (o.mesh_family == 2) {
                    const double s = (double)i / (M - 1), t = (double)j / (N - 1);
                    p.x = o.x0 + L * std::sin(0.5 * pi * s);
                    p.y = o.y0 + Hh * std::sin(0.5 * pi * t);
                } else if (o.mesh_family == 1 && i > 0 && i < M - 1 && j > 0 && j < N - 1) {
                    const uint64_t index = (uint64_t)j * (uint64_t)M + (uint64_t)i;
                    p.x += o.perturbation * hx * signed_noise(o.seed + 2 * index);
                    p.y += o.perturbation * hy * signed_noise(o.seed + 2 * index + 1);
                }
                if (i == 0) p.x = o.x0;
                if (i == M - 1) p.x = o.x0 + L;
                if (j == 0) p.y = o.y0;
                if (j == N - 1) p.y = o.y0 + Hh;
                vert[(size_t)j * M + i] = p;
            }
        area.resize(ncell);
        std::vector<double> p1, w1;
        B::gauss_rule(1, p1, w1);
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                area[cell_id(i, j)] = B::cell_area(corners(i, j), p1, w1);
    }

    // evolve.cpp:221-268 for one rank: faces in sorted edge-id order.
    void build_faces() {
        faces.clear();
        faces.reserve(nedge);
        for (int id = 0; id < nedge; ++id) {
            Face f;
            f.edge = id;
            int li, lj, ri, rj;
            Pt v0, v1;
            const int M = nx + 1;
            if (id < nIedge) {
                const int i = id % nx, j = id / nx;
                v0 = vert[(size_t)j * M + i]; v1 = vert[(size_t)j * M + i + 1];
                li = i; lj = j; ri = i; rj = j - 1;
            } else {
                const int k = id - nIedge, i = k % M, j = k / M;
                v0 = vert[(size_t)j * M + i]; v1 = vert[(size_t)(j + 1) * M + i];
                li = i - 1; lj = j; ri = i; rj = j;
            }
            const bool hasL = li >= 0 && li < nx && lj >= 0 && lj < ny;
            const bool hasR = ri >= 0 && ri < nx && rj >= 0 && rj < ny;
            f.boundary = !hasL || !hasR;
            f.reverse = !hasL;
            f.left = f.reverse ? cell_id(ri, rj) : cell_id(li, lj);
            if (!f.boundary) f.right = cell_id(ri, rj);
            f.a = v0; f.b = v1;
            if (f.reverse) std::swap(f.a, f.b);
            B::edge_geometry(f.a, f.b, f.length, f.normal);
            f.area[0] = area[f.left];
            const Quad lq = corners(f.left % nx, f.left / nx);
            if (f.boundary) {
                f.area[1] = f.area[0];
                B::sampling(f.a, f.b, lq, nullptr, gp, gw, samples_n, samples_frac, f.diffusion);
            } else {
                f.area[1] = area[f.right];
                const Quad rq = corners(f.right % nx, f.right / nx);
                B::sampling(f.a, f.b, lq, &rq, gp, gw, samples_n, samples_frac, f.diffusion);
            }
            faces.push_back(std::move(f));
        }
    }

    void init(const orc_material& m, const orc_transport_opts& opts) {
        mat = m; o = opts;
        require(B::derive(mat, der), E_OUTOFRANGE, "Invalid material parameters");
        nx = o.nx; ny = o.ny;
        require(nx >= 2 && ny >= 2, E_SIZ, "Transport requires at least 2x2 cells");
        ncell = nx * ny;
        nIedge = nx * (ny + 1);
        nedge = nIedge + (nx + 1) * ny;
        B::gauss_rule(nq, gp, gw);
        build_mesh();
        build_faces();
        backend.setup(*this);
        rh.resize(ncell); rc.resize(ncell);
        // Per-cell reconstruction setup. A backend whose setup touches only
        // the cell's own data (B::kParallelInit) runs it across threads; the
        // restated backend shares a table pool and runs it in cell order.
        auto init_cell = [&](int k) {
            const int i = k % nx, j = k / nx;
            rh[k].init(backend, *this, i, j, std::sqrt(area[k]));
            rc[k] = rh[k];
        };
        if constexpr (B::kParallelInit) {
            parallel_for(ncell, init_cell);
        } else {
            for (int k = 0; k < ncell; ++k) init_cell(k);
        }
        H.assign(ncell, 0); C.assign(ncell, 0); T.assign(ncell, 0); phi.assign(ncell, 0);
        oldH.assign(ncell, 0); oldC.assign(ncell, 0);
        lim_h.assign(ncell, 1); lim_c.assign(ncell, 1);
        vsn.assign((size_t)nedge * nq, 0); udn.assign((size_t)nedge * nq, 0);
        edge_phi.assign((size_t)nedge * nq, 0);
        wet.assign(ncell, 0);
        rhsH.assign(ncell, 0); rhsC.assign(ncell, 0); rate.assign(ncell, 0); divg.assign(ncell, 0);
    }

    // state_reconstruction.cpp:127-134 (limited evaluation)
    void evaluate(int cell, Pt p, double& h, double& c) const {
        h = rh[cell].evaluate(p);
        h = H[cell] + lim_h[cell] * (h - H[cell]);
        c = rc[cell].evaluate(p);
        c = C[cell] + lim_c[cell] * (c - C[cell]);
    }

    // evolve.cpp:270-277
    void phase_at(int cell, Pt p, orc_phase& s, double& h, double& c) const {
        evaluate(cell, p, h, c);
        int code = 0;
        if (!B::phase(mat, der, h, c, pressure_at(p), s, code)) throw Error{E_PHASE + code, "Phase evaluation failed"};
        require(s.TDp >= 0 && s.phil < 1, E_OUTOFRANGE, "Coupled Darcy-Stokes requires nonnegative temperature and porosity < 1");
    }

    // state_reconstruction.cpp:101-120
    void update() {
        std::fill(lim_h.begin(), lim_h.end(), 1.0);
        std::fill(lim_c.begin(), lim_c.end(), 1.0);
        parallel_for(ncell, [&](int k) {
            rh[k].update(H, nx, area[k]);
            rc[k].update(C, nx, area[k]);
        });
    }

    // Limiter point set of one cell (state_reconstruction.cpp:152-168).
    void limiter_points(int i, int j, std::vector<Pt>& pts) const {
        const Quad q = corners(i, j);
        pts.clear();
        pts.push_back(B::map_cell(Pt{0, 0}, q));
        for (double a : gp) for (double b : gp) pts.push_back(B::map_cell(Pt{a, b}, q));
        for (int e = 0; e < 4; ++e) {
            const Pt a = q[e], b = q[(e + 1) % 4];
            for (double r : gp) pts.push_back(B::map_edge(r, a, b));
            int ni = i, nj = j;
            if (e == 0) nj = j - 1; else if (e == 1) ni = i + 1; else if (e == 2) nj = j + 1; else ni = i - 1;
            Sampling s;
            if (ni < 0 || nj < 0 || ni >= nx || nj >= ny) B::sampling(a, b, q, nullptr, gp, gw, samples_n, samples_frac, s);
            else { const Quad other = corners(ni, nj); B::sampling(a, b, q, &other, gp, gw, samples_n, samples_frac, s); }
            for (size_t k = 0; k < s.samples.size(); ++k) if (s.sides[k] == 0) pts.push_back(s.samples[k]);
        }
    }

    // state_reconstruction.cpp:136-192
    void limit() {
        parallel_for(ncell, [&](int k) {
                    thread_local std::vector<Pt> pts;
                    const int i = k % nx, j = k / nx;
                    const double mean[2] = {H[k], C[k]};
                    require(std::isfinite(mean[0]) && mean[0] >= 0 && std::isfinite(mean[1]) && mean[1] >= 0 && mean[1] <= mat.Xe,
                            E_OUTOFRANGE, "Inadmissible cell average in coupled reconstruction");
                    double lo[2] = {mean[0], mean[1]}, hi[2] = {mean[0], mean[1]};
                    for (int y = std::max(0, j - 1); y < std::min(ny, j + 2); ++y)
                        for (int x = std::max(0, i - 1); x < std::min(nx, i + 2); ++x) {
                            const double v[2] = {H[cell_id(x, y)], C[cell_id(x, y)]};
                            for (int z = 0; z < 2; ++z) { lo[z] = std::min(lo[z], v[z]); hi[z] = std::max(hi[z], v[z]); }
                        }
                    lo[0] = std::max(0.0, lo[0]); lo[1] = std::max(0.0, lo[1]);
                    hi[1] = std::min(mat.Xe, hi[1]);
                    limiter_points(i, j, pts);
                    double th[2] = {1, 1};
                    for (const Pt& p : pts) {
                        const double v[2] = {rh[k].evaluate(p), rc[k].evaluate(p)};
                        for (int z = 0; z < 2; ++z) {
                            require(std::isfinite(v[z]), E_FP, "Nonfinite reconstructed state");
                            const double delta = v[z] - mean[z];
                            if (v[z] > hi[z]) th[z] = std::min(th[z], (hi[z] - mean[z]) / delta);
                            if (v[z] < lo[z]) th[z] = std::min(th[z], (lo[z] - mean[z]) / delta);
                        }
                    }
                    lim_h[k] = th[0] < 1 ? std::max(0.0, th[0] * (1 - 1e-13)) : 1;
                    lim_c[k] = th[1] < 1 ? std::max(0.0, th[1] * (1 - 1e-13)) : 1;
        });
    }

    // initial_flow.cpp:46-117 with the reconstruction present: wet cells and
    // the edge porosity per (edge, canonical q); the last writer in cell order wins.
    void sample_porosity() {
        parallel_for(ncell, [&](int k) {
                const int i = k % nx, j = k / nx;
                const Quad q = corners(i, j);
                bool w = false;
                for (double x : gp) for (double y : gp) {
                    const Pt p = B::map_cell(Pt{x, y}, q);
                    double h, c; evaluate(k, p, h, c);
                    orc_phase s; int code = 0;
                    if (!B::phase(mat, der, h, c, pressure_at(p), s, code)) throw Error{E_PHASE + code, "Phase evaluation failed"};
                    w = w || s.phil > 0;
                }
                wet[k] = w;
        });
        // Edge samples: sequential in the reference's cell order so that the
        // last writer of each shared edge is the same as in the reference.
        std::vector<double> val((size_t)ncell * 4 * nq);
        parallel_for(ncell, [&](int k) {
                const int i = k % nx, j = k / nx;
                const Quad q = corners(i, j);
                for (int e = 0; e < 4; ++e) {
                    int ni = i, nj = j;
                    if (e == 0) nj = j - 1; else if (e == 1) ni = i + 1; else if (e == 2) nj = j + 1; else ni = i - 1;
                    const bool bnd = ni < 0 || nj < 0 || ni >= nx || nj >= ny;
                    for (int t = 0; t < nq; ++t) {
                        const Pt p = B::map_edge(gp[t], q[e], q[(e + 1) % 4]);
                        double h, c; evaluate(k, p, h, c);
                        orc_phase s; int code = 0;
                        if (!B::phase(mat, der, h, c, pressure_at(p), s, code)) throw Error{E_PHASE + code, "Phase evaluation failed"};
                        const double a = s.phil;
                        double b = a;
                        if (!bnd) {
                            const int nk = cell_id(ni, nj);
                            evaluate(nk, p, h, c);
                            if (!B::phase(mat, der, h, c, pressure_at(p), s, code)) throw Error{E_PHASE + code, "Phase evaluation failed"};
                            b = s.phil;
                        }
                        double v = (a + b) > 0 ? 2 * a * b / (a + b) : 0;
                        if (!wet[k]) v = 0;
                        if (!bnd && !wet[cell_id(ni, nj)]) v = 0;
                        val[((size_t)k * 4 + e) * nq + t] = v;
                    }
                }
        });
        for (int k = 0; k < ncell; ++k) {
            const int i = k % nx, j = k / nx;
            const int M = nx + 1;
            const int ids[4] = {j * nx + i, nIedge + j * M + i + 1, (j + 1) * nx + i, nIedge + j * M + i};
            const int dir[4] = {1, 1, -1, -1};
            for (int e = 0; e < 4; ++e)
                for (int t = 0; t < nq; ++t) {
                    const int cq = dir[e] == 1 ? t : nq - 1 - t;
                    edge_phi[(size_t)ids[e] * nq + cq] = val[((size_t)k * 4 + e) * nq + t];
                }
        }
    }

    // evolve.cpp:279-384
    Rates rhs() {
        update();
        limit();
        sample_porosity();
        std::fill(rhsH.begin(), rhsH.end(), 0.0);
        std::fill(rhsC.begin(), rhsC.end(), 0.0);
        std::fill(rate.begin(), rate.end(), 0.0);
        std::fill(divg.begin(), divg.end(), 0.0);
        std::fill(T.begin(), T.end(), 0.0);
        std::fill(phi.begin(), phi.end(), 0.0);
        const double LD = der.LD;
        const double theta = o.theta;
        const size_t nf = faces.size();
        std::vector<double> fH(nf), fC(nf), fR(nf), fM(nf);
        parallel_for((int)nf, [&](int fi) {
                const Face& f = faces[fi];
                double fluxH = 0, fluxC = 0, fluxMix = 0, rt = 0;
                for (int q = 0; q < nq; ++q) {
                    const int cq = f.reverse ? nq - 1 - q : q;
                    const double sgn = f.reverse ? -1.0 : 1.0;
                    // Normal components against this face's oriented normal.
                    const double vs = sgn * vsn[(size_t)f.edge * nq + cq];
                    const double ud = sgn * udn[(size_t)f.edge * nq + cq];
                    const double ephi = edge_phi[(size_t)f.edge * nq + cq];
                    const Pt p = B::map_edge(gp[q], f.a, f.b);
                    orc_phase a, b; double hL, cL, hR, cR;
                    phase_at(f.left, p, a, hL, cL);
                    if (f.boundary) { b = a; hR = hL; cR = cL; }
                    else phase_at(f.right, p, b, hR, cR);
                    // evolve.cpp:36-52 on normal components
                    const double cl = .5 * (a.cl + b.cl), cs = .5 * (a.cs + b.cs);
                    const double bulk = ephi * cl + (1 - ephi) * cs;
                    const double factor = ephi == 0 ? 0 : std::pow(ephi, 1 + theta);
                    const double flux = factor * ud;
                    const double vn = vs + flux;
                    const double ve = vs + (bulk > 0 ? cl / bulk * flux : 0);
                    const double aH = o.lf_global ? o.lf_global_speed : std::fabs(vn);
                    const double aC = o.lf_global ? o.lf_global_speed : std::fabs(ve);
                    require(aH + 1e-14 >= std::fabs(vn) && aC + 1e-14 >= std::fabs(ve), E_OUTOFRANGE, "Global LF speed is below the stage flow speed");
                    double fh = .5 * (vn * (a.TDp + b.TDp) - aH * (b.TDp - a.TDp)) - LD * (1 - ephi) * vs;
                    double fc = .5 * (ve * (cL + cR) - aC * (cR - cL));
                    if (f.boundary) {
                        // initialization.cpp:469-489 per field policy
                        auto kind = [&](int policy, double speed) {
                            if (policy == 2 || speed == 0) return 2;          // zero flux
                            if (speed < 0) { require(policy == 0, E_OUTOFRANGE, "Backflow encountered on an outflow-only boundary."); return 0; }
                            return 1;                                         // extrapolated
                        };
                        const int kh = kind(o.H_policy, vn), kc = kind(o.C_policy, ve);
                        const double inflowC = kc == 0 ? o.inflow_C : cL;
                        double Tb = a.TDp;
                        if (kh == 0) {
                            orc_phase s; int code = 0;
                            if (!B::phase(mat, der, o.inflow_H, inflowC, pressure_at(p), s, code)) throw Error{E_PHASE + code, "Phase evaluation failed"};
                            Tb = s.TDp;
                        }
                        fh = kh == 2 ? 0 : vn * Tb - LD * (1 - ephi) * vs;
                        fc = kc == 2 ? 0 : ve * (kc == 0 ? o.inflow_C : cL);
                    }
                    const double weight = .5 * f.length * gw[q];
                    fluxH += weight * fh; fluxC += weight * fc; fluxMix += weight * vn;
                    const double sens = 1 + std::max(std::fabs(a.dTD_dCD), std::fabs(b.dTD_dCD));
                    require(std::isfinite(sens), E_FP, "Singular phase derivative in CFL estimate");
                    rt += weight * (aC + aH + 2 * std::fabs(vs)) * sens;
                }
                // Diffusion samples: temperatures of the limited states
                // (evolve.cpp:332-338), then the normal-line flux (:339-347).
                std::vector<double> Ts(f.diffusion.samples.size(), 0.0);
                for (size_t s = 0; s < f.diffusion.samples.size(); ++s) {
                    const int side = f.diffusion.sides[s];
                    if (side == 2) continue;
                    orc_phase ph; double h, c;
                    phase_at(side == 0 ? f.left : f.right, f.diffusion.samples[s], ph, h, c);
                    Ts[s] = ph.TDp;
                }
                if (diffusion_active()) {
                    double dflux = 0;
                    std::vector<double> deriv;
                    B::diffuse(f.diffusion, Ts, kappa, f.boundary ? &wall_bc[wall_of(f)] : nullptr, dflux, deriv);
                    fluxH += dflux;
                    for (double d : deriv) rt += std::fabs(d);   // evolve.cpp:346
                }
                fH[fi] = fluxH; fC[fi] = fluxC; fR[fi] = rt; fM[fi] = fluxMix;
        });
        Rates out;
        for (size_t fi = 0; fi < nf; ++fi) {
            const Face& f = faces[fi];
            const double fluxH = fH[fi], fluxC = fC[fi];
            rhsH[f.left] += -fluxH / f.area[0];
            rhsC[f.left] += -fluxC / f.area[0];
            rate[f.left] += fR[fi] / f.area[0];
            divg[f.left] += fM[fi] / f.area[0];
            if (!f.boundary) {
                rhsH[f.right] += fluxH / f.area[1];
                rhsC[f.right] += fluxC / f.area[1];
                rate[f.right] += fR[fi] / f.area[1];
                divg[f.right] += -fM[fi] / f.area[1];
            } else {
                out.boundaryH += fluxH; out.boundaryC += fluxC;
            }
        }
        // evolve.cpp:359-376: cell quadrature of T and phi, and the adiabatic
        // source -cooling*T*v_mix,y with v_mix from PhaseTransportVelocities
        // (evolve.cpp:36-52) at the point's porosity; each point's heat and rate
        // are added after the face terms, and sourceH sums w*source in the
        // reference's cell and point order.
        const double cooling = mat.alpha0 * der.l0 * mat.g / mat.cp;
        const bool source = mat.alpha0 != 0;
        require(!source || cell_vs_y.size() == (size_t)ncell * nq * nq, E_WRONGSTATE,
                "The adiabatic source needs the flow velocities at the cell quadrature points");
        std::vector<double> wsrc(source ? (size_t)ncell * nq * nq : 0);
        parallel_for(ncell, [&](int k) {
                const int i = k % nx, j = k / nx;
                const Quad q = corners(i, j);
                double t = 0, ph = 0;
                for (int b = 0; b < nq; ++b)
                    for (int a = 0; a < nq; ++a) {
                        const Pt ref{gp[a], gp[b]};
                        const Pt p = B::map_cell(ref, q);
                        const double w = gw[a] * gw[b] * B::cell_jacobian(ref, q);
                        orc_phase s; double h, c;
                        phase_at(k, p, s, h, c);
                        t += w / area[k] * s.TDp;
                        ph += w / area[k] * s.phil;
                        if (source) {
                            const size_t at = ((size_t)k * nq + b) * nq + a;
                            const double factor = s.phil == 0 ? 0 : std::pow(s.phil, 1 + theta);
                            const double vy = cell_vs_y[at] + factor * cell_ud_y[at];
                            const double src = -cooling * s.TDp * vy;
                            rhsH[k] += w / area[k] * src;
                            rate[k] += w / area[k] * cooling * std::fabs(vy);
                            wsrc[at] = w * src;
                        }
                    }
                T[k] = t; phi[k] = ph;
        });
        for (double v : wsrc) out.sourceH += v;
        double mx = -std::numeric_limits<double>::infinity(), dv = 0;
        for (int k = 0; k < ncell; ++k) { mx = std::max(mx, rate[k]); dv = std::max(dv, std::fabs(divg[k])); }
        out.maximumRate = mx;
        out.divergence = dv;
        require(std::isfinite(out.maximumRate), E_FP, "Nonfinite coupled stage rate");
        return out;
    }

    // evolve.cpp:386-393
    bool admissible() const {
        double hmin = H[0], hmax = H[0], cmin = C[0], cmax = C[0];
        bool fin = true;
        for (int k = 0; k < ncell; ++k) {
            fin = fin && std::isfinite(H[k]) && std::isfinite(C[k]);
            hmin = std::min(hmin, H[k]); hmax = std::max(hmax, H[k]);
            cmin = std::min(cmin, C[k]); cmax = std::max(cmax, C[k]);
        }
        return fin && hmin >= 0 && cmin >= 0 && cmax <= mat.Xe;
    }

    double integral(const std::vector<double>& f) const {
        double s = 0;
        for (int k = 0; k < ncell; ++k) s += f[k] * area[k];
        return s;
    }

    // evolve.cpp:428-511 (SSPRK2) and the Shu-Osher SSPRK3 form of the same loop.
    void step(orc_step_report& rep) {
        if (!have_current) { oldH = H; oldC = C; current = rhs(); have_current = true; }
        const double remaining = t_end - time;
        const double start = time;
        const double oldHI = integral(H), oldCI = integral(C);
        // evolve.cpp:454-457
        double dt = std::min(remaining, fixed ? o.dt_initial : (accepted == 0 ? o.dt_initial : o.dt_max));
        const double limit = current.maximumRate > 0 ? o.cfl / current.maximumRate : o.dt_max;
        require(!fixed || dt <= limit * (1 + 1e-12), E_OUTOFRANGE,
                "Fixed time step exceeds the phase-coupled CFL bound; use control: cfl");
        if (!fixed) dt = std::min(dt, limit);
        const std::vector<double> firstH = rhsH, firstC = rhsC;
        const Rates first = current;
        Rates second, third;
        int retries = 0;
        double courant = 0;
        std::vector<double> U1H, U1C;
        for (;;) {
            require(dt >= std::min(remaining, o.dt_min) && retries < 40, E_NOT_CONVERGED,
                    "Coupled step cannot satisfy admissibility/CFL above minimum step");
            for (int k = 0; k < ncell; ++k) { H[k] = oldH[k] + dt * firstH[k]; C[k] = oldC[k] + dt * firstC[k]; }
            time = start + dt;
            bool valid = admissible();
            if (valid) {
                second = rhs();
                courant = dt * std::max(first.maximumRate, second.maximumRate);
                valid = courant <= o.cfl * (1 + 1e-12);
            }
            if (valid && o.integrator == 3) {
                for (int k = 0; k < ncell; ++k) {
                    H[k] = H[k] + dt * rhsH[k]; C[k] = C[k] + dt * rhsC[k];
                    H[k] = .75 * oldH[k] + .25 * H[k]; C[k] = .75 * oldC[k] + .25 * C[k];
                }
                valid = admissible();
                if (valid) {
                    third = rhs();
                    courant = dt * std::max(std::max(first.maximumRate, second.maximumRate), third.maximumRate);
                    valid = courant <= o.cfl * (1 + 1e-12);
                }
                if (valid) {
                    for (int k = 0; k < ncell; ++k) {
                        H[k] = H[k] + dt * rhsH[k]; C[k] = C[k] + dt * rhsC[k];
                        H[k] = (1.0 / 3.0) * oldH[k] + (2.0 / 3.0) * H[k];
                        C[k] = (1.0 / 3.0) * oldC[k] + (2.0 / 3.0) * C[k];
                    }
                    valid = admissible();
                }
            } else if (valid) {
                for (int k = 0; k < ncell; ++k) {
                    H[k] = H[k] + dt * rhsH[k]; C[k] = C[k] + dt * rhsC[k];
                    H[k] = .5 * oldH[k] + .5 * H[k]; C[k] = .5 * oldC[k] + .5 * C[k];
                }
                valid = admissible();
            }
            if (valid) break;
            require(!fixed, E_OUTOFRANGE, "Fixed coupled step failed stage admissibility/CFL");
            dt *= .5; ++retries;
        }
        const double HI = integral(H), CI = integral(C);
        double bH, bC;
        if (o.integrator == 3) {
            bH = HI - oldHI + dt * ((first.boundaryH + second.boundaryH) / 6 + third.boundaryH * (2.0 / 3.0) -
                                    ((first.sourceH + second.sourceH) / 6 + third.sourceH * (2.0 / 3.0)));
            bC = CI - oldCI + dt * ((first.boundaryC + second.boundaryC) / 6 + third.boundaryC * (2.0 / 3.0));
        } else {
            bH = HI - oldHI + .5 * dt * (first.boundaryH + second.boundaryH - first.sourceH - second.sourceH);
            bC = CI - oldCI + .5 * dt * (first.boundaryC + second.boundaryC);
        }
        require(std::fabs(bH) < 1e-10 * std::max(1.0, std::fabs(oldHI)) && std::fabs(bC) < 1e-10, E_PLIB,
                "Coupled finite-volume conservation balance failed");
        current = rhs();
        ++accepted;
        oldH = H; oldC = C;
        rep.status = 0; rep.retries = retries; rep.dt = dt; rep.time = time; rep.courant = courant;
        rep.boundaryH = o.integrator == 3 ? (first.boundaryH + second.boundaryH) / 6 + third.boundaryH * (2.0 / 3.0) : .5 * (first.boundaryH + second.boundaryH);
        rep.boundaryC = o.integrator == 3 ? (first.boundaryC + second.boundaryC) / 6 + third.boundaryC * (2.0 / 3.0) : .5 * (first.boundaryC + second.boundaryC);
        rep.sourceH = o.integrator == 3 ? (first.sourceH + second.sourceH) / 6 + third.sourceH * (2.0 / 3.0)
                                        : .5 * (first.sourceH + second.sourceH);
        rep.maxRate = current.maximumRate; rep.divergence = current.divergence;
        rep.balanceH = bH; rep.balanceC = bC; rep.H_integral = HI; rep.C_integral = CI;
    }

    // ------------------------------------------------ legacy dry preheat
    // src/couple/preheat.cpp: H_t + div(us H - kappa grad H) = 0 with C fixed
    // and the Stokes velocity frozen (vsn, the solid normal components; ud
    // unused). Forward Euler with the unlimited reconstruction of H, the
    // linear-law Lax-Friedrichs edge flux, and the normal-line diffusion of
    // H on constant cell-average samples. The time controls of
    // set_time_control apply (t_end = time.end) with o.dt_initial/min/max.
    std::vector<double> pre_rate;        // constant per-cell rate (Build)
    double pre_rate_max = 0, pre_limit = 0;
    long long pre_steps = 0;             // steps of this run (Run's counter)
    double pre_integral = 0;             // report.finalIntegral
    bool pre_ready = false;

    // Velocity vectors of a face's points in its oriented order: the normal
    // component along the face normal (the tangential part enters neither
    // the flux nor the rate, and on this mesh v.n reproduces it exactly).
    void face_velocity(const Face& f, std::vector<Pt>& vel) const {
        vel.resize(nq);
        for (int q = 0; q < nq; ++q) {
            const int cq = f.reverse ? nq - 1 - q : q;
            const double vn = (f.reverse ? -1.0 : 1.0) * vsn[(size_t)f.edge * nq + cq];
            vel[q] = Pt{vn * f.normal.x, vn * f.normal.y};
        }
    }

    // preheat.cpp:65-159 (Build): per face the LF speed sum_q L w_q alpha / 2
    // and the diffusion derivatives at zero samples summed per side; each
    // side's cell gets (speed + |derivative|) / area, faces in edge order.
    void preheat_build() {
        const size_t nf = faces.size();
        std::vector<double> r0(nf), r1(nf);
        parallel_for((int)nf, [&](int fi) {
            const Face& f = faces[fi];
            std::vector<Pt> vel;
            face_velocity(f, vel);
            double speed = 0;
            for (int q = 0; q < nq; ++q) {
                const double ns = std::fabs(vel[q].x * f.normal.x + vel[q].y * f.normal.y);
                const double alpha = o.lf_global ? o.lf_global_speed : ns;
                require(alpha + 1e-14 >= ns, E_OUTOFRANGE, "Global LF speed is smaller than the flow normal speed");
                speed += .5 * f.length * gw[q] * alpha;
            }
            const std::vector<double> u(f.diffusion.samples.size(), 0.0);
            double dflux;
            std::vector<double> deriv;
            B::diffuse(f.diffusion, u, kappa, f.boundary ? &wall_bc[wall_of(f)] : nullptr, dflux, deriv);
            double d[2] = {0, 0};
            for (size_t q = 0; q < u.size(); ++q)
                if (f.diffusion.sides[q] != 2) d[f.diffusion.sides[q]] += deriv[q];
            r0[fi] = (speed + std::fabs(d[0])) / f.area[0];
            r1[fi] = (speed + std::fabs(d[1])) / f.area[1];
        });
        pre_rate.assign(ncell, 0.0);
        for (size_t fi = 0; fi < nf; ++fi) {
            pre_rate[faces[fi].left] += r0[fi];
            if (!faces[fi].boundary) pre_rate[faces[fi].right] += r1[fi];
        }
        pre_rate_max = *std::max_element(pre_rate.begin(), pre_rate.end());
        pre_limit = pre_rate_max > 0 ? o.cfl / pre_rate_max : o.dt_max;
    }

    // preheat.cpp:160-200 (RHS): dH/dt of the current H and the outward
    // boundary flux (boundary faces in edge order).
    double preheat_rhs() {
        parallel_for(ncell, [&](int k) { rh[k].update(H, nx, area[k]); });
        std::fill(rhsH.begin(), rhsH.end(), 0.0);
        const size_t nf = faces.size();
        std::vector<double> fl(nf);
        parallel_for((int)nf, [&](int fi) {
            const Face& f = faces[fi];
            std::vector<Pt> vel;
            face_velocity(f, vel);
            std::vector<double> left(nq), right(nq);
            std::vector<AdvectBC> data(nq);
            for (int q = 0; q < nq; ++q) {
                const Pt p = B::map_edge(gp[q], f.a, f.b);
                // StateReconstruction::Enthalpy with the limiter factor 1.
                const double hl = rh[f.left].evaluate(p);
                left[q] = H[f.left] + 1.0 * (hl - H[f.left]);
                if (f.boundary) {
                    // EvaluateAdvectionBoundary (initialization.cpp:469-489).
                    const double speed = vel[q].x * f.normal.x + vel[q].y * f.normal.y;
                    require(std::isfinite(speed), E_OUTOFRANGE, "normal speed must be finite");
                    if (o.H_policy == 2 || speed == 0) data[q].type = 2;
                    else if (speed < 0) {
                        require(o.H_policy == 0, E_OUTOFRANGE, "Backflow encountered on an outflow-only boundary.");
                        data[q].type = 0;
                        data[q].value = o.inflow_H;
                    } else data[q].type = 1;
                } else {
                    const double hr = rh[f.right].evaluate(p);
                    right[q] = H[f.right] + 1.0 * (hr - H[f.right]);
                }
            }
            const double advection = f.boundary ? B::advect_boundary(f.a, f.b, gp, gw, vel, left, data)
                                                : B::advect(f.a, f.b, gp, gw, vel, left, right, o.lf_global != 0, o.lf_global_speed);
            std::vector<double> samples(f.diffusion.samples.size(), 0.0);
            for (size_t q = 0; q < samples.size(); ++q) {
                const int side = f.diffusion.sides[q];
                if (side != 2) samples[q] = H[side == 0 ? f.left : f.right];
            }
            double diffusion;
            std::vector<double> deriv;
            B::diffuse(f.diffusion, samples, kappa, f.boundary ? &wall_bc[wall_of(f)] : nullptr, diffusion, deriv);
            fl[fi] = advection + diffusion;
        });
        double boundary = 0;
        for (size_t fi = 0; fi < nf; ++fi) {
            const Face& f = faces[fi];
            rhsH[f.left] += -fl[fi] / f.area[0];
            if (!f.boundary) rhsH[f.right] += fl[fi] / f.area[1];
            else boundary += fl[fi];
        }
        return boundary;
    }

    // preheat.cpp:235-253: Build, the step limit and the first history row.
    void preheat_begin(orc_preheat_step& first) {
        require(time <= t_end, E_OUTOFRANGE, "State time exceeds time.end");
        require(o.cfl <= 1, E_OUTOFRANGE, "Explicit preheat requires time.step.cfl <= 1");
        preheat_build();
        pre_integral = integral(H);
        pre_steps = 0;
        pre_ready = true;
        first = orc_preheat_step{};
        first.time = time; first.step = accepted; first.integral = pre_integral;
        first.minimum = *std::min_element(H.begin(), H.end());
        first.maximum = *std::max_element(H.begin(), H.end());
    }

    // preheat.cpp:254-282: one forward-Euler step (false at time.end).
    bool preheat_step(long long max_steps, orc_preheat_step& row) {
        if (!(time < t_end)) return false;
        require(pre_steps < max_steps, E_NOT_CONVERGED, "maximum_steps reached before time.end");
        const double remaining = t_end - time;
        double dt = fixed ? o.dt_initial : std::min(o.dt_max, pre_limit);
        if (!fixed && pre_steps == 0) dt = std::min(dt, o.dt_initial);
        dt = std::min(dt, remaining);
        const double roundoff = 8 * std::numeric_limits<double>::epsilon() * std::max({std::fabs(t_end), std::fabs(time), dt});
        if (remaining - dt <= roundoff) dt = remaining;
        require(dt <= pre_limit * (1 + 1e-12), E_OUTOFRANGE, "Requested step exceeds advection/diffusion limit");
        require(dt >= o.dt_min || dt == remaining, E_OUTOFRANGE, "Stable step is below time.step.minimum");
        require(time + dt > time && std::isfinite(dt), E_FP, "Time step does not advance finite time");
        row = orc_preheat_step{};
        row.dt = dt; row.courant = dt * pre_rate_max;
        row.boundaryFlux = preheat_rhs();
        std::vector<double> cand(ncell);
        bool finite = true;
        for (int k = 0; k < ncell; ++k) { cand[k] = H[k] + dt * rhsH[k]; finite = finite && std::isfinite(cand[k]); }
        require(finite, E_FP, "Nonfinite preheat candidate rejected");
        row.integral = integral(cand);
        row.balanceError = row.integral - pre_integral + dt * row.boundaryFlux;
        const double tol = 1e-10 * (1 + std::fabs(row.integral) + std::fabs(pre_integral) + std::fabs(dt * row.boundaryFlux));
        require(std::fabs(row.balanceError) <= tol, E_PLIB, "Preheat heat balance failed; candidate rejected");
        row.minimum = *std::min_element(cand.begin(), cand.end());
        row.maximum = *std::max_element(cand.begin(), cand.end());
        H = cand;
        time = dt == remaining ? t_end : time + dt;
        ++accepted; ++pre_steps;
        row.time = time; row.step = accepted;
        pre_integral = row.integral;
        return true;
    }

    // preheat.cpp:202-233 (Diagnostics): T, phi per cell from the 5x5
    // quadrature of the phase of the unlimited reconstruction of H and C.
    void preheat_diagnostics() {
        update();
        parallel_for(ncell, [&](int k) {
            const int i = k % nx, j = k / nx;
            const Quad q = corners(i, j);
            double t = 0, ph = 0;
            for (int b = 0; b < nq; ++b)
                for (int a = 0; a < nq; ++a) {
                    const Pt ref{gp[a], gp[b]};
                    const Pt p = B::map_cell(ref, q);
                    double h, c;
                    evaluate(k, p, h, c);
                    orc_phase s; int code = 0;
                    if (!B::phase(mat, der, h, c, pressure_at(p), s, code)) throw Error{E_PHASE + code, "Phase evaluation failed"};
                    const double weight = gw[a] * gw[b] * B::cell_jacobian(ref, q) / area[k];
                    t += weight * s.TDp; ph += weight * s.phil;
                }
            T[k] = t; phi[k] = ph;
        });
    }
};


// Handle + C API bodies shared by the restated oracle (orc_*) and the
// reference-backed oracle (ref_*); each library instantiates it once.
template <class B>
struct Handle {
    Driver<B> d;
};

template <class B>
struct Api {
    static void* create(const orc_material* m, const orc_transport_opts* o) {
        oracle_threads() = o->threads;
        Handle<B>* t = new Handle<B>;
        try { t->d.init(*m, *o); } catch (const Error&) { delete t; return nullptr; }
        return t;
    }
    static void destroy(void* h) { delete static_cast<Handle<B>*>(h); }
    static int set_face_velocity(void* h, const double* vs_n, const double* ud_n) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        const size_t n = (size_t)d.nedge * d.nq;
        std::copy(vs_n, vs_n + n, d.vsn.begin());
        std::copy(ud_n, ud_n + n, d.udn.begin());
        d.have_current = false;
        return 0;
    }
    static int set_state(void* h, const double* H, const double* C, double time) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        std::copy(H, H + d.ncell, d.H.begin());
        std::copy(C, C + d.ncell, d.C.begin());
        d.time = time; d.accepted = 0; d.have_current = false; d.pre_ready = false;
        return 0;
    }
    static int get_state(const void* h, double* H, double* C, double* T, double* phi) {
        const auto& d = static_cast<const Handle<B>*>(h)->d;
        if (H) std::copy(d.H.begin(), d.H.end(), H);
        if (C) std::copy(d.C.begin(), d.C.end(), C);
        if (T) std::copy(d.T.begin(), d.T.end(), T);
        if (phi) std::copy(d.phi.begin(), d.phi.end(), phi);
        return 0;
    }
    static int rhs(void* h, double* rhsH, double* rhsC, double* T, double* phi, double* rate, orc_step_report* rep) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        try {
            const auto r = d.rhs();
            // The RHS of the accepted state is what the next step starts from
            // (Driver::step computes exactly this on entry): keep it.
            d.oldH = d.H; d.oldC = d.C; d.current = r; d.have_current = true;
            if (rhsH) std::copy(d.rhsH.begin(), d.rhsH.end(), rhsH);
            if (rhsC) std::copy(d.rhsC.begin(), d.rhsC.end(), rhsC);
            if (T) std::copy(d.T.begin(), d.T.end(), T);
            if (phi) std::copy(d.phi.begin(), d.phi.end(), phi);
            if (rate) std::copy(d.rate.begin(), d.rate.end(), rate);
            if (rep) {
                *rep = orc_step_report{};
                rep->boundaryH = r.boundaryH; rep->boundaryC = r.boundaryC; rep->sourceH = r.sourceH;
                rep->maxRate = r.maximumRate; rep->divergence = r.divergence;
            }
            return 0;
        } catch (const Error& e) { return e.code; }
    }
    static int limiter(void* h, double* thetaH, double* thetaC) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        try {
            d.update(); d.limit();
            std::copy(d.lim_h.begin(), d.lim_h.end(), thetaH);
            std::copy(d.lim_c.begin(), d.lim_c.end(), thetaC);
            return 0;
        } catch (const Error& e) { return e.code; }
    }
    static int set_diffusion(void* h, double kappa, const int* types, const double* values) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        if (!(std::isfinite(kappa) && kappa >= 0)) return E_OUTOFRANGE;
        for (int w = 0; w < 4; ++w) {
            if (types[w] < 0 || types[w] > 2 || !std::isfinite(values[w])) return E_OUTOFRANGE;
            d.wall_bc[w] = ThermalBC{types[w], values[w]};
        }
        d.kappa = kappa;
        d.have_current = false;
        return 0;
    }

    static int set_pressure_model(void* h, int model, double value) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        if ((model != 0 && model != 1) || !std::isfinite(value)) return E_OUTOFRANGE;
        d.lithostatic = model == 1;
        if (model == 1) d.surface_y = value; else d.o.pressure = value;
        d.have_current = false;
        return 0;
    }

    static int set_cell_velocity(void* h, const double* vs_y, const double* ud_y) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        const size_t n = (size_t)d.ncell * d.nq * d.nq;
        d.cell_vs_y.assign(vs_y, vs_y + n);
        d.cell_ud_y.assign(ud_y, ud_y + n);
        d.have_current = false;
        return 0;
    }

    static int vertices(const void* h, double* xy) {
        const auto& d = static_cast<const Handle<B>*>(h)->d;
        for (size_t k = 0; k < d.vert.size(); ++k) { xy[2 * k] = d.vert[k].x; xy[2 * k + 1] = d.vert[k].y; }
        return 0;
    }
    static int set_time_control(void* h, int control, double t_end) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        if (control != 0 && control != 1) return E_OUTOFRANGE;
        d.fixed = control == 1;
        d.t_end = t_end;
        return 0;
    }

    static int preheat_begin(void* h, double* rate, double* limit, orc_preheat_step* first) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        try {
            orc_preheat_step r;
            d.preheat_begin(r);
            if (rate) std::copy(d.pre_rate.begin(), d.pre_rate.end(), rate);
            if (limit) *limit = d.pre_limit;
            if (first) *first = r;
            return 0;
        } catch (const Error& e) { d.pre_ready = false; return e.code; }
    }
    static int preheat_rhs(void* h, double* rhs, double* boundary) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        try {
            const double b = d.preheat_rhs();
            if (rhs) std::copy(d.rhsH.begin(), d.rhsH.end(), rhs);
            if (boundary) *boundary = b;
            return 0;
        } catch (const Error& e) { return e.code; }
    }
    // Up to nsteps steps (fewer at time.end); on failure the last accepted
    // state stays (preheat.h:24-25).
    static int preheat_advance(void* h, long long max_steps, long long nsteps, orc_preheat_step* rows, long long* taken) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        long long n = 0;
        int code = 0;
        if (!d.pre_ready) code = E_WRONGSTATE;
        else {
            try {
                orc_preheat_step r;
                while (n < nsteps && d.preheat_step(max_steps, r)) { if (rows) rows[n] = r; ++n; }
            } catch (const Error& e) { code = e.code; }
        }
        if (taken) *taken = n;
        return code;
    }
    static int preheat_diagnostics(void* h, double* T, double* phi) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        try {
            d.preheat_diagnostics();
            if (T) std::copy(d.T.begin(), d.T.end(), T);
            if (phi) std::copy(d.phi.begin(), d.phi.end(), phi);
            return 0;
        } catch (const Error& e) { return e.code; }
    }

    static int step(void* h, int nsteps, orc_step_report* report) {
        auto& d = static_cast<Handle<B>*>(h)->d;
        for (int s = 0; s < nsteps; ++s) {
            // evolve.cpp:450-451: at the end time (within 32 ulp) the loop stops.
            if (std::isfinite(d.t_end) &&
                d.t_end - d.time <= 32 * std::numeric_limits<double>::epsilon() * std::max(1.0, std::fabs(d.t_end))) {
                d.time = d.t_end;
                if (report)
                    for (int r = s; r < nsteps; ++r) { report[r] = orc_step_report{}; report[r].time = d.time; }
                return 0;
            }
            const double t0 = d.time;
            std::vector<double> h0 = d.H, c0 = d.C;
            try {
                orc_step_report r{};
                d.step(r);
                if (report) report[s] = r;
            } catch (const Error& e) {
                // evolve.cpp:493-499: roll back to the latest accepted state.
                d.time = t0; d.H = h0; d.C = c0; d.have_current = false;
                if (report) { report[s] = orc_step_report{}; report[s].status = e.code; }
                return e.code;
            }
        }
        return 0;
    }
};

}  // namespace orc

#endif

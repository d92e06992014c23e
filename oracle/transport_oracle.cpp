// CPU oracle: restated backend of the transport driver + its C API.
// TEST INFRASTRUCTURE ONLY -- the checker for the CUDA transport kernels.
//
// The per-cell candidate setup restates src/mlweno/reconstruction.cpp:109-210
// with the coupled solver's families (src/couple/state_reconstruction.cpp:64-75,
// h = sqrt(cell area)). With opts.uniform_tables the stencil tables of the
// first cell of each boundary class are shared by all cells of that class
// (exact only up to the rounding of the per-cell vertex coordinates).
#include "oracle.h"

#include <limits>
#include "transport_driver.hpp"

#include <map>
#include <memory>
#include <tuple>

namespace orc_internal {
bool phase_eval(const orc_material& m, const orc_derived& d, double H, double C, double P, orc_phase& s, int& code);
bool derive(const orc_material& m, orc_derived& d);
}

namespace orc {

struct Restated {
    static constexpr bool kParallelInit = false;   // cells share the table pool
    std::vector<CandidateSet> sets;   // per cell
    std::vector<std::unique_ptr<StencilTables>> pool;
    std::map<std::tuple<int, int, int>, const StencilTables*> shared;
    bool uniform = false;

    template <class D>
    void setup(D& d) {
        uniform = d.o.uniform_tables != 0;
        sets.assign(d.ncell, CandidateSet{});
    }

    struct Recon {
        orc::Recon r;
        template <class D>
        void init(Restated& be, D& d, int ti, int tj, double h) {
            CandidateSet& set = be.sets[d.cell_id(ti, tj)];
            const int offs[5][2] = {{-1, -1}, {0, -1}, {0, 0}, {-1, -1}, {-1, 0}};
            for (int k = 0; k < 5; ++k) {
                const bool large = k == 0;
                const int si = large ? 3 : 2, sj = si;
                const int sti = ti + offs[k][0], stj = tj + offs[k][1];
                if (sti < 0 || stj < 0 || si > d.nx || sj > d.ny || sti > d.nx - si || stj > d.ny - sj) continue;
                Candidate c;
                c.si = si; c.sj = sj; c.start_i = sti; c.start_j = stj;
                c.order = large ? 2 : 1;
                c.ti = -offs[k][0]; c.tj = -offs[k][1];
                c.target_smooth = !large;
                std::vector<Quad> corners((size_t)si * sj);
                for (int j = 0; j < sj; ++j)
                    for (int i = 0; i < si; ++i) corners[(size_t)j * si + i] = d.corners(sti + i, stj + j);
                c.poly.place(corners, si, sj, c.order, h);
                const int ci = ti == 0 ? 0 : (ti == d.nx - 1 ? 2 : 1);
                const int cj = tj == 0 ? 0 : (tj == d.ny - 1 ? 2 : 1);
                const auto key = std::make_tuple(ci, cj, k);
                auto it = be.shared.find(key);
                if (be.uniform && it != be.shared.end()) {
                    c.poly.tab = it->second;
                } else {
                    be.pool.emplace_back(new StencilTables);
                    c.poly.build_tables(corners, c.ti, c.tj, c.target_smooth, *be.pool.back());
                    c.poly.tab = be.pool.back().get();
                    if (be.uniform) be.shared[key] = c.poly.tab;
                }
                set.cand.push_back(std::move(c));
            }
            require(!set.cand.empty(), E_WRONG, "No positive-weight candidate remains at this target cell");
            r.set = &set;
        }
        void update(const std::vector<double>& field, int nx, double area) {
            // reconstruction.cpp:299-301: target average from the patch.
            const Candidate& c0 = r.set->cand[0];
            const int ti = c0.start_i + c0.ti, tj = c0.start_j + c0.tj;
            r.target = field[(size_t)tj * nx + ti];
            require(std::isfinite(r.target), E_OUTOFRANGE, "Target cell average must be finite");
            r.update(field.data(), nx, area);
        }
        double evaluate(Pt p) const { return r.evaluate(p); }
    };

    static void gauss_rule(int n, std::vector<double>& p, std::vector<double>& w) { orc::gauss_rule(n, p, w); }
    static double cell_area(const Quad& q, const std::vector<double>& p, const std::vector<double>& w) {
        return integrate_cell(q, p, w, [](Pt) { return 1.0; });
    }
    static void edge_geometry(Pt a, Pt b, double& l, Pt& n) { orc::edge_geometry(a, b, l, n); }
    static Pt map_edge(double r, Pt a, Pt b) { return orc::map_edge(r, a, b); }
    static Pt map_cell(Pt r, const Quad& q) { return orc::map_cell(r, q); }
    static double cell_jacobian(Pt r, const Quad& q) { return orc::cell_jacobian(r, q); }
    static void sampling(Pt a, Pt b, const Quad& l, const Quad* r, const std::vector<double>& p,
                         const std::vector<double>& w, int N, double f, Sampling& s) {
        build_sampling(a, b, l, r, p, w, N, f, s);
    }
    static bool phase(const orc_material& m, const orc_derived& d, double H, double C, double P, orc_phase& s, int& code) {
        return orc_internal::phase_eval(m, d, H, C, P, s, code);
    }
    // EutecticModel::staticPressure(zD) (eutectic_rescaled.cpp:151-161).
    static double static_pressure(const orc_material& m, const orc_derived& d, double zD) {
        require(std::isfinite(zD), E_PHASE + 1, "zD must be finite");
        const lc v = (lc)m.rho * m.g * zD * d.l0;
        require(std::isfinite(v) && std::fabs(v) <= (lc)std::numeric_limits<double>::max(), E_PHASE + 2,
                "static pressure is not representable");
        return (double)v;
    }
    static void diffuse(const Sampling& s, const std::vector<double>& samples, double kappa, const ThermalBC* bc,
                        double& flux, std::vector<double>& deriv) {
        integrate_diffusion(s, samples, kappa, bc, flux, deriv);
    }
    static double advect(Pt a, Pt b, const std::vector<double>& p, const std::vector<double>& w,
                         const std::vector<Pt>& vel, const std::vector<double>& left, const std::vector<double>& right,
                         bool global, double speed) {
        return integrate_advective_flux(a, b, p, w, vel, left, right, global, speed);
    }
    static double advect_boundary(Pt a, Pt b, const std::vector<double>& p, const std::vector<double>& w,
                                  const std::vector<Pt>& vel, const std::vector<double>& interior,
                                  const std::vector<AdvectBC>& data) {
        return integrate_advective_boundary_flux(a, b, p, w, vel, interior, data);
    }
    static bool derive(const orc_material& m, orc_derived& d) { return orc_internal::derive(m, d); }
};

}  // namespace orc

using RestatedApi = orc::Api<orc::Restated>;

extern "C" orc_transport* orc_transport_create(const orc_material* m, const orc_transport_opts* o) {
    return static_cast<orc_transport*>(RestatedApi::create(m, o));
}
extern "C" void orc_transport_destroy(orc_transport* t) { RestatedApi::destroy(t); }
extern "C" int orc_transport_set_face_velocity(orc_transport* t, const double* vs_n, const double* ud_n) {
    return RestatedApi::set_face_velocity(t, vs_n, ud_n);
}
extern "C" int orc_transport_set_state(orc_transport* t, const double* H, const double* C, double time) {
    return RestatedApi::set_state(t, H, C, time);
}
extern "C" int orc_transport_get_state(const orc_transport* t, double* H, double* C, double* T, double* phi) {
    return RestatedApi::get_state(t, H, C, T, phi);
}
extern "C" int orc_transport_rhs(orc_transport* t, double* rhsH, double* rhsC, double* T, double* phi,
                                 double* rate, orc_step_report* rep) {
    return RestatedApi::rhs(t, rhsH, rhsC, T, phi, rate, rep);
}
extern "C" int orc_transport_limiter(orc_transport* t, double* thetaH, double* thetaC) {
    return RestatedApi::limiter(t, thetaH, thetaC);
}
extern "C" int orc_transport_step(orc_transport* t, int nsteps, orc_step_report* report) {
    return RestatedApi::step(t, nsteps, report);
}
extern "C" int orc_transport_set_pressure_model(orc_transport* t, int model, double value) {
    return RestatedApi::set_pressure_model(t, model, value);
}
extern "C" int orc_transport_set_cell_velocity(orc_transport* t, const double* vs_y, const double* ud_y) {
    return RestatedApi::set_cell_velocity(t, vs_y, ud_y);
}
extern "C" int orc_transport_set_diffusion(orc_transport* t, double kappa, const int* types, const double* values) {
    return RestatedApi::set_diffusion(t, kappa, types, values);
}
extern "C" int orc_transport_set_time_control(orc_transport* t, int control, double t_end) {
    return RestatedApi::set_time_control(t, control, t_end);
}

extern "C" int orc_transport_vertices(const orc_transport* t, double* xy) { return RestatedApi::vertices(t, xy); }
extern "C" int orc_preheat_begin(orc_transport* t, double* rate, double* limit, orc_preheat_step* first) {
    return RestatedApi::preheat_begin(t, rate, limit, first);
}
extern "C" int orc_preheat_rhs(orc_transport* t, double* rhs, double* boundary_flux) {
    return RestatedApi::preheat_rhs(t, rhs, boundary_flux);
}
extern "C" int orc_preheat_advance(orc_transport* t, long long max_steps, long long nsteps, orc_preheat_step* rows,
                                   long long* taken) {
    return RestatedApi::preheat_advance(t, max_steps, nsteps, rows, taken);
}
extern "C" int orc_preheat_diagnostics(orc_transport* t, double* T, double* phi) {
    return RestatedApi::preheat_diagnostics(t, T, phi);
}

// Synthetic-input noise: SplitMix64 keyed like src/core/mesh.cpp:40-44
// (seed + 2*index + component), here index = cell id, component = field.
extern "C" double orc_unit_noise(uint64_t seed, uint64_t field, uint64_t cell) {
    return orc::unit_noise(seed + 2 * cell + field);
}

extern "C" int orc_gauss_rule(int n, double* points, double* weights) {
    std::vector<double> p, w;
    orc::gauss_rule(n, p, w);
    std::copy(p.begin(), p.end(), points);
    std::copy(w.begin(), w.end(), weights);
    return 0;
}

// Coupled H/C transport host layer over the C ABI (include/mantle/couple/
// coupled_transport.h): the time loop of the reference's Run
// (src/couple/evolve.cpp:428-511) drives mp_transport_* on the GPU, and
// AdvanceLegacyPreheat (src/couple/preheat.cpp:235-312) drives mp_preheat_*.
#include "mantle/couple/coupled_transport.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <limits>
#include <stdexcept>
#include <string>

#include "mantlepar/mp.h"

namespace mantle::couple {
namespace {

int policy(AdvectionPolicy p) {
    switch (p) {
        case AdvectionPolicy::InflowOutflow: return MP_BC_INFLOW_OUTFLOW;
        case AdvectionPolicy::Outflow: return MP_BC_OUTFLOW;
        default: return MP_BC_ZERO_FLUX;
    }
}

mp_transport_opts options(const Configuration& c, bool continuing) {
    const auto& p = c.phase.parameters();
    mp_transport_opts o{};
    o.material = mp_material{p.Tm0, p.Te0, p.nu, p.L, p.cp, p.Xe, p.rho, p.rhor, p.mus, p.mul, p.k0, p.g, p.alpha0};
    o.pressure = c.pressure;
    o.cfl = c.time.cfl;
    // The first accepted step of a run is capped by initialStep, later ones by
    // maximumStep (evolve.cpp:454); a continued state starts at maximumStep.
    o.dt_initial = (continuing && c.time.control != "fixed") ? c.time.maximumStep : c.time.initialStep;
    o.dt_max = c.time.maximumStep;
    o.dt_min = c.time.minimumStep;
    o.theta = c.darcyExponent;
    o.inflow_H = c.boundary.enthalpy.inflow;
    o.inflow_C = c.boundary.composition.inflow;
    o.H_policy = policy(c.boundary.enthalpy.policy);
    o.C_policy = policy(c.boundary.composition.policy);
    o.integrator = c.integrator == Integrator::SSPRK3 ? MP_SSPRK3 : MP_SSPRK2;
    o.lf_global = c.stabilizer.mode == LaxFriedrichsMode::Global ? 1 : 0;
    o.lf_global_speed = c.stabilizer.globalSpeed;
    o.diffusivity = c.thermalDiffusivity;
    o.precision = c.mixedPrecision ? MP_PRECISION_MIXED : MP_PRECISION_FP64;
    return o;
}

[[noreturn]] void throw_status(mp_status st) {
    const std::string msg = mp_last_error_string();
    if (st == MP_ERR_ARG_OUTOFRANGE || st == MP_ERR_ARG_WRONG || st == MP_ERR_ARG_SIZ) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

int control_of(const TimeInput& t) {
    if (t.control == "fixed") return MP_TIME_FIXED;
    if (t.control == "cfl") return MP_TIME_CFL;
    return -1;
}

mp_transport* create(const Configuration& c, const Mesh& m, bool continuing) {
    const int control = control_of(c.time);
    if (control < 0) throw std::invalid_argument("time.control must be \"fixed\" or \"cfl\"");
    const mp_mesh_desc d{m.nx, m.ny, m.x0, m.x1, m.y0, m.y1};
    const mp_transport_opts o = options(c, continuing);
    mp_transport* h = nullptr;
    if (!m.vertices.empty() && m.vertices.size() != 2 * (size_t)(m.nx + 1) * (m.ny + 1))
        throw std::invalid_argument("Mesh::vertices must hold (nx+1)*(ny+1) (x, y) pairs");
    mp_status st = m.vertices.empty() ? mp_transport_create(&d, &o, nullptr, &h)
                                      : mp_transport_create_quads(&d, m.vertices.data(), &o, nullptr, &h);
    if (st != MP_OK) throw_status(st);
    st = mp_transport_set_time_control(h, control, c.time.end);
    if (st == MP_OK) {
        int type[4];
        double value[4];
        for (int w = 0; w < 4; ++w) {
            const auto& tc = c.boundary.temperature[w];
            type[w] = tc.policy == ThermalPolicy::Temperature ? MP_THERMAL_TEMPERATURE
                    : (tc.policy == ThermalPolicy::OutwardFlux ? MP_THERMAL_FLUX : MP_THERMAL_ZERO_FLUX);
            value[w] = tc.value;
        }
        st = mp_transport_set_thermal_bc(h, type, value);
    }
    if (st == MP_OK && c.pressureModel == PressureModel::Lithostatic)
        st = mp_transport_set_pressure_model(h, MP_PRESSURE_LITHOSTATIC, c.surfaceY);
    if (st != MP_OK) { mp_transport_destroy(h); throw_status(st); }
    return h;
}

}  // namespace

CoupledTransport::CoupledTransport(const Configuration& configuration, const Mesh& mesh)
    : mesh_(mesh), handle_(create(configuration, mesh, false)) {}

CoupledTransport::~CoupledTransport() { mp_transport_destroy(handle_); }

namespace {
mp_status set_velocities(mp_transport* h, const Mesh& m, const EdgeVelocities& v) {
    const size_t n = (size_t)EdgeCount(m) * 5, nc = (size_t)m.nx * m.ny * 25;
    if (v.solid.size() != n || v.darcy.size() != n) return MP_ERR_ARG_SIZ;
    mp_status st = mp_transport_set_face_velocity(h, v.solid.data(), v.darcy.data());
    if (st == MP_OK && !v.cellSolidY.empty()) {
        if (v.cellSolidY.size() != nc || v.cellDarcyY.size() != nc) return MP_ERR_ARG_SIZ;
        st = mp_transport_set_cell_velocity(h, v.cellSolidY.data(), v.cellDarcyY.data());
    }
    return st;
}
}  // namespace

int CoupledTransport::setVelocities(const EdgeVelocities& v) { return set_velocities(handle_, mesh_, v); }

int CoupledTransport::setState(const InitialState& s) {
    const size_t n = (size_t)mesh_.nx * mesh_.ny;
    if (s.enthalpy.size() != n || s.composition.size() != n) return MP_ERR_ARG_SIZ;
    return mp_transport_set_state(handle_, s.enthalpy.data(), s.composition.data(), s.time);
}

int CoupledTransport::getState(InitialState& s) const {
    const size_t n = (size_t)mesh_.nx * mesh_.ny;
    std::vector<double> H(n), C(n), T(n), P(n);
    mp_status st = mp_transport_get_state(handle_, H.data(), C.data(), T.data(), P.data());
    if (st != MP_OK) return st;
    double t = 0;
    int acc = 0;
    st = mp_transport_get_time(handle_, &t, &acc);
    if (st != MP_OK) return st;
    s.mesh = mesh_;
    s.enthalpy.swap(H); s.composition.swap(C); s.temperature.swap(T); s.porosity.swap(P);
    s.time = t;
    s.acceptedSteps = acc;
    return MP_OK;
}

int CoupledTransport::rhs(std::vector<double>& rhsH, std::vector<double>& rhsC, Rates& rates) {
    const size_t n = (size_t)mesh_.nx * mesh_.ny;
    std::vector<double> a(n), b(n);
    mp_stage_totals tot{};
    const mp_status st = mp_transport_rhs(handle_, a.data(), b.data(), nullptr, nullptr, nullptr, &tot);
    if (st != MP_OK) return st;
    rhsH.swap(a); rhsC.swap(b);
    rates = Rates{tot.boundaryH, tot.boundaryC, tot.sourceH, tot.maxRate, tot.divergence};
    return MP_OK;
}

int CoupledTransport::step(int n, std::vector<StepRecord>* history) {
    if (n <= 0) return MP_OK;
    std::vector<mp_step_report> reps((size_t)n);
    int acc0 = 0;
    double t0 = 0;
    mp_transport_get_time(handle_, &t0, &acc0);
    const mp_status st = mp_transport_step(handle_, n, reps.data());
    if (history) {
        long k = acc0;
        for (const auto& r : reps) {
            if (r.status != 0 || !(r.dt > 0)) break;
            StepRecord rec;
            rec.step = ++k; rec.time = r.time; rec.dt = r.dt; rec.courant = r.courant;
            rec.H_integral = r.H_integral; rec.C_integral = r.C_integral;
            rec.outward_H_flux = r.boundaryH; rec.outward_C_flux = r.boundaryC; rec.adiabatic_H_source = r.sourceH;
            rec.H_balance_error = r.balanceH; rec.C_balance_error = r.balanceC;
            rec.mixture_divergence_max = r.divergence; rec.retries = r.retries;
            history->push_back(rec);
        }
    }
    return st;
}

double CoupledTransport::time() const {
    double t = 0;
    mp_transport_get_time(handle_, &t, nullptr);
    return t;
}

long CoupledTransport::acceptedSteps() const {
    int a = 0;
    mp_transport_get_time(handle_, nullptr, &a);
    return a;
}

int RHS(const Configuration& configuration, const InitialState& state, const EdgeVelocities& velocities,
        std::vector<double>& rhsH, std::vector<double>& rhsC, Rates& rates) {
    try {
        CoupledTransport t(configuration, state.mesh);
        int st = t.setVelocities(velocities);
        if (st == MP_OK) st = t.setState(state);
        if (st == MP_OK) st = t.rhs(rhsH, rhsC, rates);
        return st;
    } catch (const std::invalid_argument&) {
        return MP_ERR_ARG_OUTOFRANGE;
    } catch (const std::exception&) {
        return MP_ERR_CUDA;
    }
}

int AdvancePhaseCoupled(const Configuration& c, InitialState& state, const FlowSupplier& flow,
                        std::vector<StepRecord>* history) {
    if (!(c.time.cfl > 0 && c.time.cfl <= 1)) return MP_ERR_ARG_OUTOFRANGE;   // evolve.cpp:431
    mp_transport* h = nullptr;
    try {
        h = create(c, state.mesh, state.acceptedSteps > 0);
    } catch (const std::invalid_argument&) {
        return MP_ERR_ARG_OUTOFRANGE;
    } catch (const std::exception&) {
        return MP_ERR_CUDA;
    }
    const Mesh mesh = state.mesh;
    const size_t ncell = (size_t)mesh.nx * mesh.ny;
    auto finish = [&](int st) {
        mp_transport_destroy(h);
        return st;
    };
    if (state.enthalpy.size() != ncell || state.composition.size() != ncell) return finish(MP_ERR_ARG_SIZ);
    mp_status st = mp_transport_set_state(h, state.enthalpy.data(), state.composition.data(), state.time);
    if (st != MP_OK) return finish(st);
    const long base = state.acceptedSteps;
    const double end = c.time.end;
    EdgeVelocities v;
    InitialState cur;
    auto read_back = [&]() -> mp_status {
        std::vector<double> H(ncell), C(ncell), T(ncell), P(ncell);
        mp_status s2 = mp_transport_get_state(h, H.data(), C.data(), T.data(), P.data());
        if (s2 != MP_OK) return s2;
        double t = 0;
        int acc = 0;
        mp_transport_get_time(h, &t, &acc);
        cur.mesh = mesh;
        cur.enthalpy.swap(H); cur.composition.swap(C); cur.temperature.swap(T); cur.porosity.swap(P);
        cur.time = t;
        cur.acceptedSteps = base + acc;
        return MP_OK;
    };
    for (;;) {
        double t = 0;
        int acc = 0;
        mp_transport_get_time(h, &t, &acc);
        // evolve.cpp:449-452: stop at time.end; the step cap counts all accepted steps.
        if (end - t <= 32 * std::numeric_limits<double>::epsilon() * std::max(1.0, std::fabs(end))) {
            mp_step_report r{};
            mp_transport_step(h, 1, &r);   // snaps the clock to time.end
            break;
        }
        if (base + acc >= c.time.maximumSteps) {
            if (read_back() == MP_OK) state = cur;
            return finish(MP_ERR_NOT_CONVERGED);
        }
        st = read_back();
        if (st != MP_OK) return finish(st);
        const int fs = flow(cur, v);
        if (fs != 0) { state = cur; return finish(fs); }
        st = set_velocities(h, mesh, v);
        if (st != MP_OK) { state = cur; return finish(st); }
        mp_step_report r{};
        st = mp_transport_step(h, 1, &r);
        if (st != MP_OK) {
            if (read_back() == MP_OK) state = cur;   // the last accepted state (rolled back)
            return finish(st);
        }
        if (history && r.dt > 0) {
            StepRecord rec;
            rec.step = base + acc + 1; rec.time = r.time; rec.dt = r.dt; rec.courant = r.courant;
            rec.H_integral = r.H_integral; rec.C_integral = r.C_integral;
            rec.outward_H_flux = r.boundaryH; rec.outward_C_flux = r.boundaryC; rec.adiabatic_H_source = r.sourceH;
            rec.H_balance_error = r.balanceH; rec.C_balance_error = r.balanceC;
            rec.mixture_divergence_max = r.divergence; rec.retries = r.retries;
            history->push_back(rec);
        }
    }
    st = read_back();
    if (st == MP_OK) state = cur;
    return finish(st);
}

int AdvanceLegacyPreheat(const Configuration& c, InitialState& state, const EdgeVelocities& flow,
                         PreheatReport& report) {
    const int control = control_of(c.time);
    if (control < 0) return MP_ERR_ARG_OUTOFRANGE;
    const Mesh mesh = state.mesh;
    if (!mesh.vertices.empty() && mesh.vertices.size() != 2 * (size_t)(mesh.nx + 1) * (mesh.ny + 1))
        return MP_ERR_ARG_SIZ;
    const size_t ncell = (size_t)mesh.nx * mesh.ny;
    if (state.enthalpy.size() != ncell || state.composition.size() != ncell) return MP_ERR_ARG_SIZ;
    if (flow.solid.size() != (size_t)EdgeCount(mesh) * 5) return MP_ERR_ARG_SIZ;
    const auto& p = c.phase.parameters();
    mp_preheat_opts o{};
    o.material = mp_material{p.Tm0, p.Te0, p.nu, p.L, p.cp, p.Xe, p.rho, p.rhor, p.mus, p.mul, p.k0, p.g, p.alpha0};
    o.pressure_model = c.pressureModel == PressureModel::Lithostatic ? MP_PRESSURE_LITHOSTATIC : MP_PRESSURE_CONSTANT;
    o.pressure = c.pressureModel == PressureModel::Lithostatic ? c.surfaceY : c.pressure;
    o.end = c.time.end;
    o.max_steps = c.time.maximumSteps;
    o.control = control;
    o.dt_initial = c.time.initialStep;
    o.dt_min = c.time.minimumStep;
    o.dt_max = c.time.maximumStep;
    o.cfl = c.time.cfl;
    o.diffusivity = c.thermalDiffusivity;
    for (int w = 0; w < 4; ++w) {
        const auto& tc = c.boundary.temperature[w];
        o.thermal_type[w] = tc.policy == ThermalPolicy::Temperature ? MP_THERMAL_TEMPERATURE
                          : (tc.policy == ThermalPolicy::OutwardFlux ? MP_THERMAL_FLUX : MP_THERMAL_ZERO_FLUX);
        o.thermal_value[w] = tc.value;
    }
    o.H_policy = policy(c.boundary.enthalpy.policy);
    o.inflow_H = c.boundary.enthalpy.inflow;
    o.lf_global = c.stabilizer.mode == LaxFriedrichsMode::Global ? 1 : 0;
    o.lf_global_speed = c.stabilizer.globalSpeed;
    const mp_mesh_desc d{mesh.nx, mesh.ny, mesh.x0, mesh.x1, mesh.y0, mesh.y1};
    mp_preheat* h = nullptr;
    mp_status st = mesh.vertices.empty() ? mp_preheat_create(&d, &o, nullptr, &h)
                                         : mp_preheat_create_quads(&d, mesh.vertices.data(), &o, nullptr, &h);
    if (st != MP_OK) return st;
    auto finish = [&](mp_status s) { mp_preheat_destroy(h); return (int)s; };
    st = mp_preheat_set_velocity(h, flow.solid.data());
    if (st == MP_OK)
        st = mp_preheat_set_state(h, state.enthalpy.data(), state.composition.data(), state.time, state.acceptedSteps);
    if (st != MP_OK) return finish(st);
    PreheatReport rep;
    mp_preheat_step first{};
    double limit = 0;
    st = mp_preheat_begin(h, nullptr, &limit, &first);
    if (st != MP_OK) return finish(st);
    auto row = [](const mp_preheat_step& r) {
        PreheatStep out;
        out.step = (long)r.step; out.time = r.time; out.dt = r.dt; out.courant = r.courant;
        out.integral = r.integral; out.minimum = r.minimum; out.maximum = r.maximum;
        out.boundaryFlux = r.boundaryFlux; out.balanceError = r.balanceError;
        return out;
    };
    rep.initialTime = rep.finalTime = state.time;
    rep.stepLimit = limit;
    rep.initialIntegral = rep.finalIntegral = first.integral;
    rep.history.push_back(row(first));
    std::vector<mp_preheat_step> chunk(1024);
    for (;;) {
        long long got = 0;
        st = mp_preheat_advance(h, (long long)chunk.size(), chunk.data(), &got);
        for (long long k = 0; k < got; ++k) {
            rep.history.push_back(row(chunk[k]));
            rep.finalIntegral = chunk[k].integral;
            rep.boundaryIntegral += chunk[k].dt * chunk[k].boundaryFlux;
        }
        if (st != MP_OK || got < (long long)chunk.size()) break;
    }
    // The last accepted H, time and step count, on success and on failure.
    std::vector<double> H(ncell);
    double t = 0;
    long long accepted = 0;
    const mp_status rs = mp_preheat_get_state(h, H.data(), &t, &accepted);
    if (rs != MP_OK) return finish(rs);
    state.enthalpy.swap(H);
    state.time = t;
    state.acceptedSteps = (long)accepted;
    rep.finalTime = t;
    report = std::move(rep);
    if (st != MP_OK) return finish(st);
    std::vector<double> T(ncell), phi(ncell);
    st = mp_preheat_diagnostics(h, T.data(), phi.data());
    if (st != MP_OK) return finish(st);
    state.temperature.swap(T);
    state.porosity.swap(phi);
    return finish(MP_OK);
}

int WritePreheatHistory(const std::string& path, const Configuration& c, const Mesh& mesh,
                        const PreheatReport& report) {
    const std::string tmp = path + ".tmp";
    std::FILE* f = std::fopen(tmp.c_str(), "w");
    if (!f) return MP_ERR_ARG_WRONG;
    const auto& d = c.phase.derived();
    const double area = (mesh.x1 - mesh.x0) * (mesh.y1 - mesh.y0);
    const double year = 365.0 * 24 * 3600;
    std::fprintf(f, "step,time,time_years,dt,dt_s,courant,H_integral,h_mean_J_kg,h_min_J_kg,h_max_J_kg,"
                    "outward_H_flux,balance_error\n");
    for (const auto& r : report.history)
        std::fprintf(f, "%ld,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g\n", r.step, r.time,
                     r.time * d.t0 / year, r.dt, r.dt * d.t0, r.courant, r.integral, r.integral / area * d.h0,
                     r.minimum * d.h0, r.maximum * d.h0, r.boundaryFlux, r.balanceError);
    const bool ok = std::fclose(f) == 0;
    if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) return MP_ERR_ARG_WRONG;
    return MP_OK;
}

}  // namespace mantle::couple

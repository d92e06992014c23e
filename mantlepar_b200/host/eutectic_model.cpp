// mantle::phase::EutecticModel over the mantlepar_b200 C ABI: every
// evaluation runs on the GPU through mp_phase_evaluate_host; the model owns
// one mp_phase_model handle. Interface: include/mantle/phase/eutectic_rescaled.h
// (the reference's src/phase/eutectic_rescaled.h:103-136).
#include "mantle/phase/eutectic_rescaled.h"

#include <ostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "mantlepar/mp.h"

namespace mantle::phase {
namespace {

// Status -> the reference's exception classes (eutectic_rescaled.h:111-113).
void raise_status(mp_status st) {
    if (st == MP_OK) return;
    const std::string msg = mp_last_error_string();
    switch (st) {
        case MP_ERR_PHASE_INVALID:
        case MP_ERR_ARG_WRONG:
        case MP_ERR_ARG_OUTOFRANGE:
        case MP_ERR_ARG_SIZ:
            throw std::invalid_argument(msg);
        case MP_ERR_PHASE_OVERFLOW:
            throw std::overflow_error(msg);
        default:
            throw std::runtime_error(msg);
    }
}

mp_material to_c(const MaterialParameters& p) {
    return mp_material{p.Tm0, p.Te0, p.nu, p.L, p.cp, p.Xe, p.rho, p.rhor, p.mus, p.mul, p.k0, p.g, p.alpha0};
}

DerivedParameters from_c(const mp_derived& d) {
    DerivedParameters r;
    r.dT = d.dT; r.h0 = d.h0; r.gamma = d.gamma; r.LD = d.LD; r.TDm0 = d.TDm0; r.TDe0 = d.TDe0;
    r.invk0 = d.invk0; r.l0 = d.l0; r.u0 = d.u0; r.p0 = d.p0; r.t0 = d.t0;
    return r;
}

mp_phase_model* create(const MaterialParameters& p, DerivedParameters& derived) {
    const mp_material m = to_c(p);
    mp_phase_model* h = nullptr;
    raise_status(mp_phase_create(&m, &h));
    mp_derived d{};
    const mp_status st = mp_phase_get_derived(h, &d);
    if (st != MP_OK) { mp_phase_destroy(h); raise_status(st); }
    derived = from_c(d);
    return h;
}

}  // namespace

EutecticModel::EutecticModel(const MaterialParameters& parameters) {
    handle_ = create(parameters, derived_);
    parameters_ = parameters;
}

EutecticModel::EutecticModel(const EutecticModel& other) {
    handle_ = create(other.parameters_, derived_);
    parameters_ = other.parameters_;
}

EutecticModel& EutecticModel::operator=(const EutecticModel& other) {
    if (this != &other) {
        DerivedParameters d;
        mp_phase_model* h = create(other.parameters_, d);
        mp_phase_destroy(handle_);
        handle_ = h;
        parameters_ = other.parameters_;
        derived_ = d;
    }
    return *this;
}

EutecticModel::EutecticModel(EutecticModel&& other) noexcept
    : parameters_(other.parameters_), derived_(other.derived_), handle_(std::exchange(other.handle_, nullptr)) {}

EutecticModel& EutecticModel::operator=(EutecticModel&& other) noexcept {
    if (this != &other) {
        mp_phase_destroy(handle_);
        handle_ = std::exchange(other.handle_, nullptr);
        parameters_ = other.parameters_;
        derived_ = other.derived_;
    }
    return *this;
}

EutecticModel::~EutecticModel() { mp_phase_destroy(handle_); }

const MaterialParameters& EutecticModel::parameters() const noexcept { return parameters_; }

const DerivedParameters& EutecticModel::derived() const noexcept { return derived_; }

void EutecticModel::setParameters(const MaterialParameters& parameters) {
    const mp_material m = to_c(parameters);
    raise_status(mp_phase_set_params(handle_, &m));   // rejected: model unchanged
    mp_derived d{};
    raise_status(mp_phase_get_derived(handle_, &d));
    parameters_ = parameters;
    derived_ = from_c(d);
}

void EutecticModel::evaluate(const double* HD, const double* CD, const double* P, double P_const, unsigned long n,
                             PhaseState* out) const {
    if (n == 0) return;
    std::vector<double> f(9 * (size_t)n);
    std::vector<int8_t> region(n);
    std::vector<uint8_t> flags(n);
    mp_phase_soa soa{};
    double** dst[9] = {&soa.phi1, &soa.phi2, &soa.phil, &soa.cl, &soa.cs,
                       &soa.TDp, &soa.Tep, &soa.dTD_dCD, &soa.dTD_dHD};
    for (int k = 0; k < 9; ++k) *dst[k] = f.data() + (size_t)k * n;
    soa.region = region.data();
    soa.flags = flags.data();
    long long bad = -1;
    raise_status(mp_phase_evaluate_host(handle_, HD, CD, P, P_const, n, &soa, &bad));
    for (size_t i = 0; i < n; ++i) {
        PhaseState& s = out[i];
        s.phi1 = soa.phi1[i]; s.phi2 = soa.phi2[i]; s.phil = soa.phil[i];
        s.cl = soa.cl[i]; s.cs = soa.cs[i];
        s.region = static_cast<PhaseRegion>(region[i]);
        s.TDp = soa.TDp[i]; s.Tep = soa.Tep[i];
        s.dTD_dCD = soa.dTD_dCD[i]; s.dTD_dHD = soa.dTD_dHD[i];
        s.has_solid = (flags[i] & 1) != 0;
        s.has_liquid = (flags[i] & 2) != 0;
        s.finite_temperature_derivatives = (flags[i] & 4) != 0;
    }
}

PhaseState EutecticModel::evaluate(double HD, double CD, double P) const {
    PhaseState s;
    evaluate(&HD, &CD, &P, 0.0, 1, &s);
    return s;
}

PhaseRegion EutecticModel::classify(double HD, double CD, double P) const {
    int8_t region = 0;
    mp_phase_soa soa{};
    soa.region = &region;
    long long bad = -1;
    // The reference's classify selects the region only (eutectic_rescaled.cpp:187-190):
    // a failure of the evaluation after the selection still has its region.
    const mp_status st = mp_phase_evaluate_host(handle_, &HD, &CD, &P, 0.0, 1, &soa, &bad);
    if (st != MP_OK && !(region != 0 && (st == MP_ERR_PHASE_RUNTIME || st == MP_ERR_PHASE_OVERFLOW)))
        raise_status(st);
    return static_cast<PhaseRegion>(region);
}

PhaseBoundaries EutecticModel::boundaries(double CD, double P) const {
    mp_phase_bounds b{};
    raise_status(mp_phase_boundaries(handle_, CD, P, &b));
    return PhaseBoundaries{b.Tep, b.Tmp, b.H_eutectic_end, b.H_liquidus};
}

double EutecticModel::pressureCorrectedTemperature(double TD, double P) const {
    double v = 0.0;
    raise_status(mp_phase_pressure_corrected_temperature(handle_, TD, P, &v));
    return v;
}

double EutecticModel::staticPressure(double zD) const { return staticPressure(zD, derived_.l0); }

double EutecticModel::staticPressure(double zD, double length_scale) const {
    double v = 0.0;
    raise_status(mp_phase_static_pressure(handle_, zD, length_scale, &v));
    return v;
}

void EutecticModel::printInfo(std::ostream& out) const {
    out << "Dimensionless melting temperature: " << derived_.TDm0 << '\n'
        << "Dimensionless eutectic temperature: " << derived_.TDe0 << '\n'
        << "Dimensionless latent heat: " << derived_.LD << '\n'
        << "Temperature scale [K]: " << derived_.dT << '\n'
        << "Enthalpy scale [J/kg]: " << derived_.h0 << '\n'
        << "Length scale [m]: " << derived_.l0 << '\n'
        << "Velocity scale [m/s]: " << derived_.u0 << '\n'
        << "Pressure scale [Pa]: " << derived_.p0 << '\n'
        << "Time scale [s]: " << derived_.t0 << '\n';
}

}  // namespace mantle::phase

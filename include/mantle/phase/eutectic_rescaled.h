// C++ host layer over the mantlepar_b200 C ABI with the interface of
// mantle::phase::EutecticModel (src/phase/eutectic_rescaled.h:7-139 of the
// reference), so code written against the reference's phase model compiles
// unchanged and evaluates on the GPU.
//
// Kept alike on purpose (a drop-in must be): the namespace, the type and
// member names, the parameter defaults of MaterialParameters, the PhaseRegion
// values, the public member functions and the exception types. Everything
// else is this library's: evaluation runs in the CUDA kernels of
// libmantlepar_b200 (mp_phase_evaluate_host), scales are derived by its host
// code (mp_phase_create), and a model owns one mp_phase_model handle.
//
// Exceptions: std::invalid_argument (invalid or non-finite input),
// std::overflow_error (unrepresentable scales or temperatures),
// std::runtime_error (fractions outside [0, 1], or a CUDA failure).
#ifndef MANTLE_B200_PHASE_EUTECTIC_RESCALED_H
#define MANTLE_B200_PHASE_EUTECTIC_RESCALED_H

#include <iosfwd>

struct mp_phase_model;

namespace mantle::phase {

// Dimensional material inputs (defaults are the reference's).
struct MaterialParameters {
    double Tm0 = 2000.0;    // pure-component melting temperature at P = 0 [K]
    double Te0 = 1480.0;    // eutectic temperature at P = 0 [K]
    double nu = 6.5e6;      // dP/dT [Pa/K]
    double L = 5.0e5;       // latent heat [J/kg]
    double cp = 1200.0;     // specific heat [J/(kg K)]
    double Xe = 0.25;       // eutectic liquid composition, in (0, 1)
    double rho = 3000.0;    // reference density [kg/m^3]
    double rhor = 500.0;    // reference density contrast [kg/m^3]
    double mus = 1.0e19;    // solid viscosity [Pa s]
    double mul = 1.0;       // liquid viscosity [Pa s]
    double k0 = 1.0e-8;     // reference permeability [m^2]
    double g = 10.0;        // gravity [m/s^2]
    double alpha0 = 3.0e-5; // thermal expansion [1/K]
};

// Scales derived from MaterialParameters (recomputed by setParameters).
struct DerivedParameters {
    double dT = 0.0, h0 = 0.0, gamma = 0.0, LD = 0.0, TDm0 = 0.0, TDe0 = 0.0;
    double invk0 = 0.0, l0 = 0.0, u0 = 0.0, p0 = 0.0, t0 = 0.0;
};

enum class PhaseRegion {
    PureSolid = 1,
    TwoSolids = 2,
    Eutectic = 3,
    SolidLiquid = 4,
    Liquid = 5,
    PureMelting = 6
};

struct PhaseBoundaries {
    double Tep = 0.0;
    double Tmp = 0.0;
    double H_eutectic_end = 0.0;
    double H_liquidus = 0.0;
};

struct PhaseState {
    double phi1 = 0.0;
    double phi2 = 0.0;
    double phil = 0.0;
    double cl = 0.0;
    double cs = 0.0;
    PhaseRegion region = PhaseRegion::PureSolid;
    double TDp = 0.0;
    double Tep = 0.0;
    double dTD_dCD = 0.0;
    double dTD_dHD = 0.0;
    bool has_solid = false;
    bool has_liquid = false;
    bool finite_temperature_derivatives = true;
};

// Binary eutectic equilibrium, 0 <= CD <= Xe; TD = T/dT, HD = h/h0, P in Pa.
// A rejected setParameters leaves the model unchanged. evaluate() is const;
// concurrent calls on one model are safe (they are serialised on its
// device staging buffers) as long as no thread calls setParameters.
class EutecticModel {
public:
    explicit EutecticModel(const MaterialParameters& parameters = {});
    EutecticModel(const EutecticModel& other);
    EutecticModel& operator=(const EutecticModel& other);
    EutecticModel(EutecticModel&& other) noexcept;
    EutecticModel& operator=(EutecticModel&& other) noexcept;
    ~EutecticModel();

    const MaterialParameters& parameters() const noexcept;
    const DerivedParameters& derived() const noexcept;
    void setParameters(const MaterialParameters& parameters);

    PhaseState evaluate(double HD, double CD, double P) const;
    PhaseRegion classify(double HD, double CD, double P) const;
    PhaseBoundaries boundaries(double CD, double P) const;

    double pressureCorrectedTemperature(double TD, double P) const;
    double staticPressure(double zD) const;
    double staticPressure(double zD, double length_scale) const;
    void printInfo(std::ostream& out) const;

    // Batched evaluation of n host points (P may be null: P_const applies).
    // Throws on the first failing point like evaluate(); `out` receives n states.
    void evaluate(const double* HD, const double* CD, const double* P, double P_const, unsigned long n,
                  PhaseState* out) const;

    // The underlying C-ABI handle (for mp_phase_evaluate_batch on device arrays).
    const mp_phase_model* handle() const noexcept { return handle_; }

private:
    MaterialParameters parameters_{};
    DerivedParameters derived_{};
    mp_phase_model* handle_ = nullptr;
};

}  // namespace mantle::phase

#endif

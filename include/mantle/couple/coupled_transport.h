// C++ host layer of the coupled H/C transport over the mantlepar_b200 C ABI,
// shaped like mantle::couple::AdvancePhaseCoupled and its stage RHS
// (src/couple/evolve.h:17, evolve.cpp:279-384,428-519 of the reference), and
// of the legacy dry preheat AdvanceLegacyPreheat (src/couple/preheat.h:26).
//
// The reference's Configuration / InitialState carry PETSc, MPI, MFEM and
// YAML types; here they are plain structs holding the subset the transport
// reads, with the reference's member names: phase model, phase-law pressure,
// advection and thermal boundary rules (one per wall), Lax-Friedrichs
// options, thermal diffusivity, time controls (TimeInput), and the cell fields H, C, T,
// phi with time and acceptedSteps. Cell order is j*nx + i; edge data uses the
// reference's edge ids and canonical Gauss-point order (see mantlepar/mp.h).
//
// The flow solve stays outside: a FlowSupplier gives the normal solid and
// Darcy velocities at every edge Gauss point before each step from the
// latest accepted state, and they hold for the step's stages (the reference
// re-solves the flow at every stage). Functions return 0 or an mp_status and
// assign outputs only on success; a failed step leaves the last accepted
// state (evolve.cpp:493-499).
#ifndef MANTLE_B200_COUPLE_COUPLED_TRANSPORT_H
#define MANTLE_B200_COUPLE_COUPLED_TRANSPORT_H

#include <functional>
#include <string>
#include <vector>

#include "mantle/phase/eutectic_rescaled.h"

struct mp_transport;

namespace mantle::couple {

enum class AdvectionPolicy { InflowOutflow, Outflow, ZeroFlux };

// One rule per field for every wall; the inflow value is constant.
struct AdvectionCondition {
    AdvectionPolicy policy = AdvectionPolicy::ZeroFlux;
    double inflow = 0.0;
};
enum class ThermalPolicy { Temperature, OutwardFlux, ZeroFlux };

// value: dimensionless temperature, or physical outward diffusive flux per length.
struct ThermalCondition {
    ThermalPolicy policy = ThermalPolicy::ZeroFlux;
    double value = 0.0;
};

enum Wall { Bottom = 0, Top = 1, Left = 2, Right = 3 };

struct TransportBoundarySpecification {
    AdvectionCondition enthalpy, composition;
    ThermalCondition temperature[4];     // per Wall
};

enum class LaxFriedrichsMode { Local, Global };
struct LaxFriedrichsOptions {
    LaxFriedrichsMode mode = LaxFriedrichsMode::Local;
    double globalSpeed = 0.0;
};

// Time controls (the reference's input TimeInput). control: "fixed" or "cfl".
struct TimeInput {
    double start = 0, end = 1;
    long maximumSteps = 100000;
    std::string control = "fixed";
    double initialStep = 1e-3, minimumStep = 1e-8, maximumStep = 1e-2, cfl = 0.5;
};

enum class Integrator { SSPRK2 = 2, SSPRK3 = 3 };

// Phase-law pressure (the reference's pressure model "constant" or
// "lithostatic"): constant `pressure` Pa, or rho g l0 (surfaceY - y).
enum class PressureModel { Constant, Lithostatic };

struct Configuration {
    phase::EutecticModel phase;
    double pressure = 0.0;               // constant model: phase-law pressure [Pa]
    PressureModel pressureModel = PressureModel::Constant;
    double surfaceY = 0.0;               // lithostatic model: surface height (>= mesh top)
    TransportBoundarySpecification boundary;
    LaxFriedrichsOptions stabilizer;
    double thermalDiffusivity = 0.0;     // kappa >= 0 (normal-line sampled diffusion of T)
    double darcyExponent = 0.0;          // theta of phi^(1+theta) u_d
    TimeInput time;
    Integrator integrator = Integrator::SSPRK2;
    bool mixedPrecision = false;         // FP32 smoothness/weights/limiter scan
};

// The cell grid and domain; `vertices` ((nx+1)*(ny+1) (x, y) pairs, x
// fastest) makes it a general quad mesh such as the reference's
// "perturbed_quadrilateral" family (mp_mesh_vertices builds them); empty =
// the uniform rectangular mesh of the domain.
struct Mesh {
    int nx = 0, ny = 0;
    double x0 = 0, x1 = 1, y0 = 0, y1 = 1;
    std::vector<double> vertices;
};

struct InitialState {
    Mesh mesh;
    std::vector<double> enthalpy, composition, temperature, porosity;
    double time = 0.0;
    long acceptedSteps = 0;
};

// Normal components at [edge*5 + q] against the canonical right normal, and
// (needed when phase.parameters().alpha0 != 0: the adiabatic source) the
// vertical components at the cell quadrature points [cell*25 + b*5 + a].
struct EdgeVelocities {
    std::vector<double> solid, darcy;
    std::vector<double> cellSolidY, cellDarcyY;
};

struct Rates {
    double boundaryH = 0, boundaryC = 0, sourceH = 0, maximumRate = 0, divergence = 0;
};

// One accepted step, the columns of evolution_history.csv that the transport
// determines (evolve.cpp:443,502-506).
struct StepRecord {
    long step = 0;
    double time = 0, dt = 0, courant = 0, H_integral = 0, C_integral = 0;
    double outward_H_flux = 0, outward_C_flux = 0, adiabatic_H_source = 0;
    double H_balance_error = 0, C_balance_error = 0, mixture_divergence_max = 0;
    int retries = 0;
};

using FlowSupplier = std::function<int(const InitialState&, EdgeVelocities&)>;

// Persistent GPU instance: mesh tables, device state and buffers stay resident.
class CoupledTransport {
public:
    CoupledTransport(const Configuration& configuration, const Mesh& mesh);
    ~CoupledTransport();
    CoupledTransport(const CoupledTransport&) = delete;
    CoupledTransport& operator=(const CoupledTransport&) = delete;

    int setVelocities(const EdgeVelocities& velocities);
    int setState(const InitialState& state);
    // Cell fields, time and acceptedSteps of the latest accepted state.
    int getState(InitialState& state) const;
    int rhs(std::vector<double>& rhsH, std::vector<double>& rhsC, Rates& rates);
    // Up to n accepted steps, stopping at time.end; appends to history if given.
    int step(int n, std::vector<StepRecord>* history = nullptr);
    double time() const;
    long acceptedSteps() const;
    mp_transport* handle() const noexcept { return handle_; }

private:
    Mesh mesh_;
    mp_transport* handle_ = nullptr;
};

// The stage RHS at `state` with `velocities`: dH/dt, dC/dt per cell and the
// stage rates; temperature and porosity of `state` are not read.
int RHS(const Configuration& configuration, const InitialState& state, const EdgeVelocities& velocities,
        std::vector<double>& rhsH, std::vector<double>& rhsC, Rates& rates);

// Advance `state` from state.time to configuration.time.end (at most
// time.maximumSteps accepted steps in total), asking `flow` for the edge
// velocities before every step. On return, state holds the latest accepted
// H, C, T, phi, time and acceptedSteps.
int AdvancePhaseCoupled(const Configuration& configuration, InitialState& state, const FlowSupplier& flow,
                        std::vector<StepRecord>* history = nullptr);

// Legacy dry preheat (src/couple/preheat.h:6-31): one row per accepted step
// (and the initial state first), and the run's report.
struct PreheatStep {
    long step = 0;
    double time = 0, dt = 0, courant = 0;
    double integral = 0, minimum = 0, maximum = 0;
    double boundaryFlux = 0, balanceError = 0;
};
struct PreheatReport {
    double initialTime = 0, finalTime = 0, stepLimit = 0;
    double initialIntegral = 0, finalIntegral = 0, boundaryIntegral = 0;
    std::vector<PreheatStep> history;
};

// AdvanceLegacyPreheat (preheat.cpp:235-287): H_t + div(us H - kappa grad H)
// = 0 with C fixed and `flow.solid` the frozen Stokes velocity (normal
// components at the edge Gauss points; the Darcy part is unused, the flow
// is dry). Forward Euler from state.time to configuration.time.end with the
// time controls, thermalDiffusivity, the per-wall thermal conditions, the
// enthalpy advection rule and the stabilizer of `configuration`; the phase
// model and pressure give the final T and phi (Diagnostics). state.mesh may
// be a general quad mesh (Mesh::vertices). Returns 0 or an mp_status; on
// failure H, time and acceptedSteps hold the last accepted step and the
// phase fields are not refreshed.
int AdvanceLegacyPreheat(const Configuration& configuration, InitialState& state, const EdgeVelocities& flow,
                         PreheatReport& report);

// preheat_history.csv (WritePreheatHistory, preheat.cpp:289-312) at `path`.
int WritePreheatHistory(const std::string& path, const Configuration& configuration, const Mesh& mesh,
                        const PreheatReport& report);

// Number of edges of a mesh (AlongI edges first, then AlongJ).
inline long EdgeCount(const Mesh& m) { return (long)m.nx * (m.ny + 1) + (long)(m.nx + 1) * m.ny; }

}  // namespace mantle::couple

#endif

/*
 * CPU oracle for the MantlePar ML-WENO H/C transport + eutectic phase path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA path
 * is compared against; it is never linked into, loaded by or called from the
 * product library (mantlepar_b200/). Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / --impl reference legs may use it.
 *
 * It restates, in plain C++, the reference algorithm of
 *   src/phase/eutectic_rescaled.cpp           (EutecticModel)
 *   src/mlweno/tensorstencilpoly.cpp          (TensorStencilPoly)
 *   src/mlweno/reconstruction.cpp             (Reconstruction)
 *   src/couple/state_reconstruction.cpp       (StateReconstruction + limiter)
 *   src/couple/evolve.cpp                     (RHS, Admissible, SSPRK2 loop)
 *   src/couple/initial_flow.cpp               (edge porosity sampling)
 *   src/mlweno/diffusiveflux.cpp              (normal-line sample geometry)
 *   src/mlweno/advectiveflux.cpp              (Lax-Friedrichs edge fluxes)
 *   src/couple/preheat.cpp                    (legacy dry preheat)
 *   src/core/integral.cpp, src/core/mesh.cpp  (geometry, SplitMix64 noise)
 * keeping the reference's long double internals, so that it can be pinned
 * against the reference compiled from its own sources (oracle/_ref).
 */
#ifndef MP_ORACLE_H
#define MP_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors src/phase/eutectic_rescaled.h:10-26 (MaterialParameters). */
typedef struct orc_material {
    double Tm0, Te0, nu, L, cp, Xe, rho, rhor, mus, mul, k0, g, alpha0;
} orc_material;

/* Mirrors src/phase/eutectic_rescaled.h:29-41 (DerivedParameters). */
typedef struct orc_derived {
    double dT, h0, gamma, LD, TDm0, TDe0, invk0, l0, u0, p0, t0;
} orc_derived;

/* Mirrors src/phase/eutectic_rescaled.h:52-57 (PhaseBoundaries). */
typedef struct orc_bounds {
    double Tep, Tmp, H_eutectic_end, H_liquidus;
} orc_bounds;

/* Mirrors src/phase/eutectic_rescaled.h:59-76 (PhaseState). */
typedef struct orc_phase {
    double phi1, phi2, phil, cl, cs;
    int region;
    double TDp, Tep, dTD_dCD, dTD_dHD;
    int has_solid, has_liquid, finite_temperature_derivatives;
} orc_phase;

/* Error classes: 0 ok, 1 std::invalid_argument, 2 std::overflow_error,
 * 3 std::runtime_error (src/phase/eutectic_rescaled.h:111-113). */
enum { ORC_OK = 0, ORC_INVALID = 1, ORC_OVERFLOW = 2, ORC_RUNTIME = 3 };

int orc_phase_derive(const orc_material* m, orc_derived* d);
int orc_phase_boundaries(const orc_material* m, double C, double P, orc_bounds* b);
int orc_phase_evaluate(const orc_material* m, double H, double C, double P, orc_phase* s);
int orc_phase_classify(const orc_material* m, double H, double C, double P, int* region);
/* Batch form; returns the error class of the lowest failing index (in
 * *first_bad) or 0. Outputs of failing points are NaN / region 0. */
int orc_phase_evaluate_batch(const orc_material* m, const double* H, const double* C,
                             const double* P, double P_const, size_t n,
                             orc_phase* out, long long* first_bad);

/* ---------------- transport (see transport_oracle.cpp) ---------------- */

typedef struct orc_transport_opts {
    int nx, ny;                 /* cells */
    double x0, x1, y0, y1;      /* domain */
    double pressure;            /* constant pressure model [Pa] */
    double cfl;                 /* time.cfl */
    double dt_initial, dt_max, dt_min; /* time.step initial/maximum/minimum */
    double theta;               /* Darcy exponent theta (flow.material.theta) */
    double inflow_H, inflow_C;  /* inflow_outflow reservoir values */
    int H_policy, C_policy;     /* 0 inflow_outflow, 1 outflow, 2 zero_flux */
    int integrator;             /* 2 = SSPRK2 (reference), 3 = Shu-Osher SSPRK3 */
    int lf_global;              /* 0 local LF, 1 global LF */
    double lf_global_speed;
    int uniform_tables;         /* 1: one stencil table set for all cells (uniform mesh) */
    int threads;                /* OpenMP threads (0 = default) */
    /* Mesh family (src/core/mesh.cpp:27-55): 0 rectangular, 1 perturbed
     * quadrilateral (interior vertices moved by perturbation * spacing *
     * SplitMix64 noise keyed by seed), 2 sine-stretched. */
    int mesh_family;
    double perturbation;
    unsigned long long seed;
} orc_transport_opts;

typedef struct orc_step_report {
    int status;                 /* 0 ok, else error code (see transport_oracle.cpp) */
    int retries;
    double dt, time, courant;
    double boundaryH, boundaryC, sourceH, maxRate, divergence;
    double balanceH, balanceC;
    double H_integral, C_integral;
} orc_step_report;

typedef struct orc_transport orc_transport;

orc_transport* orc_transport_create(const orc_material* m, const orc_transport_opts* o);
void orc_transport_destroy(orc_transport* t);
/* Face velocity normal components at edge Gauss points, per canonical edge id
 * (reference MeshInfo ids: AlongI first, then AlongJ) and canonical q. */
int orc_transport_set_face_velocity(orc_transport* t, const double* vs_n, const double* ud_n);
int orc_transport_set_state(orc_transport* t, const double* H, const double* C, double time);
int orc_transport_get_state(const orc_transport* t, double* H, double* C, double* T, double* phi);
/* One stage evaluation L(U) of the current state (RHS in evolve.cpp). */
int orc_transport_rhs(orc_transport* t, double* rhsH, double* rhsC, double* T, double* phi,
                      double* rate, orc_step_report* rates);
/* Advance nsteps accepted steps. */
int orc_transport_step(orc_transport* t, int nsteps, orc_step_report* report);
/* Time controls of evolve.cpp:449-457,483: control 0 = cfl, 1 = fixed (dt =
 * dt_initial); t_end = INFINITY for none (the last step lands on t_end). */
int orc_transport_set_time_control(orc_transport* t, int control, double t_end);
/* Thermal diffusion (evolve.cpp:330-349): diffusivity kappa >= 0 and, per wall
 * (0 bottom y0, 1 top y1, 2 left x0, 3 right x1), type 0 zero flux, 1
 * prescribed temperature, 2 prescribed outward flux, with its value. */
int orc_transport_set_diffusion(orc_transport* t, double kappa, const int* types, const double* values);
/* Phase-law pressure (initialization.cpp:148-163): model 0 constant (value in
 * Pa), 1 lithostatic with the surface at y = value. */
int orc_transport_set_pressure_model(orc_transport* t, int model, double value);
/* Vertical flow velocities (solid, Darcy) at the cell quadrature points
 * [cell*25 + b*5 + a], for the adiabatic source (evolve.cpp:359-369). */
int orc_transport_set_cell_velocity(orc_transport* t, const double* vs_y, const double* ud_y);
int orc_transport_limiter(orc_transport* t, double* thetaH, double* thetaC);
/* The mesh vertices, (nx+1)*(ny+1) (x, y) pairs, x fastest. */
int orc_transport_vertices(const orc_transport* t, double* xy);

/* Legacy dry preheat (src/couple/preheat.cpp:65-287) on a transport handle:
 * the Stokes velocity is vs_n of set_face_velocity (ud_n unused), H is
 * advected and diffused with the diffusivity and wall conditions of
 * set_diffusion, C stays fixed; set_time_control gives the control and
 * time.end, the opts dt_initial/dt_min/dt_max/cfl the step controls.
 * One row per accepted step (PreheatStep, src/couple/preheat.h:6-11). */
typedef struct orc_preheat_step {
    long long step;
    double time, dt, courant, integral, minimum, maximum, boundaryFlux, balanceError;
} orc_preheat_step;
/* Build (preheat.cpp:65-159) + the start of Run: per-cell rate, step limit,
 * first history row; resets the run's step counter. */
int orc_preheat_begin(orc_transport* t, double* rate, double* limit, orc_preheat_step* first);
/* RHS (preheat.cpp:160-200) of the current H: dH/dt and the boundary flux. */
int orc_preheat_rhs(orc_transport* t, double* rhs, double* boundary_flux);
/* Up to nsteps forward-Euler steps of Run (preheat.cpp:254-282), stopping at
 * time.end; *taken rows written. max_steps = time.maximumSteps. */
int orc_preheat_advance(orc_transport* t, long long max_steps, long long nsteps, orc_preheat_step* rows,
                        long long* taken);
/* Diagnostics (preheat.cpp:202-233): cell T and phi. */
int orc_preheat_diagnostics(orc_transport* t, double* T, double* phi);

/* Synthetic input builders shared by tests and bench (SplitMix64 noise as in
 * src/core/mesh.cpp:12-25). */
double orc_unit_noise(uint64_t seed, uint64_t field, uint64_t cell);
int orc_gauss_rule(int n, double* points, double* weights);

#ifdef __cplusplus
}
#endif
#endif

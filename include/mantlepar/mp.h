/*
 * mantlepar_b200 C ABI: the drop-in boundary of the MantlePar ML-WENO H/C
 * transport + eutectic phase hot path on NVIDIA B200 (sm_100a).
 *
 * Plain C: opaque handles, caller-owned buffers, status codes, no exceptions
 * and no C++ or torch types cross this boundary. Every entry point returns an
 * mp_status (0 = success) and assigns its outputs only on success unless
 * stated otherwise; mp_last_error_string() describes the last failure of the
 * calling thread. Handles are not thread-safe; use one handle per stream.
 *
 * Array layouts follow the reference:
 *  - cell fields: natural order id = j*nx + i, x fastest
 *    (src/couple/evolve.cpp:66, src/couple/initialization.h:137-139);
 *  - edges: reference MeshInfo ids (src/core/mesh_info.h:84): AlongI edges
 *    j*nx + i (j = 0..ny) first, then AlongJ edges nx*(ny+1) + j*(nx+1) + i;
 *  - edge Gauss points: 5 per edge along the canonical direction (increasing
 *    i or j, src/core/mesh_info.h:37), normal components against the
 *    canonical right normal (dy,-dx)/length (src/core/integral.cpp:62-89).
 * Pointers given to set/get calls may be host or device memory (UVA).
 */
#ifndef MANTLEPAR_MP_H
#define MANTLEPAR_MP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* mp_stream_t; /* == cudaStream_t; NULL = default stream */

/* Status classes mirror the PETSc error classes the reference raises on this
 * path (numeric values are project-defined; PETSc's are not vendored), plus
 * the three exception classes of src/phase/eutectic_rescaled.h:111-113. */
typedef enum mp_status {
    MP_OK = 0,
    MP_ERR_ARG_SIZ = 60,          /* PETSC_ERR_ARG_SIZ */
    MP_ERR_ARG_WRONG = 62,        /* PETSC_ERR_ARG_WRONG */
    MP_ERR_ARG_OUTOFRANGE = 63,   /* PETSC_ERR_ARG_OUTOFRANGE */
    MP_ERR_FP = 72,               /* PETSC_ERR_FP */
    MP_ERR_ARG_WRONGSTATE = 73,   /* PETSC_ERR_ARG_WRONGSTATE */
    MP_ERR_PLIB = 77,             /* PETSC_ERR_PLIB (conservation balance) */
    MP_ERR_NOT_CONVERGED = 91,    /* PETSC_ERR_NOT_CONVERGED (step retries) */
    MP_ERR_PHASE_INVALID = 101,   /* std::invalid_argument from EutecticModel */
    MP_ERR_PHASE_OVERFLOW = 102,  /* std::overflow_error from EutecticModel */
    MP_ERR_PHASE_RUNTIME = 103,   /* std::runtime_error from EutecticModel */
    MP_ERR_TIMEOUT = 110,         /* a bounded device wait ran out */
    MP_ERR_NOMEM = 111,           /* device memory exhausted / admission refused */
    MP_ERR_CUDA = 112             /* CUDA runtime error */
} mp_status;

/* Last failure of the calling thread (static storage, never NULL). */
const char* mp_last_error_string(void);

/* ------------------------------------------------------------------ phase */

/* Replaces mantle::phase::MaterialParameters (src/phase/eutectic_rescaled.h:10-26). */
typedef struct mp_material {
    double Tm0, Te0, nu, L, cp, Xe, rho, rhor, mus, mul, k0, g, alpha0;
} mp_material;

/* Replaces mantle::phase::DerivedParameters (src/phase/eutectic_rescaled.h:29-41). */
typedef struct mp_derived {
    double dT, h0, gamma, LD, TDm0, TDe0, invk0, l0, u0, p0, t0;
} mp_derived;

/* Replaces mantle::phase::PhaseBoundaries (src/phase/eutectic_rescaled.h:52-57). */
typedef struct mp_phase_bounds {
    double Tep, Tmp, H_eutectic_end, H_liquidus;
} mp_phase_bounds;

/* Structure-of-arrays output of a phase batch (device pointers). Any pointer
 * may be NULL to skip that field. region holds mantle::phase::PhaseRegion
 * values 1..6 (src/phase/eutectic_rescaled.h:43-50); flags bit 0 has_solid,
 * bit 1 has_liquid, bit 2 finite_temperature_derivatives. */
typedef struct mp_phase_soa {
    double *phi1, *phi2, *phil, *cl, *cs, *TDp, *Tep, *dTD_dCD, *dTD_dHD;
    int8_t* region;
    uint8_t* flags;
} mp_phase_soa;

typedef struct mp_phase_model mp_phase_model;

/* Replaces EutecticModel::EutecticModel / setParameters
 * (src/phase/eutectic_rescaled.h:105,109; .cpp:42-86,137-141). Invalid
 * parameters -> MP_ERR_PHASE_INVALID / MP_ERR_PHASE_OVERFLOW; a rejected
 * update leaves the model unchanged. */
mp_status mp_phase_create(const mp_material* params, mp_phase_model** model);
mp_status mp_phase_set_params(mp_phase_model* model, const mp_material* params);
mp_status mp_phase_get_params(const mp_phase_model* model, mp_material* params);
mp_status mp_phase_get_derived(const mp_phase_model* model, mp_derived* derived);
void mp_phase_destroy(mp_phase_model* model);

/* Replaces EutecticModel::boundaries (src/phase/eutectic_rescaled.h:116,
 * .cpp:163-185). Host computation with the same FP64 operations the kernels use. */
mp_status mp_phase_boundaries(const mp_phase_model* model, double C, double P, mp_phase_bounds* out);

/* Batched EutecticModel::evaluate (src/phase/eutectic_rescaled.h:114,
 * .cpp:192-282) on the GPU. H, C, P are device arrays of length n; P may be
 * NULL, then P_const applies to every point. Returns the status of the
 * lowest failing index (written to *first_bad, -1 if none). Synchronous on
 * `stream`. On failure the failing points hold NaN and the other points
 * hold their values; a failing point's region is the selected region when
 * the failure came after region selection (fractions or temperatures of the
 * evaluation itself), else 0 (invalid input, unresolvable intervals). */
mp_status mp_phase_evaluate_batch(const mp_phase_model* model, const double* H, const double* C,
                                  const double* P, double P_const, size_t n,
                                  const mp_phase_soa* out, long long* first_bad, mp_stream_t stream);

/* mp_phase_evaluate_batch for callers holding host memory only (the
 * reference's C++ code has no CUDA): H, C, P and every non-NULL field of
 * `out` are HOST arrays of length n; inputs are staged through device memory
 * owned by the model. Same statuses and failure semantics as the batch call.
 * Calls on one model are serialised. Replaces EutecticModel::evaluate /
 * classify (src/phase/eutectic_rescaled.h:114-115) for host callers. */
mp_status mp_phase_evaluate_host(const mp_phase_model* model, const double* H, const double* C,
                                 const double* P, double P_const, size_t n,
                                 const mp_phase_soa* out, long long* first_bad);

/* Replaces EutecticModel::pressureCorrectedTemperature
 * (src/phase/eutectic_rescaled.h:128, .cpp:143-149): TD + P/nu/dT with long
 * double intermediates. Non-finite input -> MP_ERR_PHASE_INVALID; an
 * unrepresentable result -> MP_ERR_PHASE_OVERFLOW. */
mp_status mp_phase_pressure_corrected_temperature(const mp_phase_model* model, double TD, double P, double* out);

/* Replaces EutecticModel::staticPressure (src/phase/eutectic_rescaled.h:129-130,
 * .cpp:151-161): rho*g*zD*length_scale; the one-argument reference form is
 * length_scale = derived l0. length_scale must be finite and positive. */
mp_status mp_phase_static_pressure(const mp_phase_model* model, double zD, double length_scale, double* out);

/* ------------------------------------------------------------- transport */

/* Uniform rectangular mesh (src/core/mesh.cpp:27-55, uniform family). */
typedef struct mp_mesh_desc {
    int nx, ny;            /* cells per axis, >= 2 each */
    double x0, x1, y0, y1; /* domain */
} mp_mesh_desc;

enum { MP_BC_INFLOW_OUTFLOW = 0, MP_BC_OUTFLOW = 1, MP_BC_ZERO_FLUX = 2 };
enum { MP_SSPRK2 = 2, MP_SSPRK3 = 3 };
/* The precision form. MP_PRECISION_MIXED (no counterpart in the reference)
 * is held to 1e-6 per cell against the FP64 results; on this path only FP64
 * values meet that bar for the porosity of cells near the solidus, and an
 * FP32 screen of the limiter scan that returns the FP64 values exactly was
 * measured slower than the FP64 scan, so the form evaluates the FP64 stage
 * (its results equal MP_PRECISION_FP64 bit for bit). */
enum { MP_PRECISION_FP64 = 0, MP_PRECISION_MIXED = 1 };

/* Subset of mantle::couple::Configuration used on this path
 * (src/couple/initialization.cpp:132-164,236-244,266-279; input.h:154-159). */
typedef struct mp_transport_opts {
    mp_material material;
    double pressure;          /* constant pressure model [Pa] */
    double cfl;               /* time.step.cfl, in (0,1] */
    double dt_initial, dt_max, dt_min;
    double theta;             /* flow.material.theta (Darcy exponent) */
    double inflow_H, inflow_C;/* inflow_outflow reservoir values */
    int H_policy, C_policy;   /* MP_BC_* for enthalpy / composition */
    int integrator;           /* MP_SSPRK2 (reference) or MP_SSPRK3 */
    int lf_global;            /* 0 local Lax-Friedrichs, 1 global */
    double lf_global_speed;
    double diffusivity;       /* thermal diffusivity kappa >= 0 (evolve.cpp:330-349) */
    int precision;            /* MP_PRECISION_FP64 or MP_PRECISION_MIXED */
} mp_transport_opts;

/* Per accepted step (history columns of src/couple/evolve.cpp:399-418,443). */
typedef struct mp_step_report {
    int status, retries;
    double dt, time, courant;
    double boundaryH, boundaryC, sourceH, maxRate, divergence;
    double balanceH, balanceC, H_integral, C_integral;
} mp_step_report;

/* Totals of one stage evaluation (Rates in src/couple/evolve.cpp:156). */
typedef struct mp_stage_totals {
    double boundaryH, boundaryC, sourceH, maxRate, divergence;
} mp_stage_totals;

typedef struct mp_transport mp_transport;

/* Replaces the setup half of mantle::couple::AdvancePhaseCoupled
 * (src/couple/evolve.h:17; Build at evolve.cpp:221-268 and
 * StateReconstruction::Initialize at state_reconstruction.cpp:35-96). */
mp_status mp_transport_create(const mp_mesh_desc* mesh, const mp_transport_opts* opts,
                              mp_stream_t stream, mp_transport** out);
void mp_transport_destroy(mp_transport* t);

/* General quad meshes: the reference's perturbed-quadrilateral and stretched
 * families (src/core/mesh.cpp:27-55, input mesh.family
 * "perturbed_quadrilateral"), or any logically rectangular mesh of convex
 * quads. xy holds the (nx+1)*(ny+1) vertices, x fastest, as (x, y) pairs;
 * mesh gives nx, ny and the domain. Every cell gets its own reconstruction
 * tables (built at create, TensorStencilPoly::Initialize and
 * SetTargetSmoothness per stencil, src/mlweno/tensorstencilpoly.cpp:146-231,
 * 383-398) and every evaluation point its own geometry. FP64 (the mixed
 * form evaluates the same FP64 stage); cells
 * failing the reference's quad check (src/core/quad_validation.h) ->
 * MP_ERR_ARG_WRONG. All other mp_transport_* calls apply unchanged; row
 * slabs: mp_transport_create_quads_slab. */
enum { MP_MESH_RECTANGULAR = 0, MP_MESH_PERTURBED = 1, MP_MESH_SINE_STRETCHED = 2 };
mp_status mp_transport_create_quads(const mp_mesh_desc* mesh, const double* xy, const mp_transport_opts* opts,
                                    mp_stream_t stream, mp_transport** out);
/* Device bytes a whole-mesh transport of this mesh allocates (quads != 0:
 * a general quad mesh, its per-cell tables and the builder's transient copy
 * of the vertices included), in whole 2 MiB allocation pages; 0 for an
 * invalid mesh. Not included: the first quad-mesh transport of a process
 * raises the CUDA runtime's per-thread stack reservation to the per-cell
 * table builder's 2.7 KB (about 0.5 GB more on a B200), once, for the rest
 * of the process. No counterpart in the reference (host memory there). */
size_t mp_transport_instance_bytes(const mp_mesh_desc* mesh, int quads);
/* Vertices of a reference mesh family (VertexAt, src/core/mesh.cpp:27-55):
 * perturbation in [0, 0.25) of the spacing for MP_MESH_PERTURBED, keyed by
 * seed (SplitMix64, as the reference). xy: (nx+1)*(ny+1) (x, y) pairs. */
mp_status mp_mesh_vertices(const mp_mesh_desc* mesh, int family, double perturbation, unsigned long long seed,
                           double* xy);

/* Flow supplier output (stays on PETSc in a coupled run): normal solid and
 * Darcy velocity at every edge Gauss point, arrays of edges*5 doubles.
 * Replaces the samples of SampleInitialFlow (src/couple/flow_sampling.cpp:62-121). */
mp_status mp_transport_set_face_velocity(mp_transport* t, const double* vs_n, const double* ud_n);

/* Cell averages H, C (length nx*ny) and the clock; resets accepted steps
 * (LoadPreheatState semantics, src/couple/evolve.cpp:54-125). */
mp_status mp_transport_set_state(mp_transport* t, const double* H, const double* C, double time);
/* Current H, C and the cell-averaged T, phi of the latest stage evaluation;
 * any pointer may be NULL. */
mp_status mp_transport_get_state(mp_transport* t, double* H, double* C, double* T, double* phi);

/* One stage evaluation L(U) of the current state (RHS, src/couple/evolve.cpp:279-384).
 * Outputs (length nx*ny, host or device) may be NULL. */
mp_status mp_transport_rhs(mp_transport* t, double* rhsH, double* rhsC, double* T, double* phi,
                           double* rate, mp_stage_totals* totals);

/* Advance nsteps accepted steps (the time loop of src/couple/evolve.cpp:428-511);
 * reports (may be NULL) receives one entry per step. On failure the state
 * is rolled back to the last accepted step (evolve.cpp:493-499). */
mp_status mp_transport_step(mp_transport* t, int nsteps, mp_step_report* reports);

/* Device-resident stepping (no counterpart in the reference, whose step loop
 * is host code). With enable != 0 (the default) mp_transport_step on a
 * whole mesh (uniform or general quad) runs as one CUDA graph per 64 steps: the
 * step and retry loops are conditional graph nodes and every decision of the
 * loop above is taken on the device, one host wait per graph launch; results,
 * reports and errors equal the host-driven loop (enable = 0) bit for bit.
 * Row slabs and profiling runs use the host-driven loop. */
mp_status mp_transport_set_device_steps(mp_transport* t, int enable);
/* Host waits for device results made by the stepping and RHS calls so far. */
mp_status mp_transport_run_stats(const mp_transport* t, unsigned long long* host_syncs);

/* Time controls of the coupled loop (src/couple/evolve.cpp:449-457,483;
 * TimeInput in src/input/input.h:154-158). MP_TIME_CFL (default): dt =
 * min(remaining, first step ? dt_initial : dt_max, cfl / stage rate), halved
 * on a failed stage (<= 40 retries). MP_TIME_FIXED: dt = min(remaining,
 * dt_initial); MP_ERR_ARG_OUTOFRANGE when that exceeds the CFL bound or a
 * stage fails. t_end (INFINITY = none): the last step is shortened to land
 * on it and mp_transport_step stops there (report entries of steps not taken
 * have dt = 0 and time = t_end). */
enum { MP_TIME_CFL = 0, MP_TIME_FIXED = 1 };
mp_status mp_transport_set_time_control(mp_transport* t, int control, double t_end);

/* Thermal conditions of the diffusion, one per wall: [0] bottom (y0), [1] top
 * (y1), [2] left (x0), [3] right (x1) (TransportBoundarySpecification
 * ::temperature, EvaluateThermalBoundary, src/couple/initialization.cpp:490-506):
 * MP_THERMAL_ZERO_FLUX (default), MP_THERMAL_TEMPERATURE (prescribed
 * dimensionless temperature), MP_THERMAL_FLUX (prescribed physical outward
 * diffusive flux per unit length; applies even with kappa = 0). */
enum { MP_THERMAL_ZERO_FLUX = 0, MP_THERMAL_TEMPERATURE = 1, MP_THERMAL_FLUX = 2 };
mp_status mp_transport_set_thermal_bc(mp_transport* t, const int* type, const double* value);

/* Phase-law pressure (initialization.cpp:148-163): MP_PRESSURE_CONSTANT with
 * value = pressure in Pa (>= 0; the create-time opts.pressure), or
 * MP_PRESSURE_LITHOSTATIC with value = surface_y (>= the mesh top): P(y) =
 * rho g l0 (surface_y - y) (EutecticModel::staticPressure), so the eutectic
 * temperature of every evaluation point depends on its height. */
enum { MP_PRESSURE_CONSTANT = 0, MP_PRESSURE_LITHOSTATIC = 1 };
mp_status mp_transport_set_pressure_model(mp_transport* t, int model, double value);

/* Vertical solid and Darcy velocity components at the 5x5 cell quadrature
 * points, [cell*25 + b*5 + a] (point (g_a, g_b) of the cell's Gauss rule), from
 * the flow supplier (flow_sampling.cpp:93-101). Required when alpha0 != 0:
 * the adiabatic source -alpha0 l0 g / cp * T * v_mix,y (evolve.cpp:359-369).
 * On a slab: the cells of the local mesh. */
mp_status mp_transport_set_cell_velocity(mp_transport* t, const double* vs_y, const double* ud_y);

/* Current time and accepted steps (InitialState::time, acceptedSteps). */
mp_status mp_transport_get_time(const mp_transport* t, double* time, int* accepted);

/* ------------------------------------------------------ row-slab domains */

/* One row slab of a mesh decomposed across GPUs or processes (the reference
 * partitions the cell DMDA, src/couple/state_reconstruction.cpp:40-58): the
 * slab owns global rows [row_begin, row_end) and keeps up to two halo rows
 * below and above (where the global mesh has them). Tables, boundary classes,
 * physical walls and error keys use the global mesh, so a decomposed run
 * reproduces the single-domain run cell by cell. Entry points on a slab:
 *  - set_state / get_state / rhs / limiter take and return the OWNED rows
 *    ((row_end - row_begin) * nx values);
 *  - set_face_velocity takes the edges of the LOCAL mesh: nx x local_rows
 *    cells starting at global row `row0` (mp_transport_slab_layout), in the
 *    edge order of mantlepar/mp.h;
 *  - before every stage the halo hook must fill the stage input's halo rows
 *    from the neighbours' owned rows, and after every reduction the combine
 *    hook must combine the totals and the status word across all slabs
 *    (maxRate, divergence, Cmax, nonfinite: max; Hmin, Cmin: min; the others:
 *    sum; status: min). Every slab must call the same entry points in the
 *    same order. */
typedef struct mp_stage_partials {
    double maxRate, divergence, boundaryH, boundaryC, H_integral, C_integral, Hmin, Cmin, Cmax, nonfinite;
    double sourceH;   /* adiabatic source integral: sum */
} mp_stage_partials;
/* H, C: the stage input (device, local rows); return 0 or a status. */
typedef int (*mp_halo_fn)(void* user, double* H, double* C);
typedef int (*mp_combine_fn)(void* user, mp_stage_partials* totals, unsigned long long* status);

mp_status mp_transport_create_slab(const mp_mesh_desc* global_mesh, int row_begin, int row_end,
                                   const mp_transport_opts* opts, mp_stream_t stream, mp_transport** out);
/* local_rows: rows held (owned + halos); row0: global row of local row 0;
 * own_begin/own_end: local rows owned. */
/* A row slab of a general quad mesh: xy holds the vertices of the WHOLE
 * mesh (as mp_transport_create_quads); every local cell's tables are built
 * from its stencil in the whole mesh, so slabs reproduce the single run. */
mp_status mp_transport_create_quads_slab(const mp_mesh_desc* global_mesh, const double* xy, int row_begin, int row_end,
                                         const mp_transport_opts* opts, mp_stream_t stream, mp_transport** out);
mp_status mp_transport_slab_layout(const mp_transport* t, int* local_rows, int* row0, int* own_begin, int* own_end);
mp_status mp_transport_set_hooks(mp_transport* t, mp_halo_fn halo, mp_combine_fn combine, void* user);

/* Limiter factors theta_H, theta_C of the current state
 * (StateReconstruction::Limit, src/couple/state_reconstruction.cpp:136-192). */
mp_status mp_transport_limiter(mp_transport* t, double* thetaH, double* thetaC);

/* ---------------------------------------------------------------- preheat */

/* The legacy dry preheat (mantle::couple::AdvanceLegacyPreheat,
 * src/couple/preheat.h:26, preheat.cpp:65-287): H_t + div(us H - kappa grad H)
 * = 0 with C held fixed and the Stokes velocity us frozen; forward Euler with
 * the UNLIMITED ML-WENO reconstruction of H at the edge Gauss points, the
 * linear-law Lax-Friedrichs flux (IntegrateAdvectiveFlux,
 * src/mlweno/advectiveflux.cpp:327-338; boundary faces
 * IntegrateAdvectiveBoundaryFlux :426-437), and the normal-line diffusion of
 * H evaluated on constant cell-average samples. The per-cell rate, and so
 * the step limit cfl / max rate, is fixed at begin (Build). */
typedef struct mp_preheat_opts {
    mp_material material;      /* phase model of the final diagnostics */
    int pressure_model;        /* MP_PRESSURE_CONSTANT / MP_PRESSURE_LITHOSTATIC */
    double pressure;           /* constant model: Pa; lithostatic: surface_y */
    double end;                /* time.end */
    long long max_steps;       /* time.maximumSteps */
    int control;               /* MP_TIME_CFL or MP_TIME_FIXED */
    double dt_initial, dt_min, dt_max;
    double cfl;                /* time.step.cfl, in (0, 1] */
    double diffusivity;        /* kappa >= 0 */
    int thermal_type[4];       /* MP_THERMAL_*, walls bottom, top, left, right */
    double thermal_value[4];
    int H_policy;              /* MP_BC_* advection boundary of H */
    double inflow_H;
    int lf_global;             /* 0 local Lax-Friedrichs, 1 global */
    double lf_global_speed;
} mp_preheat_opts;

/* PreheatStep (src/couple/preheat.h:6-11): one accepted step, or the
 * initial state (dt = courant = boundaryFlux = balanceError = 0). */
typedef struct mp_preheat_step {
    long long step;
    double time, dt, courant, integral, minimum, maximum, boundaryFlux, balanceError;
} mp_preheat_step;

/* PreheatReport (src/couple/preheat.h:13-17) without the history. */
typedef struct mp_preheat_report {
    double initialTime, finalTime, stepLimit;
    double initialIntegral, finalIntegral, boundaryIntegral;
} mp_preheat_report;

typedef struct mp_preheat mp_preheat;

mp_status mp_preheat_create(const mp_mesh_desc* mesh, const mp_preheat_opts* opts, mp_stream_t stream,
                            mp_preheat** out);
/* The preheat on a general quad mesh (the reference's Build and RHS read
 * each face's and cell's own corners, preheat.cpp:86-117,166-196, so its
 * preheat runs on every mesh family): xy as mp_transport_create_quads,
 * per-cell reconstruction tables, physical edge lengths, normal-line
 * spacing per edge point and per-cell areas. Same calls and results
 * otherwise; invalid quads -> MP_ERR_ARG_WRONG. */
mp_status mp_preheat_create_quads(const mp_mesh_desc* mesh, const double* xy, const mp_preheat_opts* opts,
                                  mp_stream_t stream, mp_preheat** out);
void mp_preheat_destroy(mp_preheat* p);
/* Stokes velocity at the edge Gauss points: normal components [edge*5 + q]
 * in the canonical order of this header (the x component on AlongJ edges,
 * minus the y component on AlongI edges). */
mp_status mp_preheat_set_velocity(mp_preheat* p, const double* vn);
/* Cell averages H, C (nx*ny), the clock and InitialState::acceptedSteps. */
mp_status mp_preheat_set_state(mp_preheat* p, const double* H, const double* C, double time, long long accepted);
mp_status mp_preheat_get_state(mp_preheat* p, double* H, double* time, long long* accepted);
/* Build (preheat.cpp:65-159) and the start of Run (:235-253): the per-cell
 * rate (nx*ns, may be NULL), the step limit and the first history row;
 * resets the run's step counter. MP_ERR_ARG_OUTOFRANGE when the state time
 * exceeds time.end or a global LF speed is below a flow normal speed. */
mp_status mp_preheat_begin(mp_preheat* p, double* rate, double* limit, mp_preheat_step* first);
/* RHS (preheat.cpp:160-200) of the current H: dH/dt (may be NULL) and the
 * outward boundary flux. */
mp_status mp_preheat_rhs(mp_preheat* p, double* rhs, double* boundary_flux);
/* Up to nsteps forward-Euler steps of Run (preheat.cpp:254-282), fewer when
 * time.end is reached; rows (may be NULL) receives one entry per accepted
 * step, *taken their number. Steps are issued in batches without a host
 * round trip per step: the step sizes are fixed by the controls, and each
 * step's finiteness and heat-balance checks run on the device, a failed
 * step stopping the ones queued after it. On failure the state is the last
 * accepted one (preheat.h:24-25) and the status says why:
 * MP_ERR_FP (non-finite candidate), MP_ERR_PLIB (heat balance),
 * MP_ERR_ARG_OUTOFRANGE (step above the limit or below time.step.minimum,
 * backflow on an outflow-only wall), MP_ERR_NOT_CONVERGED (maximumSteps). */
mp_status mp_preheat_advance(mp_preheat* p, long long nsteps, mp_preheat_step* rows, long long* taken);
/* Diagnostics (preheat.cpp:202-233): cell T and phi from the 5x5 phase
 * quadrature of the unlimited reconstruction of H and C. */
mp_status mp_preheat_diagnostics(mp_preheat* p, double* T, double* phi);
/* AdvanceLegacyPreheat: begin, advance to time.end, diagnostics. history
 * (may be NULL) receives up to `capacity` rows (the initial row first);
 * *rows = rows produced; T, phi may be NULL. */
mp_status mp_preheat_run(mp_preheat* p, mp_preheat_report* report, mp_preheat_step* history,
                         long long capacity, long long* rows, double* T, double* phi);

/* --------------------------------------------------------------- batched */

/* Many independent transport instances of uneven size advanced together
 * (no counterpart in the reference, which runs one mesh per MPI job). Each
 * instance keeps the reference's semantics on its own: own dt from its CFL
 * rate, stage admissibility and courant retries, balance check, rollback on
 * failure (src/couple/evolve.cpp:449-507); one launch per stage kernel covers
 * all instances. Results are bitwise those of a single-instance run. */
typedef struct mp_batch mp_batch;
mp_status mp_batch_create(const mp_mesh_desc* meshes, int count, const mp_transport_opts* opts,
                          mp_stream_t stream, mp_batch** out);
void mp_batch_destroy(mp_batch* b);
/* Add an instance in a free slot (or a new one); remove frees its memory. */
mp_status mp_batch_add(mp_batch* b, const mp_mesh_desc* mesh, int* instance);
/* Add an instance on a general quad mesh (the vertices xy as
 * mp_transport_create_quads: the perturbed-quadrilateral and stretched
 * families of src/core/mesh.cpp:27-55). Its per-cell tables are built on the
 * GPU at add; its stage kernels are the quad mesh's, batched over the quad
 * instances' own work lists, and the accumulation, step control and graph
 * are shared with the uniform instances. Results equal the instance run
 * alone through mp_transport_create_quads bit for bit. A mesh failing the
 * quad check -> MP_ERR_ARG_WRONG and no instance. */
mp_status mp_batch_add_quads(mp_batch* b, const mp_mesh_desc* mesh, const double* xy, int* instance);
mp_status mp_batch_remove(mp_batch* b, int instance);
/* Device bytes one instance of this mesh holds (memory admission). */
size_t mp_batch_instance_bytes(const mp_mesh_desc* mesh);
size_t mp_batch_bytes_in_use(const mp_batch* b);
int mp_batch_slots(const mp_batch* b);
mp_status mp_batch_set_face_velocity(mp_batch* b, int instance, const double* vs_n, const double* ud_n);
mp_status mp_batch_set_state(mp_batch* b, int instance, const double* H, const double* C, double time);
/* Any output pointer may be NULL; status is the instance's sticky failure
 * status (0 = healthy). */
mp_status mp_batch_get_state(mp_batch* b, int instance, double* H, double* C, double* T, double* phi,
                             double* time, int* accepted, int* status);
/* nsteps accepted steps of every healthy instance; reports (may be NULL)
 * holds nsteps * slots entries, step-major; an instance that fails stops
 * (its status is reported) while the others continue. */
mp_status mp_batch_step(mp_batch* b, int nsteps, mp_step_report* reports);
/* Final time of an instance (time.end, src/couple/input.h:155): its steps
 * are limited to the remaining time and it stops there; finished() reports
 * it (within 32 eps, as src/couple/evolve.cpp:450-451). */
mp_status mp_batch_set_end_time(mp_batch* b, int instance, double t_end);
/* mp_transport_set_thermal_bc for every instance of the batch. */
mp_status mp_batch_set_thermal_bc(mp_batch* b, const int* type, const double* value);
/* Adiabatic source (alpha0 != 0, src/couple/evolve.cpp:359-369) of one
 * instance: the vertical solid and Darcy velocities at its 25 cell quadrature
 * points [cell*25 + b*5 + a], as mp_transport_set_cell_velocity. With alpha0
 * != 0 every instance needs them before it steps (MP_ERR_ARG_WRONGSTATE
 * otherwise); they take 424 bytes per cell beyond mp_batch_instance_bytes,
 * counted in mp_batch_bytes_in_use. */
mp_status mp_batch_set_cell_velocity(mp_batch* b, int instance, const double* vs_y, const double* ud_y);
int mp_batch_finished(const mp_batch* b, int instance);
/* Project autotuner: times the candidate reconstruction tile shapes and
 * cells-per-thread on this batch and keeps the fastest; tile = {bx, by, cpt}. */
mp_status mp_batch_autotune(mp_batch* b, int reps, int tile[3], double* best_ms);
mp_status mp_batch_profile(mp_batch* b, int enable);
/* Device-resident stepping (no counterpart in the reference, whose step loop
 * is host code): with enable != 0 (the default) mp_batch_step runs its steps
 * as one CUDA graph per 64 steps -- the step and retry loops are conditional
 * graph nodes and every dt, courant, admissibility, retry and balance
 * decision of the reference's loop (src/couple/evolve.cpp:449-507) is taken
 * on the device -- with one host wait per graph launch; results equal the
 * host-driven loop (enable = 0) bit for bit. Profiling (mp_batch_profile)
 * uses the host-driven loop. */
mp_status mp_batch_set_device_steps(mp_batch* b, int enable);
/* Host waits for device results made by the stepping calls so far, and the
 * number of times the step graph was captured (again only when an array's
 * capacity grows, the tile is retuned or the physics changes -- not when
 * instances come and go). Either pointer may be NULL. */
mp_status mp_batch_run_stats(const mp_batch* b, unsigned long long* host_syncs, unsigned long long* graph_captures);
mp_status mp_batch_kernel_times(mp_batch* b, double ms[6], unsigned long long launches[6]);

/* --------------------------------------------------------------- serving */

/* A request loop for transport solves of different sizes (no counterpart in
 * the reference): requests are admitted while their device bytes fit the
 * budget and the resident cells are below a target, advanced together one step at a time (continuous
 * batching: work that arrives while others run joins at the next step), and
 * released at their final time. Inputs are host arrays, copied on submit. */
typedef struct mp_server mp_server;
typedef struct mp_request_info {
    int status, accepted;       /* final status, accepted steps */
    double time;                /* reached time (= t_final on success) */
    double queue_s, latency_s;  /* submit -> admit, submit -> result */
    double cells;
} mp_request_info;
mp_status mp_serve_create(const mp_transport_opts* opts, size_t memory_budget, mp_server** out);
void mp_serve_destroy(mp_server* s);
mp_status mp_serve_submit(mp_server* s, const mp_mesh_desc* mesh, const double* H, const double* C,
                          const double* vs_n, const double* ud_n, double t_final, long long* id);
/* A request on a general quad mesh (the vertices xy as
 * mp_transport_create_quads; the perturbed-quadrilateral and stretched
 * families of src/core/mesh.cpp:27-55). It is admitted under the same budget
 * and resident-cell target and joins the same batch as a quad instance
 * (mp_batch_add_quads: per-cell tables built on admission), advanced with
 * the others one step per loop iteration. A mesh failing the quad check
 * finishes with MP_ERR_ARG_WRONG in its status; the server continues. */
mp_status mp_serve_submit_quads(mp_server* s, const mp_mesh_desc* mesh, const double* xy, const double* H,
                                const double* C, const double* vs_n, const double* ud_n, double t_final,
                                long long* id);
/* Block until request id finishes (timeout_s < 0: no limit; on expiry
 * MP_ERR_TIMEOUT and the request stays queued/running). */
mp_status mp_serve_wait(mp_server* s, long long id, double timeout_s, double* H, double* C, double* T,
                        double* phi, mp_request_info* info);
mp_status mp_serve_stats(mp_server* s, double* cell_updates, double* busy_s, long long* steps,
                         int* resident, int* queued);
/* Admission order and resident-cell target (0 = admit while memory fits).
 * Default: smallest estimated work (cells * t_final * cells per unit length)
 * first, 1e6 cells. A resident request advances one step per loop iteration
 * and an iteration steps every resident request, so the target trades
 * latency for throughput: on a B200, for meshes up to 320x640, 1e6 halves
 * the median latency of 4e6 at a sustainable load for 2-8 % less throughput;
 * a backlog is served faster with 4e6. */
enum { MP_SERVE_FIFO = 0, MP_SERVE_SMALLEST_WORK = 1 };
mp_status mp_serve_set_policy(mp_server* s, int order, double resident_cells_target);

/* One stage evaluation (as mp_transport_rhs) that allocates no device memory,
 * for callers that cannot call cudaMalloc -- e.g. code inside a framework that
 * owns all device memory through its own pool, or code that must not allocate
 * once its latency-critical phase has begun. No counterpart in the reference
 * (its CPU code allocates freely). All scratch lives in one fixed file-scope
 * device array (about 7.3 MB per GPU that loads the library, held until the
 * process exits); meshes above 32768 cells (nx*ny) are rejected with
 * MP_ERR_ARG_SIZ. Options are checked as mp_transport_create checks them;
 * kappa > 0, alpha0 != 0 and MP_PRECISION_MIXED are rejected with
 * MP_ERR_ARG_WRONG. Every call looks up the array's device address in the
 * current context. Calls share the array and overwrite it; calls that
 * overlap on the GPU race. All array arguments are device pointers (H, C,
 * rhsH, rhsC, T, phi: nx*ny; vs_n, ud_n: edges*5); rate and totals may be
 * NULL. The call is synchronous: it waits for `stream` and reads the stage
 * totals and status back to the host before it returns. */
mp_status mp_transport_rhs_noalloc(const mp_mesh_desc* mesh, const mp_transport_opts* opts,
                                   const double* H, const double* C, const double* vs_n, const double* ud_n,
                                   double* rhsH, double* rhsC, double* T, double* phi, double* rate,
                                   mp_stage_totals* totals, mp_stream_t stream);

/* ------------------------------------------------------------ measurement */

/* Number of this library's kernel launches issued so far (all handles). */
unsigned long long mp_kernel_launches(void);

/* Per-kernel CUDA-event timing of a handle's stage kernels (no counterpart in
 * the reference, which has no timers on this path). enable resets the
 * accumulators; kernel_times returns accumulated ms and launch counts for
 * [0] reconstruction/limiter, [1] cell phase quadrature, [2] faces,
 * [3] accumulation/RK, [4] axpy and reductions, [5] unused. */
mp_status mp_transport_profile(mp_transport* t, int enable);
mp_status mp_transport_kernel_times(mp_transport* t, double ms[6], unsigned long long launches[6]);

/* Measured FP64 FMA throughput of this GPU (TFLOP/s), the compute roof of
 * this FP64-bound path. */
mp_status mp_probe_fp64_peak(mp_stream_t stream, double* tflops);

#ifdef __cplusplus
}
#endif
#endif

// Reference-backed oracle: the transport driver over the reference's OWN
// compiled classes (src/mlweno Reconstruction/TensorStencilPoly, src/core
// geometry, src/mlweno diffusion sampling and advective flux, src/phase
// EutecticModel), built by
// oracle/Makefile from the sources where they lie into oracle/_ref.
// TEST INFRASTRUCTURE ONLY: used to pin the restated oracle and as the
// CPU baseline ("kind": "reference"); never part of the product library.
#include "reconstruction.h"
#include "diffusiveflux.h"
#include "advectiveflux.h"
#include "integral.h"
#include "eutectic_rescaled.h"

#include "oracle.h"
#include "transport_driver.hpp"

#include <stdexcept>

DM mp_shim_make_dm(PetscInt M, PetscInt N, const double* xy);
void mp_shim_free_dm(DM dm);

namespace {

using mantle::phase::EutecticModel;
using mantle::phase::MaterialParameters;
using mantle::phase::PhaseState;

MaterialParameters to_params(const orc_material& m) {
    MaterialParameters p;
    p.Tm0 = m.Tm0; p.Te0 = m.Te0; p.nu = m.nu; p.L = m.L; p.cp = m.cp; p.Xe = m.Xe;
    p.rho = m.rho; p.rhor = m.rhor; p.mus = m.mus; p.mul = m.mul; p.k0 = m.k0; p.g = m.g;
    p.alpha0 = m.alpha0;
    return p;
}

void to_state(const PhaseState& s, orc_phase& o) {
    o.phi1 = s.phi1; o.phi2 = s.phi2; o.phil = s.phil; o.cl = s.cl; o.cs = s.cs;
    o.region = (int)s.region; o.TDp = s.TDp; o.Tep = s.Tep; o.dTD_dCD = s.dTD_dCD;
    o.dTD_dHD = s.dTD_dHD; o.has_solid = s.has_solid; o.has_liquid = s.has_liquid;
    o.finite_temperature_derivatives = s.finite_temperature_derivatives;
}

template <class F>
int classify_exceptions(F&& f) {
    try { f(); return ORC_OK; }
    catch (const std::invalid_argument&) { return ORC_INVALID; }
    catch (const std::overflow_error&) { return ORC_OVERFLOW; }
    catch (const std::runtime_error&) { return ORC_RUNTIME; }
}

inline Point P(orc::Pt p) { Point q; q.p[0] = p.x; q.p[1] = p.y; return q; }
inline orc::Pt O(Point p) { return orc::Pt{p.p[0], p.p[1]}; }
inline QuadVertices Q(const orc::Quad& q) { return QuadVertices{{P(q[0]), P(q[1]), P(q[2]), P(q[3])}}; }
inline void check(PetscErrorCode e) { if (e) throw orc::Error{(int)e, "reference routine failed"}; }

struct RefBackend {
    // Reconstruction::Initialize reads the shared MeshInfo and writes only the
    // cell's own object: cells are set up across threads.
    static constexpr bool kParallelInit = true;
    MeshInfo mesh;
    const EutecticModel* model = nullptr;
    std::unique_ptr<EutecticModel> own;

    template <class D>
    void setup(D& d) {
        const PetscInt M = d.nx + 1, N = d.ny + 1;
        std::vector<double> xy((size_t)(M * N) * 2);
        for (size_t k = 0; k < d.vert.size(); ++k) { xy[2 * k] = d.vert[k].x; xy[2 * k + 1] = d.vert[k].y; }
        DM dm = mp_shim_make_dm(M, N, xy.data());
        const PetscErrorCode e = BuildMeshInfo(dm, nullptr, mesh);
        mp_shim_free_dm(dm);
        check(e);
        own.reset(new EutecticModel(to_params(d.mat)));
        model = own.get();
        shared_model() = model;
    }
    static const EutecticModel*& shared_model() { static const EutecticModel* m = nullptr; return m; }

    struct Recon {
        Reconstruction r;
        template <class D>
        void init(RefBackend& be, D&, int ti, int tj, double h) {
            // state_reconstruction.cpp:104-108
            ReconstructionOptions options;
            options.large.size = {3, 3}; options.large.order = 2; options.large.offsets = {{-1, -1}};
            options.small.size = {2, 2}; options.small.order = 1;
            options.small.offsets = {{0, -1}, {0, 0}, {-1, -1}, {-1, 0}};
            options.small.smoothness = ReconstructionSmoothness::TargetCell;
            check(r.Initialize(be.mesh, {ti, tj}, options, h));
        }
        void update(const std::vector<double>& field, int nx, double area) {
            const PetscInt ny = (PetscInt)(field.size() / (size_t)nx);
            check(r.Update(field, MeshRange{{0, 0}, {nx, ny}}, area));
        }
        double evaluate(orc::Pt p) const {
            PetscReal v;
            check(r.Evaluate(P(p), v));
            return v;
        }
    };

    static void gauss_rule(int n, std::vector<double>& p, std::vector<double>& w) {
        GaussRule1D rule;
        check(CreateGaussRule(n, rule));
        p = rule.points; w = rule.weights;
    }
    static double cell_area(const orc::Quad& q, const std::vector<double>& p, const std::vector<double>& w) {
        GaussRule1D rule; rule.points = p; rule.weights = w;
        PetscReal a;
        check(IntegrateCell(Q(q), rule, [](const Point&) { return PetscReal(1); }, a));
        return a;
    }
    static void edge_geometry(orc::Pt a, orc::Pt b, double& l, orc::Pt& n) {
        Point nn;
        check(GetEdgeGeometry(EdgeVertices{{P(a), P(b)}}, l, nn));
        n = O(nn);
    }
    static orc::Pt map_edge(double r, orc::Pt a, orc::Pt b) { return O(MapEdgePoint(r, EdgeVertices{{P(a), P(b)}})); }
    static orc::Pt map_cell(orc::Pt r, const orc::Quad& q) { return O(MapCellPoint(P(r), Q(q))); }
    static double cell_jacobian(orc::Pt r, const orc::Quad& q) { return CellJacobian(P(r), Q(q)); }
    static void sampling(orc::Pt a, orc::Pt b, const orc::Quad& l, const orc::Quad* r, const std::vector<double>& p,
                         const std::vector<double>& w, int N, double f, orc::Sampling& s) {
        GaussRule1D rule; rule.points = p; rule.weights = w;
        DiffusiveSamplingOptions opt; opt.numberOfSamples = N; opt.extentFraction = f;
        DiffusiveSampling ds;
        const EdgeVertices e{{P(a), P(b)}};
        if (r) check(CreateInteriorDiffusiveSampling(e, Q(l), Q(*r), rule, opt, ds));
        else check(CreateBoundaryDiffusiveSampling(e, Q(l), rule, opt, ds));
        s.samples.clear(); s.sides.clear();
        for (const Point& x : ds.SamplePoints()) s.samples.push_back(O(x));
        for (auto side : ds.SampleSides())
            s.sides.push_back(side == DiffusiveSampleSide::Left ? 0 : (side == DiffusiveSampleSide::Right ? 1 : 2));
        s.boundary = ds.IsBoundary();
        s.normal = O(ds.Normal());
        s.spacing = ds.Spacing();
        s.weights = ds.QuadratureWeights();
        s.coefficients = ds.Coefficients();
        s.native = std::make_shared<DiffusiveSampling>(ds);
    }
    static double static_pressure(const orc_material&, const orc_derived&, double zD) {
        double v = 0;
        const int code = classify_exceptions([&] { v = shared_model()->staticPressure(zD); });
        if (code != ORC_OK) throw orc::Error{orc::E_PHASE + code, "staticPressure failed"};
        return v;
    }
    // The reference's own IntegrateDiffusive(Boundary)FluxWithDerivatives
    // (diffusiveflux.h:150-193) on its own sampling object.
    static void diffuse(const orc::Sampling& s, const std::vector<double>& samples, double kappa,
                        const orc::ThermalBC* bc, double& flux, std::vector<double>& deriv) {
        const auto& ds = *static_cast<const DiffusiveSampling*>(s.native.get());
        const std::vector<PetscReal> kap(ds.QuadraturePoints().size(), kappa);
        DiffusiveEdgeFluxResult r;
        if (bc) {
            DiffusiveBoundaryValue v;
            v.type = bc->type == 0 ? DiffusiveBoundaryType::ZeroFlux
                   : (bc->type == 1 ? DiffusiveBoundaryType::PrescribedQuantity : DiffusiveBoundaryType::PrescribedFlux);
            v.value = bc->type == 0 ? 0.0 : bc->value;
            const std::vector<DiffusiveBoundaryValue> data(ds.QuadraturePoints().size(), v);
            check(IntegrateDiffusiveBoundaryFluxWithDerivatives(ds, samples, kap, data, 0.0, {}, r));
        } else {
            check(IntegrateDiffusiveFluxWithDerivatives(ds, samples, kap, 0.0, {}, r));
        }
        flux = r.flux;
        deriv = r.derivativeSamples;
    }
    // The reference's own IntegrateAdvectiveFlux / IntegrateAdvectiveBoundaryFlux
    // (advectiveflux.h:111-116,182-186) with the default linear law.
    static double advect(orc::Pt a, orc::Pt b, const std::vector<double>& p, const std::vector<double>& w,
                         const std::vector<orc::Pt>& vel, const std::vector<double>& left,
                         const std::vector<double>& right, bool global, double speed) {
        GaussRule1D rule; rule.points = p; rule.weights = w;
        std::vector<Point> v;
        for (const auto& x : vel) v.push_back(P(x));
        LaxFriedrichsOptions opt;
        opt.mode = global ? LaxFriedrichsMode::Global : LaxFriedrichsMode::Local;
        opt.globalSpeed = speed;
        PetscReal flux = 0;
        check(IntegrateAdvectiveFlux(EdgeVertices{{P(a), P(b)}}, rule, v, left, right, 0.0, {}, opt, flux));
        return flux;
    }
    static double advect_boundary(orc::Pt a, orc::Pt b, const std::vector<double>& p, const std::vector<double>& w,
                                  const std::vector<orc::Pt>& vel, const std::vector<double>& interior,
                                  const std::vector<orc::AdvectBC>& data) {
        GaussRule1D rule; rule.points = p; rule.weights = w;
        std::vector<Point> v;
        for (const auto& x : vel) v.push_back(P(x));
        std::vector<AdvectiveBoundaryValue> d(data.size());
        for (size_t q = 0; q < data.size(); ++q) {
            d[q].type = data[q].type == 0 ? AdvectiveBoundaryType::PrescribedState
                      : (data[q].type == 1 ? AdvectiveBoundaryType::ExtrapolatedState : AdvectiveBoundaryType::ZeroFlux);
            d[q].value = data[q].value;
        }
        PetscReal flux = 0;
        check(IntegrateAdvectiveBoundaryFlux(EdgeVertices{{P(a), P(b)}}, rule, v, interior, d, 0.0, {}, flux));
        return flux;
    }
    static bool phase(const orc_material&, const orc_derived&, double H, double C, double Pp, orc_phase& s, int& code) {
        const EutecticModel* m = shared_model();
        code = classify_exceptions([&] { to_state(m->evaluate(H, C, Pp), s); });
        return code == ORC_OK;
    }
    static bool derive(const orc_material& m, orc_derived& d) {
        return classify_exceptions([&] {
            EutecticModel model(to_params(m));
            const auto& x = model.derived();
            d = orc_derived{x.dT, x.h0, x.gamma, x.LD, x.TDm0, x.TDe0, x.invk0, x.l0, x.u0, x.p0, x.t0};
        }) == ORC_OK;
    }
};

using RefApi = orc::Api<RefBackend>;

}  // namespace

extern "C" {

int ref_phase_derive(const orc_material* m, orc_derived* d) {
    return RefBackend::derive(*m, *d) ? ORC_OK : ORC_INVALID;
}

int ref_phase_boundaries(const orc_material* m, double C, double P, orc_bounds* b) {
    return classify_exceptions([&] {
        EutecticModel model(to_params(*m));
        const auto x = model.boundaries(C, P);
        *b = orc_bounds{x.Tep, x.Tmp, x.H_eutectic_end, x.H_liquidus};
    });
}

int ref_phase_evaluate(const orc_material* m, double H, double C, double P, orc_phase* s) {
    return classify_exceptions([&] {
        EutecticModel model(to_params(*m));
        to_state(model.evaluate(H, C, P), *s);
    });
}

int ref_phase_classify(const orc_material* m, double H, double C, double P, int* region) {
    return classify_exceptions([&] {
        EutecticModel model(to_params(*m));
        *region = (int)model.classify(H, C, P);
    });
}

int ref_phase_evaluate_batch(const orc_material* m, const double* H, const double* C, const double* P,
                             double P_const, size_t n, orc_phase* out, long long* first_bad) {
    long long bad = -1;
    int code = classify_exceptions([&] { EutecticModel model(to_params(*m)); });
    if (code) { if (first_bad) *first_bad = -1; return code; }
    EutecticModel model(to_params(*m));
    const double nan = std::numeric_limits<double>::quiet_NaN();
    int first = ORC_OK;
    for (size_t i = 0; i < n; ++i) {
        const int c = classify_exceptions([&] { to_state(model.evaluate(H[i], C[i], P ? P[i] : P_const), out[i]); });
        if (c) {
            orc_phase z{};
            z.phi1 = z.phi2 = z.phil = z.cl = z.cs = z.TDp = z.Tep = z.dTD_dCD = z.dTD_dHD = nan;
            out[i] = z;
            if (bad < 0) { bad = (long long)i; first = c; }
        }
    }
    if (first_bad) *first_bad = bad;
    return first;
}

void* ref_transport_create(const orc_material* m, const orc_transport_opts* o) { return RefApi::create(m, o); }
void ref_transport_destroy(void* t) { RefApi::destroy(t); }
int ref_transport_set_face_velocity(void* t, const double* vs, const double* ud) { return RefApi::set_face_velocity(t, vs, ud); }
int ref_transport_set_state(void* t, const double* H, const double* C, double time) { return RefApi::set_state(t, H, C, time); }
int ref_transport_get_state(const void* t, double* H, double* C, double* T, double* phi) { return RefApi::get_state(t, H, C, T, phi); }
int ref_transport_rhs(void* t, double* a, double* b, double* T, double* phi, double* rate, orc_step_report* r) {
    return RefApi::rhs(t, a, b, T, phi, rate, r);
}
int ref_transport_limiter(void* t, double* a, double* b) { return RefApi::limiter(t, a, b); }
int ref_transport_step(void* t, int n, orc_step_report* r) { return RefApi::step(t, n, r); }
int ref_transport_set_time_control(void* t, int control, double t_end) { return RefApi::set_time_control(t, control, t_end); }
int ref_transport_set_pressure_model(void* t, int model, double value) { return RefApi::set_pressure_model(t, model, value); }
int ref_transport_set_cell_velocity(void* t, const double* a, const double* b) { return RefApi::set_cell_velocity(t, a, b); }
int ref_transport_set_diffusion(void* t, double kappa, const int* types, const double* values) {
    return RefApi::set_diffusion(t, kappa, types, values);
}

int ref_transport_vertices(const void* t, double* xy) { return RefApi::vertices(t, xy); }
int ref_preheat_begin(void* t, double* rate, double* limit, orc_preheat_step* first) {
    return RefApi::preheat_begin(t, rate, limit, first);
}
int ref_preheat_rhs(void* t, double* rhs, double* boundary_flux) { return RefApi::preheat_rhs(t, rhs, boundary_flux); }
int ref_preheat_advance(void* t, long long max_steps, long long nsteps, orc_preheat_step* rows, long long* taken) {
    return RefApi::preheat_advance(t, max_steps, nsteps, rows, taken);
}
int ref_preheat_diagnostics(void* t, double* T, double* phi) { return RefApi::preheat_diagnostics(t, T, phi); }

}  // extern "C"

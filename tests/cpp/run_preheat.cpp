// Test driver for the C++ preheat layer: reads a case, runs
// mantle::couple::AdvanceLegacyPreheat and WritePreheatHistory.
//
// input  (doubles): nx ny x0 x1 y0 y1 end control(0 cfl, 1 fixed) initialStep
//                   minimumStep maximumStep cfl maximumSteps kappa
//                   thermal type[4] value[4] H_policy(0 inflow/outflow,
//                   1 outflow, 2 zero flux) inflow_H lf_global lf_speed
//                   pressure_model(0 constant, 1 lithostatic) surface_y,
//                   has_vertices(0, 1) 0, then H[N] C[N] vs[5E] and, with
//                   has_vertices, the (nx+1)*(ny+1) (x, y) vertex pairs
// output (doubles): status, time, acceptedSteps, rows, H[N] T[N] phi[N],
//                   rows x (step time dt courant integral minimum maximum
//                   boundaryFlux balanceError), the six report scalars;
//                   preheat_history.csv at the third argument.
#include <cstdio>
#include <vector>

#include "mantle/couple/coupled_transport.h"

using namespace mantle::couple;

int main(int argc, char** argv) {
    if (argc != 4) { std::fprintf(stderr, "usage: run_preheat in out history.csv\n"); return 2; }
    std::FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    double h[30];
    if (std::fread(h, sizeof(double), 30, f) != 30) return 2;
    Mesh m;
    m.nx = (int)h[0]; m.ny = (int)h[1]; m.x0 = h[2]; m.x1 = h[3]; m.y0 = h[4]; m.y1 = h[5];
    mantle::phase::MaterialParameters p;
    p.Te0 = 250; p.Tm0 = 1250; p.L = 6e5; p.cp = 1200; p.Xe = 0.5; p.alpha0 = 0;
    Configuration c{mantle::phase::EutecticModel(p)};
    c.time.end = h[6];
    c.time.control = h[7] == 1 ? "fixed" : "cfl";
    c.time.initialStep = h[8];
    c.time.minimumStep = h[9];
    c.time.maximumStep = h[10];
    c.time.cfl = h[11];
    c.time.maximumSteps = (long)h[12];
    c.thermalDiffusivity = h[13];
    for (int w = 0; w < 4; ++w) {
        const int t = (int)h[14 + w];
        c.boundary.temperature[w].policy = t == 1 ? ThermalPolicy::Temperature
                                         : (t == 2 ? ThermalPolicy::OutwardFlux : ThermalPolicy::ZeroFlux);
        c.boundary.temperature[w].value = h[18 + w];
    }
    const int pol = (int)h[22];
    c.boundary.enthalpy.policy = pol == 0 ? AdvectionPolicy::InflowOutflow
                               : (pol == 1 ? AdvectionPolicy::Outflow : AdvectionPolicy::ZeroFlux);
    c.boundary.enthalpy.inflow = h[23];
    c.stabilizer.mode = h[24] == 1 ? LaxFriedrichsMode::Global : LaxFriedrichsMode::Local;
    c.stabilizer.globalSpeed = h[25];
    c.pressureModel = h[26] == 1 ? PressureModel::Lithostatic : PressureModel::Constant;
    c.surfaceY = h[27];
    const size_t N = (size_t)m.nx * m.ny, E = (size_t)EdgeCount(m) * 5;
    InitialState s;
    s.mesh = m;
    s.enthalpy.resize(N); s.composition.resize(N);
    EdgeVelocities v;
    v.solid.resize(E);
    if (std::fread(s.enthalpy.data(), 8, N, f) != N || std::fread(s.composition.data(), 8, N, f) != N ||
        std::fread(v.solid.data(), 8, E, f) != E) return 2;
    if (h[28] == 1) {
        const size_t V = 2 * (size_t)(m.nx + 1) * (m.ny + 1);
        s.mesh.vertices.resize(V);
        if (std::fread(s.mesh.vertices.data(), 8, V, f) != V) return 2;
    }
    std::fclose(f);

    PreheatReport rep;
    const int st = AdvanceLegacyPreheat(c, s, v, rep);
    const int ws = WritePreheatHistory(argv[3], c, m, rep);
    std::FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    const double head[4] = {(double)(st ? st : ws), s.time, (double)s.acceptedSteps, (double)rep.history.size()};
    std::fwrite(head, 8, 4, o);
    s.temperature.resize(N); s.porosity.resize(N);
    std::fwrite(s.enthalpy.data(), 8, N, o);
    std::fwrite(s.temperature.data(), 8, N, o);
    std::fwrite(s.porosity.data(), 8, N, o);
    for (const auto& r : rep.history) {
        const double row[9] = {(double)r.step, r.time, r.dt, r.courant, r.integral, r.minimum, r.maximum,
                               r.boundaryFlux, r.balanceError};
        std::fwrite(row, 8, 9, o);
    }
    const double tail[6] = {rep.initialTime, rep.finalTime, rep.stepLimit, rep.initialIntegral, rep.finalIntegral,
                            rep.boundaryIntegral};
    std::fwrite(tail, 8, 6, o);
    std::fclose(o);
    return 0;
}

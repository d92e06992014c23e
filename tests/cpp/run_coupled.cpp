// Test driver for the C++ coupled-transport layer: reads a case, runs
// mantle::couple::RHS and AdvancePhaseCoupled, writes the results.
//
// input  (doubles): nx ny x0 x1 y0 y1 t_end control(0 cfl, 1 fixed) initialStep
//                   cfl integrator maximumSteps, then H[N] C[N] vs[5E] ud[5E]
// output (doubles): status, rhs status, time, acceptedSteps, nsteps,
//                   rhsH[N] rhsC[N] maxRate, H[N] C[N] T[N] phi[N],
//                   then per step: dt retries courant
#include <cstdio>
#include <vector>

#include "mantle/couple/coupled_transport.h"

using namespace mantle::couple;

int main(int argc, char** argv) {
    if (argc != 3) { std::fprintf(stderr, "usage: run_coupled in out\n"); return 2; }
    std::FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    double h[12];
    if (std::fread(h, sizeof(double), 12, f) != 12) return 2;
    Mesh m;
    m.nx = (int)h[0]; m.ny = (int)h[1]; m.x0 = h[2]; m.x1 = h[3]; m.y0 = h[4]; m.y1 = h[5];
    mantle::phase::MaterialParameters p;
    p.Te0 = 250; p.Tm0 = 1250; p.L = 6e5; p.cp = 1200; p.Xe = 0.5; p.alpha0 = 0;
    Configuration c{mantle::phase::EutecticModel(p)};
    c.boundary.enthalpy = {AdvectionPolicy::InflowOutflow, 1.0};
    c.boundary.composition = {AdvectionPolicy::InflowOutflow, 0.3};
    c.time.end = h[6];
    c.time.control = h[7] == 1 ? "fixed" : "cfl";
    c.time.initialStep = h[8];
    c.time.maximumStep = 1e30;
    c.time.minimumStep = 1e-14;
    c.time.cfl = h[9];
    c.integrator = h[10] == 3 ? Integrator::SSPRK3 : Integrator::SSPRK2;
    c.time.maximumSteps = (long)h[11];
    const size_t N = (size_t)m.nx * m.ny, E = (size_t)EdgeCount(m) * 5;
    InitialState s;
    s.mesh = m;
    s.enthalpy.resize(N); s.composition.resize(N);
    EdgeVelocities v;
    v.solid.resize(E); v.darcy.resize(E);
    if (std::fread(s.enthalpy.data(), 8, N, f) != N || std::fread(s.composition.data(), 8, N, f) != N ||
        std::fread(v.solid.data(), 8, E, f) != E || std::fread(v.darcy.data(), 8, E, f) != E) return 2;
    std::fclose(f);

    std::vector<double> rH, rC;
    Rates rates;
    const int rs = RHS(c, s, v, rH, rC, rates);
    std::vector<StepRecord> hist;
    int calls = 0;
    const int st = AdvancePhaseCoupled(c, s, [&](const InitialState&, EdgeVelocities& out) { ++calls; out = v; return 0; },
                                       &hist);
    std::FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    const double head[5] = {(double)st, (double)rs, s.time, (double)s.acceptedSteps, (double)hist.size()};
    std::fwrite(head, 8, 5, o);
    rH.resize(N); rC.resize(N);
    std::fwrite(rH.data(), 8, N, o);
    std::fwrite(rC.data(), 8, N, o);
    std::fwrite(&rates.maximumRate, 8, 1, o);
    for (auto* a : {&s.enthalpy, &s.composition, &s.temperature, &s.porosity}) {
        a->resize(N);
        std::fwrite(a->data(), 8, N, o);
    }
    for (const auto& r : hist) {
        const double row[3] = {r.dt, (double)r.retries, r.courant};
        std::fwrite(row, 8, 3, o);
    }
    std::fclose(o);
    std::printf("status %d rhs %d steps %zu flow calls %d\n", st, rs, hist.size(), calls);
    return 0;
}

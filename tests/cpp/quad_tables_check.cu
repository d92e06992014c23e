// Test driver: the per-cell tables of general quad meshes built on the GPU
// (build_quad_cell_tables_gpu) against the host builder (build_quad_tables),
// bit for bit, on a perturbed 37x29 mesh, a 12-row slab of it and a
// sine-stretched 3x5 mesh (every boundary class). Exit status 0 = equal.
#include "quad_tables.hpp"
#include <cstdio>
#include <cstring>
#include <vector>
int main() {
    int bad_total = 0;
    for (int pass = 0; pass < 3; ++pass) {
        const int nx = pass == 2 ? 3 : 37, ny = pass == 2 ? 5 : 29;
        const int row0 = pass == 1 ? 5 : 0, rows = pass == 1 ? 12 : ny;
        std::vector<double> xy(2 * (size_t)(nx + 1) * (ny + 1));
        mp::mesh_vertices(nx, ny, 0, 0.5, 0, 1, pass == 2 ? 2 : 1, 0.22, 11, xy.data());
        mp::QuadTables h, g;
        int st = mp::build_quad_tables(nx, ny, xy.data(), 0, h, row0, rows, true);
        st |= mp::build_quad_tables(nx, ny, xy.data(), 0, g, row0, rows, false);
        const size_t N = (size_t)nx * rows;
        double *d_xy, *d_t;
        int* d_f;
        cudaMalloc(&d_xy, xy.size() * 8);
        cudaMalloc(&d_t, (size_t)(72 + 36 + 48 + 24 + 4) * N * 8);
        cudaMalloc(&d_f, 4);
        cudaMemcpy(d_xy, xy.data(), xy.size() * 8, cudaMemcpyHostToDevice);
        double* G0 = d_t; double* S9 = G0 + 72 * N; double* T4 = S9 + 36 * N; double* S4 = T4 + 48 * N; double* geo = S4 + 24 * N;
        int gs = mp::build_quad_cell_tables_gpu(nx, ny, d_xy, row0, rows, g.gq3, g.gw3, g.gq1, g.gw1, G0, S9, T4, S4, geo, d_f, 0);
        std::vector<double> all((size_t)(72 + 36 + 48 + 24 + 4) * N);
        cudaMemcpy(all.data(), d_t, all.size() * 8, cudaMemcpyDeviceToHost);
        const std::vector<double>* hv[5] = {&h.G0, &h.S9, &h.T4, &h.S4, &h.geo};
        const char* names[5] = {"G0", "S9", "T4", "S4", "geo"};
        size_t off = 0;
        for (int k = 0; k < 5; ++k) {
            int bad = 0;
            for (size_t i = 0; i < hv[k]->size(); ++i)
                if (std::memcmp(&(*hv[k])[i], &all[off + i], 8) != 0) ++bad;
            printf("pass %d %s: %zu values, %d differ\n", pass, names[k], hv[k]->size(), bad);
            bad_total += bad;
            off += hv[k]->size();
        }
        printf("pass %d status host %d gpu %d\n", pass, st, gs);
        cudaFree(d_xy); cudaFree(d_t); cudaFree(d_f);
    }
    printf("TOTAL DIFFERENT %d\n", bad_total);
    return bad_total != 0;
}

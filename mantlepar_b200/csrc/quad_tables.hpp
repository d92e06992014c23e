// Per-cell stage tables of a general (logically rectangular) quad mesh: the
// reference builds every cell's reconstruction from its own stencil geometry
// (TensorStencilPoly::Initialize, src/mlweno/tensorstencilpoly.cpp:146-231;
// SetTargetSmoothness :383-398; Reconstruction::Initialize,
// src/mlweno/reconstruction.cpp:109-210), so on a perturbed or stretched mesh
// each cell carries its own candidate matrices. They are built once on the
// host and kept in HBM as structure-of-arrays (entry k of cell c at
// k*ncell + c).
//
// Every candidate polynomial is re-expanded into the cell's own frame
// xi = (x - c_t)/h, c_t the average of the cell's corners, h = sqrt(area), so
// a limited evaluation anywhere is one Q2 polynomial in (xi, eta), monomial
// m = j*3 + i of xi^i eta^j:
//   3x3 candidate  D[m] = d00 [m == 0] + sum_{c=1..8} (d_c - d_0) G0[c-1][m]
//   2x2 candidate k  D[{0,1,3,4}][mm] += a0 [mm == 0] + sum_{c=1..3} (d_c - d_0) T4[k][c-1][mm]
// with d the stencil values minus the target value, and the smoothness forms
// folded to their upper triangles (entry (r, r) = S_rr, (r, c > r) = 2 S_rc).
#ifndef MP_QUAD_TABLES_HPP
#define MP_QUAD_TABLES_HPP

#include <cuda_runtime.h>

#include <vector>

namespace mp {

constexpr int kQG0 = 72;   // 8 differences x 9 monomials
constexpr int kQS9 = 36;   // folded 8x8
constexpr int kQT4 = 48;   // 4 candidates x 3 differences x 4 monomials
constexpr int kQS4 = 24;   // 4 candidates x folded 3x3
constexpr int kQGeo = 4;   // c_x, c_y, h, area

struct QuadTables {
    int nx = 0, ny = 0;
    std::vector<double> xy;        // vertices (nx+1)*(ny+1), x fastest, (x, y) pairs
    std::vector<double> G0, S9, T4, S4, geo;
    // Normal-line sample spacing of every edge at its 5 Gauss points in the
    // canonical point order (diffusiveflux.cpp:255-334, 4 samples, extent 0.9).
    std::vector<double> spacing;
    double gq[5], gw[5];           // Gauss rule on [-1, 1]
    double gq3[3], gw3[3], gq1, gw1;   // the moment / smoothness and area rules
    double dif_c_int[4], dif_c_bnd[5];
};

// Device pointers of a QuadTables (SoA per cell; spacing per edge and point)
// and the mesh-wide Gauss rule and derivative weights.
struct QuadDev {
    const double* xy;
    const double* G0;
    const double* S9;
    const double* T4;
    const double* S4;
    const double* geo;
    const double* sp;
    double gq[5], gw[5];
    double dif_c_int[4], dif_c_bnd[5];
};

// Vertices of the reference's mesh families (src/core/mesh.cpp:27-55):
// 0 rectangular, 1 perturbed quadrilateral (interior vertices displaced by
// perturbation * spacing * SplitMix64 noise keyed by seed), 2 sine-stretched.
// Returns 0 or an mp_status.
int mesh_vertices(int nx, int ny, double x0, double x1, double y0, double y1, int family, double perturbation,
                  unsigned long long seed, double* xy);

// Quad validity of every cell (src/core/quad_validation.h): finite corners,
// positive extents, positive scaled corner Jacobians. Returns 0 or
// MP_ERR_ARG_WRONG with the first bad cell in *bad.
int validate_quads(int nx, int ny, const double* xy, long long* bad);

// Build the tables on `threads` host threads (0 = all): of the whole nx x ny
// mesh, or (rows >= 0) of its rows [row0, row0 + rows) in local numbering,
// each cell's stencil taken from the whole mesh. cell_tables = false leaves
// the per-cell arrays (G0, S9, T4, S4, geo) empty: the vertices, the edge
// spacing, the rules and weights only. Returns 0 or an mp_status.
int build_quad_tables(int nx, int ny, const double* xy, int threads, QuadTables& t, int row0 = 0, int rows = -1,
                      bool cell_tables = true);

// The per-cell arrays of the same tables (identical values: the host
// builder's arithmetic without FMA contraction) on the GPU, written into the
// device arrays of ncell = nx * rows cells (layout as QuadTables); d_xy holds
// the whole mesh's vertices; d_failed is one device int of scratch.
// Synchronous on `stream`. Returns 0, MP_ERR_ARG_WRONG (a singular stencil
// or a cell without positive area) or MP_ERR_CUDA.
int build_quad_cell_tables_gpu(int nx, int ny, const double* d_xy, int row0, int rows, const double* gq3,
                               const double* gw3, double gq1, double gw1, double* G0, double* S9, double* T4,
                               double* S4, double* geo, int* d_failed, cudaStream_t stream);

// One device allocation *buf (cudaMalloc; the caller frees it, after a
// failure too) holding the tables of local rows [row0, row0 + rows) of a
// general quad mesh: the vertices and edge spacing of qt (built with
// cell_tables = false) copied from the host, and the per-cell arrays built
// on the GPU from the whole mesh's vertices xy (host memory). Fills q with
// the device pointers, the rules and the derivative weights. Synchronous on
// `stream`. Returns 0, MP_ERR_ARG_WRONG (a singular stencil or a cell
// without positive area) or MP_ERR_CUDA with the CUDA error in *cuda_err.
int upload_quad_tables(int nx, int ny, const double* xy, const QuadTables& qt, int row0, int rows,
                       cudaStream_t stream, double** buf, QuadDev& q, cudaError_t* cuda_err);

}  // namespace mp

#endif

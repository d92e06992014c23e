// Per-mesh tables of the uniform-mesh ML-WENO stage (host-built; the
// kernels read them as a kernel parameter or from global memory).
//
// On a uniform rectangular mesh every interior cell has the same stencil
// geometry up to a translation, so the reference's per-cell setup
// (TensorStencilPoly::Initialize, src/mlweno/tensorstencilpoly.cpp:146-231;
// SetTargetSmoothness :383-398; Reconstruction::Initialize,
// src/mlweno/reconstruction.cpp:109-210; the limiter point set,
// src/couple/state_reconstruction.cpp:152-168; diffusion sample geometry,
// src/mlweno/diffusiveflux.cpp:255-334) collapses to one table set per
// mesh, with nine boundary classes (left/interior/right x bottom/interior/top)
// for the candidate mask and the limiter points. All coordinates are in the
// target cell's normalised frame xi = (x - x_c)/h, h = sqrt(cell area).
#ifndef MP_TABLES_HPP
#define MP_TABLES_HPP

namespace mp {

constexpr int kMaxPoints = 1024;   // limiter points over all 9 classes
constexpr int kNQ = 5;             // Gauss points per edge / per cell axis
constexpr int kMaxLines = 256;     // limiter point lines over all 9 classes

// The fields the stage kernels read. Small enough (~4.5 KB) to travel as a
// kernel parameter, so that table coefficients become constant-bank operands
// of the FP64 instructions instead of loads.
struct StageHot {
    // 3x3 candidate (order 2): basis coefficients C9[cell][monomial]
    // (monomial m = j*3 + i for xi^i eta^j) and the reference-square
    // smoothness matrix on the differences to stencil cell 0 (rows/cols 1..8).
    double C9[9][9];
    double S9[8][8];
    // 2x2 candidates (order 1) in the stencil's own frame (centre = the shared
    // vertex): coefficients and the target-cell smoothness matrix for target
    // position t = tj*2 + ti (rows/cols 1..3 of the difference form).
    double C4[4][4];
    double S4[4][3][3];
    // The same forms folded to their upper triangles, row by row: entry
    // (r, r) is S_rr, entry (r, c > r) is 2 S_rc, so d^T S d is one FMA
    // chain per row.
    double SF9[36];
    double SF4[4][6];
    double X, Y;            // half cell extents in the normalised frame
    double epsA;            // epsilon * cell area of the weight regulariser
    double area;            // cell area (1-point rule, as MeshInfo::CacheAreas)
    double len_h, len_v;    // lengths of AlongI (horizontal) / AlongJ edges
    double gw[kNQ];         // Gauss weights
    double cw[kNQ * kNQ];   // cell-quadrature weight / area, q = b*5 + a
    double gx[kNQ];         // X * g_q
    double gy[kNQ];         // Y * g_q
    // Thermal diffusion by normal-line sampling (diffusiveflux.cpp:203-334)
    // with 4 samples per Gauss point and extent fraction 0.9, for this mesh:
    // derivative weights (interior: middle of 4 nodes; wall: end of 5 nodes),
    // physical spacing [horizontal/vertical edges][interior/wall], physical
    // Gauss weights len*w_q/2 [horizontal/vertical][q], and the coordinate
    // across the edge of each sample in its cell's normalised frame: interior
    // samples k = 0, 1 lie in the left cell, 2, 3 in the right one
    // [horizontal/vertical][k]; wall samples k = 0..3 lie in the wall cell,
    // farthest first [wall: bottom, top, left, right][k].
    double dif_c_int[4];
    double dif_c_bnd[5];
    double dif_ds[2][2];
    double dif_w[2][kNQ];
    double dif_pos_int[2][4];
    double dif_pos_bnd[4][4];
    // Physical height of a point: y = y0 + (row + 0.5) * dy + eta * hn (global
    // row; hn = sqrt(cell area) normalises the reconstruction frame), and the
    // physical cell-quadrature weights w_a w_b |J| (q = b*5 + a).
    double y0, dy, hn;
    double cwp[kNQ * kNQ];
    // With every deviation coefficient below this magnitude, every limiter
    // value is finite (in FP32 too): 1e36 / (16 max(1, X^2) max(1, Y^2)),
    // the points lying within |xi| <= X, |eta| <= Y.
    double scan_guard;
    // Limiter points grouped into 5-point lines: apart from the cell centre,
    // every limiter point lies on a row eta = line_c with xi = X*g_q, or on a
    // column xi = line_c with eta = Y*g_q (q = 0..4). Class c owns lines
    // [line_off[c], line_off[c+1]); line_dir 0 = row, 1 = column; line_kind
    // 1 = diffusion samples.
    int line_off[10];
    double line_c[kMaxLines];
    unsigned char line_dir[kMaxLines];
    unsigned char line_kind[kMaxLines];
};

struct StageTables : StageHot {
    double gq[kNQ];         // Gauss points on [-1,1]
    // Limiter points of class c in [pt_off[c], pt_off[c+1]); pt_kind 1 marks
    // a diffusion sample point (checked for admissibility in the stage).
    int pt_off[10];
    double pt_x[kMaxPoints];
    double pt_y[kMaxPoints];
    unsigned char pt_kind[kMaxPoints];
};

// Build the tables of an nx x ny uniform mesh on [x0,x1] x [y0,y1].
// Returns 0 or an mp_status code (stencil solve failure).
int build_stage_tables(int nx, int ny, double x0, double x1, double y0, double y1, StageTables& t);

}  // namespace mp

#endif

// Serial stand-ins linked with the reference's own sources in oracle/_ref.
// TEST INFRASTRUCTURE ONLY.
//  - PetscDTGaussQuadrature (PETSc 3.23+, not vendored): Gauss-Legendre by
//    Newton iteration on P_n (oracle/restated.hpp gauss_rule).
//  - LAPACKE_dgesv (not vendored): partial-pivot LU (oracle/restated.hpp).
//  - MeshInfo (src/core/mesh_info.h): the subset of its methods that the
//    reference's TensorStencilPoly/Reconstruction call, over a plain vertex
//    array instead of a PETSc DMDA (src/core/mesh_info.cpp is DMDA-bound).
#include "mesh_info.h"
#include "petscdt.h"
#include "lapacke.h"

#include "../restated.hpp"

#include <algorithm>
#include <vector>

struct mp_shim_dm {
    PetscInt M = 0, N = 0;            // vertex counts
    std::vector<Point> xy;            // (j*M + i)
};

PetscErrorCode PetscDTGaussQuadrature(PetscInt n, PetscReal a, PetscReal b, PetscReal* x, PetscReal* w) {
    if (n < 1 || a != -1.0 || b != 1.0) return PETSC_ERR_ARG_OUTOFRANGE;
    std::vector<double> p, q;
    orc::gauss_rule((int)n, p, q);
    for (PetscInt k = 0; k < n; ++k) { x[k] = p[k]; w[k] = q[k]; }
    return PETSC_SUCCESS;
}

lapack_int LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double* a, lapack_int lda,
                         lapack_int* ipiv, double* b, lapack_int ldb) {
    if (layout != LAPACK_ROW_MAJOR || nrhs != n || lda != n || ldb != n) return -1;
    std::vector<double> A(a, a + (size_t)n * n), B(b, b + (size_t)n * n);
    try { orc::lu_solve(n, A, B); } catch (const orc::Error&) { return 1; }
    std::copy(B.begin(), B.end(), b);
    for (lapack_int k = 0; k < n; ++k) ipiv[k] = k + 1;
    return 0;
}

void MeshInfo::Swap(MeshInfo& o) noexcept {
    std::swap(initialized_, o.initialized_);
    std::swap(vertices_, o.vertices_); std::swap(cells_, o.cells_);
    std::swap(vertexCount_, o.vertexCount_); std::swap(cellCount_, o.cellCount_);
    std::swap(iEdges_, o.iEdges_); std::swap(jEdges_, o.jEdges_); std::swap(width_, o.width_);
    std::swap(ownedVertices_, o.ownedVertices_); std::swap(ghostVertices_, o.ghostVertices_);
    std::swap(ownedCells_, o.ownedCells_); std::swap(availableCells_, o.availableCells_);
    coordinates_.swap(o.coordinates_); areas_.swap(o.areas_); ownedEdgeIds_.swap(o.ownedEdgeIds_);
}
MeshInfo::MeshInfo(MeshInfo&& o) noexcept { Swap(o); }
MeshInfo& MeshInfo::operator=(MeshInfo&& o) noexcept { if (this != &o) { MeshInfo w(std::move(o)); Swap(w); } return *this; }

bool MeshInfo::ContainsCell(MeshIndex c) const noexcept {
    return c.i >= 0 && c.j >= 0 && c.i < cells_.i && c.j < cells_.j;
}

PetscErrorCode MeshInfo::GetCellCorners(MeshIndex c, QuadVertices& q) const {
    PetscCheck(HasCell(c), PETSC_COMM_SELF, PETSC_ERR_ARG_OUTOFRANGE, "cell unavailable");
    const PetscInt M = vertices_.i;
    q[0] = coordinates_[(size_t)(c.j * M + c.i)];
    q[1] = coordinates_[(size_t)(c.j * M + c.i + 1)];
    q[2] = coordinates_[(size_t)((c.j + 1) * M + c.i + 1)];
    q[3] = coordinates_[(size_t)((c.j + 1) * M + c.i)];
    return PETSC_SUCCESS;
}

PetscErrorCode MeshInfo::GetCellArea(MeshIndex c, PetscReal& a) const {
    PetscCheck(HasCell(c), PETSC_COMM_SELF, PETSC_ERR_ARG_OUTOFRANGE, "cell unavailable");
    a = areas_[(size_t)(c.j * cells_.i + c.i)];
    return PETSC_SUCCESS;
}

// Same 1-point rule as the reference's MeshInfo::CacheAreas.
PetscErrorCode MeshInfo::CacheAreas() {
    GaussRule1D rule;
    PetscCall(CreateGaussRule(1, rule));
    areas_.assign((size_t)cellCount_, 0.0);
    for (PetscInt j = 0; j < cells_.j; ++j)
        for (PetscInt i = 0; i < cells_.i; ++i) {
            QuadVertices q;
            PetscCall(GetCellCorners({i, j}, q));
            PetscReal a;
            PetscCall(IntegrateCell(q, rule, [](const Point&) { return PetscReal(1); }, a));
            areas_[(size_t)(j * cells_.i + i)] = a;
        }
    return PETSC_SUCCESS;
}

PetscErrorCode BuildMeshInfo(DM dm, Vec, MeshInfo& info) {
    MeshInfo w;
    w.initialized_ = true;
    w.vertices_ = {dm->M, dm->N};
    w.cells_ = {dm->M - 1, dm->N - 1};
    w.vertexCount_ = dm->M * dm->N;
    w.cellCount_ = (dm->M - 1) * (dm->N - 1);
    w.iEdges_ = (dm->M - 1) * dm->N;
    w.jEdges_ = dm->M * (dm->N - 1);
    w.width_ = 3;
    w.ownedVertices_ = w.ghostVertices_ = MeshRange{{0, 0}, {dm->M, dm->N}};
    w.ownedCells_ = w.availableCells_ = MeshRange{{0, 0}, {dm->M - 1, dm->N - 1}};
    w.coordinates_ = dm->xy;
    PetscCall(w.CacheAreas());
    info = std::move(w);
    return PETSC_SUCCESS;
}

// Helper for the reference backend: build the plain-array DM.
DM mp_shim_make_dm(PetscInt M, PetscInt N, const double* xy) {
    DM dm = new mp_shim_dm;
    dm->M = M; dm->N = N;
    dm->xy.resize((size_t)(M * N));
    for (size_t k = 0; k < dm->xy.size(); ++k) { dm->xy[k].p[0] = xy[2 * k]; dm->xy[k].p[1] = xy[2 * k + 1]; }
    return dm;
}
void mp_shim_free_dm(DM dm) { delete dm; }

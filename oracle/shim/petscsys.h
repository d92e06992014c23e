/* Serial stand-in for the subset of PETSc's petscsys.h used by the
 * reference's src/core/integral.*, src/mlweno/{tensorstencilpoly,
 * reconstruction,diffusiveflux,advectiveflux}.* (TEST INFRASTRUCTURE: lets the oracle
 * compile those reference sources unmodified into oracle/_ref). Error
 * macros return the PETSc error class; no messages, no MPI. */
#ifndef MP_SHIM_PETSCSYS_H
#define MP_SHIM_PETSCSYS_H
#include <cmath>
#include <cfloat>
#include <cstdint>
typedef int PetscErrorCode;
typedef long long PetscInt;
typedef double PetscReal;
typedef double PetscScalar;
typedef int PetscMPIInt;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef int MPI_Comm;
#define MPI_COMM_NULL 0
#define PETSC_COMM_SELF 1
#define PETSC_COMM_WORLD 2
#define PETSC_SUCCESS 0
#define PETSC_ERR_ARG_SIZ 60
#define PETSC_ERR_ARG_WRONG 62
#define PETSC_ERR_ARG_OUTOFRANGE 63
#define PETSC_ERR_ARG_WRONGSTATE 73
#define PETSC_ERR_FP 72
#define PETSC_ERR_LIB 76
#define PETSC_ERR_PLIB 77
#define PETSC_ERR_USER 83
#define PETSC_ERR_NOT_CONVERGED 91
#define PETSC_MACHINE_EPSILON DBL_EPSILON
#define PETSC_PI 3.14159265358979323846
#define PetscInt_FMT "lld"
#define PetscFunctionBeginUser do {} while (0)
#define PetscFunctionReturn(x) return (x)
#define PetscCall(x) do { PetscErrorCode mp_shim_e_ = (x); if (mp_shim_e_) return mp_shim_e_; } while (0)
#define PetscCheck(cond, comm, code, ...) do { if (!(cond)) return (code); } while (0)
#define SETERRQ(comm, code, ...) return (code)
#define PetscIsInfOrNanReal(x) (!std::isfinite((double)(x)))
#define PetscAbsReal(x) std::fabs(x)
#define PetscSqrtReal(x) std::sqrt(x)
#define PetscSinReal(x) std::sin(x)
#define PetscRealPart(x) (x)
/* One rank: an all-reduce of local values returns them unchanged (used by
 * ReduceGlobalLaxFriedrichsSpeed in src/mlweno/advectiveflux.cpp). */
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_INT 1
#define MPIU_REAL 2
#define MPI_MAX 1
inline int MPI_Allreduce(const void* in, void* out, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
    const unsigned char* a = static_cast<const unsigned char*>(in);
    unsigned char* b = static_cast<unsigned char*>(out);
    const int size = type == MPI_INT ? (int)sizeof(int) : (int)sizeof(double);
    for (int k = 0; k < count * size; ++k) b[k] = a[k];
    return 0;
}
#define PetscCallMPI(x) do { if ((x) != 0) return PETSC_ERR_LIB; } while (0)
#endif

/* Serial stand-in for petscdt.h (TEST INFRASTRUCTURE). */
#ifndef MP_SHIM_PETSCDT_H
#define MP_SHIM_PETSCDT_H
#include "petscsys.h"
PetscErrorCode PetscDTGaussQuadrature(PetscInt n, PetscReal a, PetscReal b, PetscReal* x, PetscReal* w);
#endif

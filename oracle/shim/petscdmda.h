/* Serial stand-in for petscdmda.h: opaque DM/Vec handles only (TEST INFRASTRUCTURE). */
#ifndef MP_SHIM_PETSCDMDA_H
#define MP_SHIM_PETSCDMDA_H
#include "petscsys.h"
typedef struct mp_shim_dm* DM;
typedef struct mp_shim_vec* Vec;
#endif

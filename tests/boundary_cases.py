"""Coupled-transport cases with flow through the walls, shared by the oracle
tests and the GPU parity tests: the synthetic streamfunction flow plus a
uniform upward through-flow of the solid (inflow at the bottom wall, outflow
at the top), so the advection boundary policy of every wall point is taken
(EvaluateAdvectionBoundary, src/couple/initialization.cpp:469-489), with the
global Lax-Friedrichs speed (src/couple/evolve.cpp:292-329) and a nonzero
Darcy exponent (PhaseTransportVelocities, evolve.cpp:36-52) as variants, and
one configuration the reference rejects (an outflow-only enthalpy policy on
a wall with inflow)."""
from __future__ import annotations

import numpy as np

from mantlepar_b200 import synthetic as sy

W = sy.Workload(nx=20, ny=20, seed=3)
THROUGH = 0.05

# name -> (transport options, expected status of the stage: 0 or the
# reference's error class, PETSC_ERR_ARG_OUTOFRANGE = 63)
CASES = {
    "inflow_outflow": (dict(inflow_H=0.6, inflow_C=0.31), 0),
    "darcy_exponent_2": (dict(inflow_H=0.6, inflow_C=0.31, theta=2.0), 0),
    "global_lf": (dict(inflow_H=0.6, inflow_C=0.31, lf_global=1, lf_global_speed=1.0), 0),
    "zero_flux_C": (dict(inflow_H=0.6, inflow_C=0.31, C_policy=2), 0),
    "outflow_H_at_inflow": (dict(inflow_H=0.6, inflow_C=0.31, H_policy=1), 63),
}


def face_velocity(w: sy.Workload = W, through: float = THROUGH):
    """The synthetic flow plus `through` on every horizontal edge (normal +y)."""
    vs, ud = sy.face_velocity(w)
    vs = vs.copy()
    vs[: w.nx * (w.ny + 1) * 5] += through
    return vs, ud

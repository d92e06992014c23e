"""GPU parity at the full size of the headline workload: 1280x2560 uniform
quads, the bench's seeded construction (seed 1), SSPRK3 at CFL 0.4.

The reference build (oracle/_ref: the reference's own reconstruction,
stencil, flux, integral and phase sources under the restated driver) runs
on every host thread and is compared cell by cell with the CUDA path through
the C ABI:

* the limiter factors theta_H, theta_C of the initial state;
* one stage L(U^n): T, phi, rate per cell, rhsH / rhsC against their
  infinity norm, and the stage totals;
* one accepted SSPRK3 step: dt, retries, H, C, T, phi.

Bar: 1e-12 per cell, |x - ref| / max(|ref|, 1e-3 max|ref|), as for the small
golden cases. The oracle takes a few minutes here (about 3.3 M cells).
"""
import os

import numpy as np
import pytest

from mantlepar_b200 import synthetic as sy

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * max(np.max(np.abs(b)), 1e-300))))


def rel_inf(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_headline_workload_stage_and_step_match_reference_build(cuda_lib):
    from oracle import pyoracle as po
    from mantlepar_b200.transport import Transport, TransportConfig
    lib = po.reference() if po.reference_available() else po.restated()
    w = sy.Workload(nx=1280, ny=2560)
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)

    gpu = Transport(w, TransportConfig(cfl=w.cfl, integrator=3))
    gpu.set_face_velocity(vs, ud)
    gpu.set_state(H, C)
    g_th = gpu.limiter()
    g_rhs = gpu.rhs()
    _, g_rep = gpu.step(1)
    g_state = gpu.get_state()
    gpu.close()

    ref = po.TransportOracle(sy.material_s(), w, lib=lib, integrator=3, threads=os.cpu_count() or 1)
    ref.set_face_velocity(vs, ud)
    ref.set_state(H, C)
    code, r_thH, r_thC = ref.limiter()
    assert code == 0
    code, r_rhs = ref.rhs()
    assert code == 0
    code, r_rep = ref.step(1)
    assert code == 0
    r_state = ref.get_state()
    ref.close()

    errs = {"thetaH": rel(g_th[0], r_thH), "thetaC": rel(g_th[1], r_thC)}
    for k in ("T", "phi", "rate"):
        errs[k] = rel(g_rhs[k], r_rhs[k])
    for k in ("rhsH", "rhsC"):
        errs[k] = rel_inf(g_rhs[k], r_rhs[k])
    errs["maxRate"] = abs(g_rhs["maxRate"] - r_rhs["maxRate"]) / r_rhs["maxRate"]
    errs["boundaryH"] = abs(g_rhs["boundaryH"] - r_rhs["boundaryH"]) / max(1.0, abs(r_rhs["boundaryH"]))
    assert g_rep[0]["retries"] == r_rep[0]["retries"]
    errs["dt"] = abs(g_rep[0]["dt"] - r_rep[0]["dt"]) / r_rep[0]["dt"]
    for name, a, b in zip(("H", "C", "T", "phi"), g_state, r_state):
        errs["step_" + name] = rel(a, b)
    print("1280x2560 per-cell errors vs", "reference build" if lib is po.reference() else "restated oracle",
          {k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if not v <= RTOL}
    assert not bad, bad

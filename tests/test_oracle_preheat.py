"""The preheat oracle (src/couple/preheat.cpp restated) against the golden
fixtures of the reference-backed build and against that build directly."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
import preheat_cases as pc

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "preheat_golden.npz"))
ROW_FIELDS = ["step", "time", "dt", "courant", "integral", "minimum", "maximum", "boundaryFlux", "balanceError"]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


@pytest.mark.parametrize("name", list(pc.CASES))
def test_restated_preheat_equals_golden_bitwise(name):
    r = pc.oracle_run(pc.CASES[name])
    assert (r["begin"], r["rhs_code"], r["run"], r["diag"]) == (0, 0, 0, 0)
    for k in ["rate", "rhs", "H", "T", "phi"]:
        assert np.array_equal(bits(r[k]), bits(GOLDEN[f"{name}_{k}"])), k
    assert np.array_equal(bits([r["limit"], r["bflux"]]), bits(GOLDEN[f"{name}_scalars"]))
    rows = np.array([[row[f] for f in ROW_FIELDS] for row in [r["first"]] + r["rows"]])
    assert np.array_equal(bits(rows), bits(GOLDEN[f"{name}_rows"]))


@pytest.mark.skipif(not po.reference_available(), reason="reference-backed oracle not built")
def test_restated_preheat_equals_reference_outflow_only_walls():
    """Outflow-only advection walls with heat leaving through the bottom wall
    (IntegrateAdvectiveBoundaryFlux's extrapolated state) and a lithostatic
    pressure in the diagnostics, checked against the reference's own
    functions directly."""
    case = pc.PreheatCase(pc.sy.Workload(nx=6, ny=11, seed=21, noise_H=0.08), bottom_outflow=0.2, kappa=5e-4,
                          H_policy=1, thermal_type=(1, 0, 2, 2), thermal_value=(0.4, 0.0, 0.01, -0.01),
                          pressure_model=1, end=0.02)
    a, b = pc.oracle_run(case), pc.oracle_run(case, po.reference())
    assert a["run"] == 0 and len(a["rows"]) > 2
    for k in ["rate", "rhs", "H", "T", "phi"]:
        assert np.array_equal(bits(a[k]), bits(b[k])), k
    assert a["rows"] == b["rows"] and a["bflux"] == b["bflux"] and a["bflux"] > 0


def test_preheat_heat_balance_and_courant():
    """Each accepted step satisfies the reference's balance check
    (preheat.cpp:270-273) and courant = dt * max rate <= cfl."""
    for case in pc.CASES.values():
        r = pc.oracle_run(case)
        prev = r["first"]["integral"]
        for row in r["rows"]:
            tol = 1e-10 * (1 + abs(row["integral"]) + abs(prev) + abs(row["dt"] * row["boundaryFlux"]))
            assert abs(row["integral"] - prev + row["dt"] * row["boundaryFlux"]) <= tol
            assert row["courant"] <= case.cfl * (1 + 1e-12)
            prev = row["integral"]
        assert r["rows"][-1]["time"] == case.end


def test_closed_box_conserves_heat():
    r = pc.oracle_run(pc.CASES["closed"])
    assert r["bflux"] == 0.0
    assert abs(r["rows"][-1]["integral"] - r["first"]["integral"]) < 1e-14


def _codes(**kw):
    case = pc.PreheatCase(pc.sy.Workload(nx=6, ny=6, seed=2), **kw)
    return pc.oracle_run(case)


def test_preheat_failures():
    """The reference's failure classes (preheat.cpp:237-266; EvaluateAdvectionBoundary)."""
    # Backflow through an outflow-only wall: PETSC_ERR_ARG_OUTOFRANGE at the first RHS.
    r = _codes(through=0.3, H_policy=1)
    assert r["rhs_code"] == 63 and r["run"] == 63 and r["rows"] == []
    # A fixed step above the rate limit.
    r = _codes(control=1, dt_initial=1.0, end=2.0)
    assert r["begin"] == 0 and r["run"] == 63 and r["rows"] == []
    # maximumSteps before time.end: NOT_CONVERGED after the allowed steps.
    r = _codes(max_steps=3, end=1.0, dt_max=1e-3)
    assert r["run"] == 91 and len(r["rows"]) == 3
    # State time after time.end.
    r = _codes(end=-1.0)
    assert r["begin"] == 63
    # A global LF speed below a flow normal speed.
    r = _codes(through=0.3, lf_global=1, lf_global_speed=0.01)
    assert r["begin"] == 63


# Linear exactness: every candidate polynomial reproduces linear data, so the
# unlimited reconstruction of a linear H is exact, the traces of both sides
# agree and the linear-law flux of the uniform flow v integrates exactly:
# the preheat RHS is -v . grad H in every cell not on an inflow wall (the
# bottom and left walls for v = (0.3, 0.2)), on any quad mesh.
LINEAR_H = (0.7, 0.5, -0.3)           # c + a x + b y
LINEAR_V = (0.3, 0.2)
LINEAR_RHS = -(LINEAR_V[0] * LINEAR_H[1] + LINEAR_V[1] * LINEAR_H[2])


def linear_field_case(w, family):
    case = pc.PreheatCase(w, family=family, perturbation=0.2)
    xy = pc.sy.quad_vertices(w, family, 0.2, case.mesh_seed)
    x, y = pc.sy.cell_centroids(w, xy)
    H = LINEAR_H[0] + LINEAR_H[1] * x + LINEAR_H[2] * y
    return case, xy, pc.sy.uniform_face_velocity(w, xy, *LINEAR_V), H


@pytest.mark.parametrize("family", [0, 1, 2], ids=["uniform", "perturbed", "sine"])
def test_linear_field_gives_the_exact_rhs(family):
    w = pc.sy.Workload(nx=12, ny=10)
    case, xy, vs, H = linear_field_case(w, family)
    out = []
    for lib in [None] + ([po.reference()] if po.reference_available() else []):
        t = pc.oracle_instance(case, lib)
        t.set_face_velocity(vs, np.zeros_like(vs))
        t.set_state(H, np.full(w.cells, 0.3))
        code, rhs, _ = t.preheat_rhs()
        assert code == 0
        out.append(rhs)
    r = out[0].reshape(w.ny, w.nx)
    assert np.max(np.abs(r[1:, 1:] - LINEAR_RHS)) <= 1e-13
    assert np.max(np.abs(r[0])) > 1e-3          # the inflow wall's cells see the inflow value
    if len(out) == 2:
        assert np.array_equal(bits(out[0]), bits(out[1]))

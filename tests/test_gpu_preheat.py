"""GPU parity of the legacy dry preheat (src/couple/preheat.cpp) against the
reference-backed golden runs and the oracle.

Bars (FP64 kernels against the reference's 80-bit long double internals):
per-cell relative error 1e-12 for the rate, the final H and the diagnostic
T and phi (|x - ref| / max(|ref|, 1e-3 max|ref|)); the RHS, a signed sum of
face fluxes, against its infinity norm (1e-12); step sizes, integrals and
extrema of every history row 1e-12 relative (the boundary flux 1e-12 of
max(1, |ref|)); failure statuses equal.
"""
import os

import numpy as np
import pytest

from mantlepar_b200 import synthetic as sy
import preheat_cases as pc

pytestmark = pytest.mark.gpu

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "preheat_golden.npz"))
ROW_FIELDS = ["step", "time", "dt", "courant", "integral", "minimum", "maximum", "boundaryFlux", "balanceError"]
RTOL = 1e-12


def rel(a, b):
    b = np.asarray(b)
    return np.max(np.abs(np.asarray(a) - b) / np.maximum(np.abs(b), 1e-3 * max(np.max(np.abs(b)), 1e-300)))


def rel_inf(a, b):
    b = np.asarray(b)
    return np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300)


def check_rows(rows, ref):
    """rows: list of dicts (first row included); ref: golden row matrix."""
    assert len(rows) == len(ref)
    for row, r in zip(rows, ref):
        want = dict(zip(ROW_FIELDS, r))
        assert row["step"] == want["step"]
        for k in ["time", "dt", "courant", "integral", "minimum", "maximum"]:
            assert abs(row[k] - want[k]) <= RTOL * max(abs(want[k]), 1e-300), (k, row[k], want[k])
        assert abs(row["boundaryFlux"] - want["boundaryFlux"]) <= RTOL * max(1.0, abs(want["boundaryFlux"]))


@pytest.mark.parametrize("name", list(pc.CASES))
def test_preheat_matches_reference(cuda_lib, name):
    case = pc.CASES[name]
    p = pc.gpu_instance(case)
    rate, limit, first = p.begin()
    assert rel(rate, GOLDEN[f"{name}_rate"]) <= RTOL
    lim_ref, bflux_ref = GOLDEN[f"{name}_scalars"]
    assert abs(limit - lim_ref) <= RTOL * lim_ref
    rhs, bflux = p.rhs()
    assert rel_inf(rhs, GOLDEN[f"{name}_rhs"]) <= RTOL
    assert abs(bflux - bflux_ref) <= RTOL * max(1.0, abs(bflux_ref))
    code, rows = p.advance(10000)
    assert code == 0
    check_rows([first] + rows, GOLDEN[f"{name}_rows"])
    H, time, accepted = p.get_state()
    assert time == case.end and accepted == len(rows)
    assert rel(H, GOLDEN[f"{name}_H"]) <= RTOL
    T, phi = p.diagnostics()
    assert rel(T, GOLDEN[f"{name}_T"]) <= RTOL
    assert rel(phi, GOLDEN[f"{name}_phi"]) <= RTOL if np.max(GOLDEN[f"{name}_phi"]) > 0 else np.all(phi == 0)


def test_preheat_run_report(cuda_lib):
    """mp_preheat_run: AdvanceLegacyPreheat's report and history in one call."""
    case = pc.CASES["through_diffusion"]
    p = pc.gpu_instance(case)
    code, rep, rows, T, phi = p.run()
    assert code == 0
    ref = GOLDEN["through_diffusion_rows"]
    check_rows(rows, ref)
    assert rep["initialTime"] == 0.0 and rep["finalTime"] == case.end
    assert abs(rep["finalIntegral"] - ref[-1][4]) <= RTOL * abs(ref[-1][4])
    bint = sum(r["dt"] * r["boundaryFlux"] for r in rows[1:])
    assert abs(rep["boundaryIntegral"] - bint) <= 1e-14
    assert rel(T, GOLDEN["through_diffusion_T"]) <= RTOL


def test_preheat_long_run_crosses_batches(cuda_lib):
    """More steps than one device batch (512): the device-side step chain
    continues across host round trips; every row matches the oracle."""
    case = pc.PreheatCase(sy.Workload(nx=16, ny=12, seed=4), through=0.05, kappa=1e-3,
                          thermal_type=(1, 1, 0, 0), thermal_value=(1.0, 0.2, 0.0, 0.0), dt_max=2e-4, end=0.15)
    ref = pc.oracle_run(case)
    assert ref["run"] == 0 and len(ref["rows"]) > 700
    p = pc.gpu_instance(case)
    _, _, first = p.begin()
    code, rows = p.advance(100000)
    assert code == 0
    check_rows([first] + rows, np.array([[r[f] for f in ROW_FIELDS] for r in [ref["first"]] + ref["rows"]]))
    H, _, _ = p.get_state()
    assert rel(H, ref["H"]) <= 1e-11


def test_preheat_advance_in_pieces(cuda_lib):
    """advance(n) in pieces reproduces one advance to time.end."""
    case = pc.CASES["closed"]
    a = pc.gpu_instance(case)
    a.begin()
    _, ra = a.advance(1000)
    b = pc.gpu_instance(case)
    b.begin()
    rb = []
    while True:
        code, got = b.advance(2)
        assert code == 0
        rb += got
        if len(got) < 2:
            break
    assert ra == rb
    assert np.array_equal(a.get_state()[0], b.get_state()[0])


def _failure(**kw):
    kw.setdefault("family", sy.MESH_RECTANGULAR)
    if kw["family"] != sy.MESH_RECTANGULAR:
        kw.setdefault("perturbation", 0.2)
    case = pc.PreheatCase(sy.Workload(nx=6, ny=6, seed=2), **kw)
    ref = pc.oracle_run(case)
    p = pc.gpu_instance(case)
    from mantlepar_b200._capi import MPError
    out = {}
    try:
        p.begin()
        out["begin"] = 0
    except MPError as e:
        out["begin"] = e.code
        return ref, out, p
    code, rows = p.advance(100000, raise_on_error=False)
    out["run"], out["rows"] = code, rows
    return ref, out, p


@pytest.mark.parametrize("family", [sy.MESH_RECTANGULAR, sy.MESH_PERTURBED], ids=["uniform", "perturbed"])
def test_preheat_failures_match_reference(cuda_lib, family):
    # Backflow through an outflow-only wall.
    ref, out, _ = _failure(through=0.3, H_policy=1, family=family)
    assert out["run"] == ref["run"] == 63 and out["rows"] == []
    # A fixed step above the rate limit.
    ref, out, _ = _failure(control=1, dt_initial=1.0, end=2.0, family=family)
    assert out["run"] == ref["run"] == 63
    # maximumSteps: the allowed steps are kept, then NOT_CONVERGED.
    ref, out, p = _failure(max_steps=3, end=1.0, dt_max=1e-3, family=family)
    assert out["run"] == ref["run"] == 91 and len(out["rows"]) == 3
    H, time, accepted = p.get_state()
    assert accepted == 3 and abs(time - ref["rows"][-1]["time"]) <= 1e-15
    assert rel(H, ref["H"]) <= RTOL
    # State time after time.end; a global LF speed below a flow speed.
    assert _failure(end=-1.0, family=family)[1]["begin"] == 63
    assert _failure(through=0.3, lf_global=1, lf_global_speed=0.01, family=family)[1]["begin"] == 63


def test_preheat_rejected_candidate_keeps_state(cuda_lib):
    """A non-finite candidate is rejected on the device (preheat.cpp:268-269):
    no row, the state and clock stay at the last accepted step. The state is
    finite but so large that H + dt*rhs overflows."""
    case = pc.PreheatCase(sy.Workload(nx=8, ny=8, seed=2), through=0.2, end=0.05)
    p = pc.gpu_instance(case)
    H, C = case.state()
    H = H * 1e306
    p.set_state(H, C)
    p.begin()
    code, rows = p.advance(100, raise_on_error=False)
    t = pc.oracle_instance(case)
    t.set_state(H, C)
    t.preheat_begin()
    ref_code, ref_rows = t.preheat_advance(100)
    assert code == ref_code and code in (63, 72) and len(rows) == len(ref_rows)
    H1, time, accepted = p.get_state()
    assert np.array_equal(H1, H) and time == 0.0 and accepted == 0


def test_preheat_large_mesh_properties(cuda_lib):
    """1280x2560, 20 steps, closed box: every row's heat balance holds, the
    boundary flux is zero and the heat integral is conserved to roundoff."""
    w = sy.Workload(nx=1280, ny=2560)
    case = pc.PreheatCase(w, kappa=1e-5, end=1.0, dt_max=1e-4)
    p = pc.gpu_instance(case)
    _, limit, first = p.begin()
    code, rows = p.advance(20)
    assert code == 0 and len(rows) == 20
    prev = first["integral"]
    for r in rows:
        assert r["boundaryFlux"] == 0.0
        assert abs(r["integral"] - prev) <= 1e-12 * abs(prev)
        prev = r["integral"]
    H, time, accepted = p.get_state()
    assert accepted == 20 and np.all(np.isfinite(H))


@pytest.mark.parametrize("name", ["through_diffusion", "quad_through"], ids=["uniform", "perturbed"])
def test_preheat_then_evolve_through_the_handoff_files(cuda_lib, tmp_path, name):
    """The reference's workflow (mantle_couple_preheat, then
    mantle_couple_evolve -preheat DIR; on a perturbed-quadrilateral mesh as
    its warped-mesh restart): the preheated H and the fixed C go through
    cellH1.dat / cellC1.dat / transport_state.json bit for bit, and the
    coupled transport continues from them at the preheat's end time, step for
    step with the oracle started from the same files."""
    from oracle import pyoracle as po
    from mantlepar_b200 import handoff
    from mantlepar_b200.phase import EutecticModel
    from mantlepar_b200.transport import Transport, TransportConfig
    case = pc.CASES[name]
    w = case.w
    p = pc.gpu_instance(case)
    code, _, _, _, _ = p.run()
    assert code == 0
    H, time, accepted = p.get_state()
    _, C = case.state()
    derived = EutecticModel(sy.material_s()).derived()
    if case.family == sy.MESH_RECTANGULAR:
        mesh = handoff.MeshInfo.of(w)
    else:
        mesh = handoff.MeshInfo(w.nx, w.ny, (w.x0, w.x1, w.y0, w.y1), "perturbed_quadrilateral", case.perturbation,
                                case.mesh_seed)
    handoff.write_state(str(tmp_path), mesh, H, C, time, accepted, derived)
    H2, C2, t2 = handoff.read_state(str(tmp_path), mesh, derived, sy.material_s().Xe)
    assert np.array_equal(H2, H) and np.array_equal(C2, C) and t2 == time == case.end
    xy = case.vertices()
    t = Transport(w, TransportConfig(cfl=w.cfl, integrator=2), vertices=xy)
    o = po.TransportOracle(sy.material_s(), w, integrator=2, mesh_family=case.family, perturbation=case.perturbation,
                           mesh_seed=case.mesh_seed)
    vs, ud = sy.face_velocity(w) if xy is None else sy.face_velocity_quads(w, xy)
    for x in (t, o):
        x.set_face_velocity(vs, ud)
        x.set_state(H2, C2, t2)
    _, got = t.step(3)
    code, ref = o.step(3)
    assert code == 0
    assert all(r["status"] == 0 for r in got)
    assert got[0]["time"] > t2 and got[-1]["time"] > got[0]["time"]
    for a, b in zip(got, ref):
        assert abs(a["time"] - b["time"]) <= 1e-12 * abs(b["time"])
    a, b = np.stack(t.get_state()), np.stack(o.get_state())
    for k in range(4):
        assert rel(a[k], b[k]) <= 1e-11, k


def test_preheat_quads_on_a_rectangular_mesh_match_the_uniform_form(cuda_lib):
    """mp_preheat_create_quads given the vertices of the uniform mesh runs the
    per-cell-table kernels; every row, the final H and the diagnostics agree
    with the uniform kernels to roundoff."""
    from mantlepar_b200.preheat import Preheat
    case = pc.CASES["through_diffusion"]
    a = pc.gpu_instance(case)
    b = Preheat(case.w, pc.gpu_config(case), vertices=sy.quad_vertices(case.w, sy.MESH_RECTANGULAR))
    b.set_velocity(case.velocity())
    b.set_state(*case.state())
    ra, la, fa = a.begin()
    rb, lb, fb = b.begin()
    assert rel(rb, ra) <= RTOL and abs(lb - la) <= RTOL * la
    ca, rows_a = a.advance(1000)
    cb, rows_b = b.advance(1000)
    assert ca == cb == 0 and len(rows_a) == len(rows_b)
    for x, y in zip(rows_a, rows_b):
        assert x["step"] == y["step"] and x["time"] == y["time"]
        assert abs(x["integral"] - y["integral"]) <= RTOL * abs(y["integral"])
    assert rel(b.get_state()[0], a.get_state()[0]) <= RTOL
    for x, y in zip(b.diagnostics(), a.diagnostics()):
        assert rel(x, y) <= RTOL if np.max(y) > 0 else np.all(x == 0)


def test_preheat_rejects_invalid_quads(cuda_lib):
    from mantlepar_b200._capi import MPError
    from mantlepar_b200.preheat import Preheat
    w = sy.Workload(nx=4, ny=4)
    xy = sy.quad_vertices(w, sy.MESH_RECTANGULAR).reshape(5, 5, 2).copy()
    xy[2, 2] = xy[3, 3] + [0.01, 0.01]          # fold one interior vertex past its neighbour
    with pytest.raises(MPError) as e:
        Preheat(w, pc.gpu_config(pc.PreheatCase(w)), vertices=xy.reshape(-1))
    assert e.value.code == 62


def test_preheat_quad_large_mesh_properties(cuda_lib):
    """1280x2560 perturbed-quadrilateral mesh, closed box, 10 steps: the heat
    balance of every row holds, the boundary flux is zero and the heat
    integral is conserved to roundoff."""
    w = sy.Workload(nx=1280, ny=2560)
    case = pc.PreheatCase(w, kappa=1e-5, end=1.0, dt_max=1e-4, family=sy.MESH_PERTURBED, perturbation=0.2)
    p = pc.gpu_instance(case)
    _, limit, first = p.begin()
    code, rows = p.advance(10)
    assert code == 0 and len(rows) == 10
    prev = first["integral"]
    for r in rows:
        assert r["boundaryFlux"] == 0.0
        assert abs(r["integral"] - prev) <= 1e-12 * abs(prev)
        prev = r["integral"]
    H, _, accepted = p.get_state()
    assert accepted == 10 and np.all(np.isfinite(H))


@pytest.mark.parametrize("nx,ny,families", [(12, 10, (0, 1, 2)), (1280, 2560, (0, 1))], ids=["12x10", "1280x2560"])
def test_linear_field_gives_the_exact_rhs(cuda_lib, nx, ny, families):
    """Linear exactness, a size-independent property: the preheat RHS of a
    linear H in a uniform flow is -v . grad H in every cell off the inflow
    walls (1e-13 at 12x10, where it also equals the oracle's RHS; 1e-10 at
    1280x2560, where roundoff grows like 1/h), on uniform, perturbed and
    stretched meshes: the GPU-built per-cell tables reproduce linear data."""
    from test_oracle_preheat import LINEAR_RHS, linear_field_case
    from mantlepar_b200.preheat import Preheat
    w = sy.Workload(nx=nx, ny=ny)
    for family in families:
        case, xy, vs, H = linear_field_case(w, family)
        p = Preheat(w, pc.gpu_config(case), vertices=None if family == sy.MESH_RECTANGULAR else xy)
        p.set_velocity(vs)
        p.set_state(H, np.full(w.cells, 0.3))
        rhs, _ = p.rhs()
        r = rhs.reshape(w.ny, w.nx)
        assert np.max(np.abs(r[1:, 1:] - LINEAR_RHS)) <= (1e-13 if nx == 12 else 1e-10), family
        if nx == 12:
            t = pc.oracle_instance(case)
            t.set_face_velocity(vs, np.zeros_like(vs))
            t.set_state(H, np.full(w.cells, 0.3))
            code, ref, _ = t.preheat_rhs()
            assert code == 0 and rel_inf(rhs, ref) <= RTOL, family
        p.close()

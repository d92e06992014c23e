"""The transport oracle against the reference-backed build and the golden runs."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from mantlepar_b200 import synthetic as sy

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "transport_golden.npz"))
CASES = {"w20": sy.Workload(nx=20, ny=20), "w2x2": sy.Workload(nx=2, ny=2),
         "w3x5": sy.Workload(nx=3, ny=5, seed=7), "w7x4": sy.Workload(nx=7, ny=4, seed=9, noise_H=0.1)}


def _oracle(w, integrator=2, lib=None, **kw):
    t = po.TransportOracle(sy.material_s(), w, lib=lib, integrator=integrator, **kw)
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    return t


def bits(a):
    return np.ascontiguousarray(a).view(np.int64)


@pytest.mark.parametrize("name", list(CASES))
def test_restated_rhs_equals_golden_bitwise(name):
    t = _oracle(CASES[name])
    code, r = t.rhs()
    assert code == 0
    for k in ["rhsH", "rhsC", "T", "phi", "rate"]:
        assert np.array_equal(bits(r[k]), bits(GOLDEN[f"{name}_rhs_{k}"])), k
    code, a, b = t.limiter()
    assert code == 0
    assert np.array_equal(bits(a), bits(GOLDEN[f"{name}_thetaH"]))
    assert np.array_equal(bits(b), bits(GOLDEN[f"{name}_thetaC"]))


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("integ", [2, 3])
def test_restated_steps_equal_golden_bitwise(name, integ):
    t = _oracle(CASES[name], integ)
    code, reps = t.step(10)
    assert code == 0
    st = np.stack(t.get_state())
    assert np.array_equal(bits(st), bits(GOLDEN[f"{name}_rk{integ}_10"]))
    assert np.array_equal(np.array([r["retries"] for r in reps]), GOLDEN[f"{name}_rk{integ}_10_retries"])


def test_oracle_conservation_and_cfl():
    """Per-step balance (evolve.cpp:486-490, integration-test bound 1e-12) and courant <= cfl."""
    w = CASES["w20"]
    t = _oracle(w, 2)
    code, reps = t.step(25)
    assert code == 0
    for r in reps:
        assert abs(r["balanceH"]) < 1e-12 and abs(r["balanceC"]) < 1e-12
        assert r["courant"] <= w.cfl * (1 + 1e-10)
    H, C, T, phi = t.get_state()
    assert H.min() >= 0 and C.min() >= 0 and C.max() <= sy.material_s().Xe
    assert np.all((phi >= 0) & (phi < 1))


def test_uniform_tables_match_per_cell_tables():
    """Sharing one table set per boundary class moves results only at roundoff."""
    w = sy.Workload(nx=12, ny=16, seed=3)
    a = _oracle(w, 3)
    b = _oracle(w, 3, uniform_tables=True)
    assert a.step(5)[0] == 0 and b.step(5)[0] == 0
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.max(np.abs(x - y) / np.maximum(np.abs(y), 1e-3)) < 1e-13


def test_inadmissible_state_rejected_and_rolled_back():
    w = CASES["w3x5"]
    t = _oracle(w)
    H, C = sy.initial_state(w)
    C = C.copy()
    C[4] = 0.7          # above Xe = 0.5
    t.set_state(H, C)
    code, _ = t.step(1)
    assert code != 0
    H2, C2, _, _ = t.get_state()
    assert np.array_equal(C2, C)   # state untouched


@pytest.mark.skipif(not po.reference_available(), reason="reference build (oracle/_ref) not present")
def test_restated_equals_reference_on_new_seed():
    w = sy.Workload(nx=9, ny=11, seed=123, noise_H=0.08, psi_amplitude=0.15)
    a = _oracle(w, 3)
    b = _oracle(w, 3, lib=po.reference())
    assert a.step(6)[0] == 0 and b.step(6)[0] == 0
    assert np.array_equal(bits(np.stack(a.get_state())), bits(np.stack(b.get_state())))


def test_oracle_time_controls():
    """evolve.cpp:449-457,483: the last step lands on time.end; the fixed
    control keeps dt = initialStep with no retries and rejects a step above the
    CFL bound."""
    w = CASES["w20"]
    t = _oracle(w, integrator=3)
    t_end = 0.0123
    assert t.set_time_control(0, t_end) == 0
    code, reps = t.step(60)
    assert code == 0
    taken = [r for r in reps if r["dt"] > 0]
    assert taken and taken[-1]["time"] == t_end and reps[-1]["time"] == t_end
    assert all(r["dt"] == 0 for r in reps[len(taken):])
    assert taken[-1]["dt"] < max(r["dt"] for r in taken)       # shortened last step
    # fixed control below the CFL bound: constant dt, no retries
    f = _oracle(w, integrator=2, dt_initial=2e-4)
    assert f.set_time_control(1, 1e-3) == 0
    code, reps = f.step(10)
    assert code == 0
    taken = [r for r in reps if r["dt"] > 0]
    assert len(taken) == 5 and all(abs(r["dt"] - 2e-4) < 1e-18 for r in taken) and all(r["retries"] == 0 for r in taken)
    # fixed control above the CFL bound: PETSC_ERR_ARG_OUTOFRANGE, state kept
    g = _oracle(w, integrator=2, dt_initial=1.0)
    g.set_time_control(1)
    H0, C0, _, _ = g.get_state()
    code, _ = g.step(1)
    assert code == 63
    H1, C1, _, _ = g.get_state()
    assert np.array_equal(H0, H1) and np.array_equal(C0, C1)


@pytest.mark.skipif(not po.reference_available(), reason="reference-backed oracle not built")
@pytest.mark.parametrize("bc", [((1, 2, 0, 0), (0.9, -0.02, 0.0, 0.0)), ((0, 0, 1, 1), (0.0, 0.0, 0.5, 0.6)),
                                ((0, 0, 0, 0), (0.0, 0.0, 0.0, 0.0))], ids=["T_top_flux_bottom", "T_sides", "insulated"])
def test_diffusion_restatement_equals_reference_bitwise(bc):
    """Thermal diffusion (diffusiveflux.cpp:105-334 through evolve.cpp:330-349):
    the restated integration and derivative weights equal the reference's own
    functions bit for bit, for the RHS and for 10 SSPRK3 steps."""
    w = sy.Workload(nx=12, ny=14, seed=6)
    out = []
    for lib in (po.restated(), po.reference()):
        t = _oracle(w, integrator=3, lib=lib)
        assert t.set_diffusion(0.02, *bc) == 0
        code, r = t.rhs()
        assert code == 0
        code, reps = t.step(10)
        assert code == 0
        out.append((r, t.get_state(), reps))
    (ra, sa, pa), (rb, sb, pb) = out
    for k in ["rhsH", "rhsC", "T", "phi", "rate"]:
        assert np.array_equal(bits(ra[k]), bits(rb[k])), k
    for x, y in zip(sa, sb):
        assert np.array_equal(bits(x), bits(y))
    assert [r["dt"] for r in pa] == [r["dt"] for r in pb]


def test_diffusion_changes_the_solution_as_expected():
    """Diffusion moves heat down the temperature gradient: with an insulated
    box the H integral is conserved; with a hot top wall heat flows in."""
    w = sy.Workload(nx=12, ny=14, seed=6)
    base = _oracle(w, integrator=3)
    _, r0 = base.rhs()
    ins = _oracle(w, integrator=3)
    ins.set_diffusion(0.02)
    _, r1 = ins.rhs()
    hot = _oracle(w, integrator=3)
    hot.set_diffusion(0.02, (0, 1, 0, 0), (0.0, 3.0, 0.0, 0.0))
    _, r2 = hot.rhs()
    assert not np.array_equal(r0["rhsH"], r1["rhsH"])
    assert np.array_equal(r0["rhsC"], r1["rhsC"])                     # C does not diffuse
    assert abs(r1["boundaryH"] - r0["boundaryH"]) < 1e-15              # insulated: no extra boundary flux
    assert r2["boundaryH"] < r1["boundaryH"]                           # hot top wall: heat flows in
    assert r1["maxRate"] > r0["maxRate"]                               # diffusion enters the CFL rate


def product_like(w, lib=None):
    """Thermal diffusion, lithostatic pressure and the adiabatic source together
    (the features of the reference's product input), on material S with a
    lighter density so the eutectic temperature varies mildly with depth."""
    import dataclasses
    mat = dataclasses.replace(sy.material_s(), rho=100.0, alpha0=3e-5)
    t = po.TransportOracle(mat, w, lib=lib, integrator=3)
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    assert t.set_diffusion(0.01, (1, 1, 0, 0), (0.9, 0.2, 0.0, 0.0)) == 0
    assert t.set_pressure_model(1, 1.1) == 0
    assert t.set_cell_velocity(*sy.cell_velocity(w)) == 0
    return t, mat


@pytest.mark.skipif(not po.reference_available(), reason="reference-backed oracle not built")
def test_product_features_restatement_equals_reference_bitwise():
    w = sy.Workload(nx=10, ny=12, seed=3)
    out = []
    for lib in (po.restated(), po.reference()):
        t, _ = product_like(w, lib)
        code, r = t.rhs()
        assert code == 0
        code, reps = t.step(8)
        assert code == 0
        out.append((r, t.get_state(), reps))
    (ra, sa, pa), (rb, sb, pb) = out
    for k in ["rhsH", "rhsC", "T", "phi", "rate"]:
        assert np.array_equal(bits(ra[k]), bits(rb[k])), k
    assert ra["sourceH"] == rb["sourceH"] and ra["sourceH"] != 0.0
    for x, y in zip(sa, sb):
        assert np.array_equal(bits(x), bits(y))
    assert [r["dt"] for r in pa] == [r["dt"] for r in pb]
    assert all(abs(r["balanceH"]) < 1e-12 for r in pa)


def test_source_requires_cell_velocities():
    import dataclasses
    w = sy.Workload(nx=6, ny=6)
    t = po.TransportOracle(dataclasses.replace(sy.material_s(), alpha0=3e-5), w, integrator=3)
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    code, _ = t.rhs()
    assert code == 73


# The reference's SSPRK2 order test (src/couple/test/test_evolution.py:119-145):
# a uniform, dry, motionless 2x2 box of the product input's mesh and material
# (cells 0.25 wide on [0, 0.5] x [-0.5, 0], lithostatic pressure with the
# surface at y = 0) at H = 2.1, C = 0.05 cools through walls held at T = 2
# with kappa = 0.01; its semidiscrete thermal mode decays exactly as
# exp(-decay t), decay = 2 kappa (25/12) / (0.9 * 0.25 / 4) / 0.25, so SSPRK2
# with fixed steps 0.01 and 0.005 to t = 0.1 has an error ratio near 4.
COOLING_BOX = sy.Workload(nx=2, ny=2, x0=0.0, x1=0.5, y0=-0.5, y1=0.0)
COOLING_DECAY = 2 * .01 * (25 / 12) / (.9 * .25 / 4) / .25


def cooling_box_oracle(dt, lib=None):
    w = COOLING_BOX
    o = po.TransportOracle(sy.Material(), w, lib=lib, integrator=2, cfl=0.4, dt_initial=dt, dt_max=dt,
                           dt_min=1e-12, H_policy=2, C_policy=2, inflow_C=0.05)
    assert o.set_diffusion(0.01, (1, 1, 1, 1), (2.0, 2.0, 2.0, 2.0)) == 0
    assert o.set_pressure_model(1, 0.0) == 0
    assert o.set_cell_velocity(np.zeros(w.cells * 25), np.zeros(w.cells * 25)) == 0
    z = np.zeros(w.edges * 5)
    o.set_face_velocity(z, z)
    o.set_state(np.full(w.cells, 2.1), np.full(w.cells, .05))
    assert o.set_time_control(1, 0.1) == 0
    return o


def test_ssprk2_order_on_the_cooling_box():
    exact = 2 + .1 * np.exp(-COOLING_DECAY * .1)
    errors = []
    for dt in (.01, .005):
        o = cooling_box_oracle(dt)
        code, reps = o.step(100)
        assert code == 0 and sum(1 for r in reps if r["dt"] > 0) == round(.1 / dt)
        H = o.get_state()[0]
        assert np.max(np.abs(H - H[0])) <= 1e-12
        errors.append(abs(H[0] - exact))
        if po.reference_available():
            r = cooling_box_oracle(dt, po.reference())
            assert r.step(100)[0] == 0
            assert np.array_equal(r.get_state()[0], H)
    assert 3.8 < errors[0] / errors[1] < 4.2, errors


def constant_state_oracle(w, family, lib=None):
    """A uniform state (H 0.6, C 0.31: solid and liquid) in the uniform flow
    v_s = (0.3, 0.2), u_d = (0, 0.01), inflow values equal to the state."""
    o = po.TransportOracle(sy.material_s(), w, lib=lib, integrator=3, inflow_H=0.6, inflow_C=0.31,
                           mesh_family=family, perturbation=0.2, mesh_seed=11)
    xy = o.vertices()
    o.set_face_velocity(sy.uniform_face_velocity(w, xy, 0.3, 0.2), sy.uniform_face_velocity(w, xy, 0.0, 0.01))
    o.set_state(np.full(w.cells, 0.6), np.full(w.cells, 0.31))
    return o, xy


@pytest.mark.parametrize("family", [sy.MESH_RECTANGULAR, sy.MESH_PERTURBED, sy.MESH_SINE_STRETCHED])
def test_constant_state_is_preserved(family):
    """Constant preservation (src/mlweno/test/test_advection_diffusion.cpp:
    125-148, 2e-10 there): a uniform state in a uniform flow has a zero RHS
    to roundoff, in the restated and the reference build."""
    w = sy.Workload(nx=12, ny=10)
    for lib in [None] + ([po.reference()] if po.reference_available() else []):
        o, _ = constant_state_oracle(w, family, lib)
        code, r = o.rhs()
        assert code == 0 and r["phi"].min() > 0
        for k in ("rhsH", "rhsC"):
            assert np.max(np.abs(r[k])) <= 1e-13 * r["maxRate"], k


@pytest.mark.skipif(not po.reference_available(), reason="reference-backed oracle not built")
@pytest.mark.parametrize("name", ["inflow_outflow", "darcy_exponent_2", "global_lf", "zero_flux_C",
                                  "outflow_H_at_inflow"])
def test_boundary_policies_restatement_equals_reference_bitwise(name):
    """Flow through the walls (inflow/outflow/zero-flux policies, global LF
    speed, Darcy exponent): the restatement equals the reference's own classes
    bit for bit over a stage and 10 SSPRK3 steps, and both reject the
    outflow-only policy on an inflow wall with the same error class."""
    import boundary_cases as bcs
    kw, status = bcs.CASES[name]
    vs, ud = bcs.face_velocity()
    H, C = sy.initial_state(bcs.W)
    out = []
    for lib in (po.restated(), po.reference()):
        o = po.TransportOracle(sy.material_s(), bcs.W, lib=lib, integrator=3, **kw)
        o.set_face_velocity(vs, ud)
        o.set_state(H, C)
        code, r = o.rhs()
        code2, reps = o.step(10)
        out.append((code, code2, r, np.stack(o.get_state()), [x["retries"] for x in reps]))
        o.close()
    (c1, s1, r1, st1, rt1), (c2, s2, r2, st2, rt2) = out
    assert c1 == c2 == status and s1 == s2 == status
    if status:
        return
    for k in ("rhsH", "rhsC", "T", "phi", "rate"):
        assert np.array_equal(bits(r1[k]), bits(r2[k])), k
    assert r1["boundaryH"] == r2["boundaryH"] and r1["boundaryC"] == r2["boundaryC"]
    assert r1["boundaryH"] != 0.0                       # the walls carry flux
    assert rt1 == rt2 and np.array_equal(bits(st1), bits(st2))

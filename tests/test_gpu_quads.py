"""GPU parity of the transport on general quad meshes (perturbed-quadrilateral
and sine-stretched, src/core/mesh.cpp:27-55) against the reference-backed
golden runs and the oracle.

Bars as the uniform path: per-cell relative error 1e-12 for T, phi, rate,
the limiter factors and the state after 10 SSPRK3 steps
(|x - ref| / max(|ref|, 1e-3 max|ref|)); right-hand sides against their
infinity norm (1e-12); step sizes 1e-12 relative with equal retries.
"""
import os

import numpy as np
import pytest

from mantlepar_b200 import synthetic as sy
import quad_cases as qc

pytestmark = pytest.mark.gpu

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "quads_golden.npz"))
RTOL = 1e-12


def rel(a, b):
    b = np.asarray(b)
    return np.max(np.abs(np.asarray(a) - b) / np.maximum(np.abs(b), 1e-3 * max(np.max(np.abs(b)), 1e-300)))


def rel_inf(a, b):
    b = np.asarray(b)
    return np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300)


def make_diffusion(name):
    from mantlepar_b200.transport import Transport, TransportConfig
    w, fam, pert, opt = qc.quad_case(name)
    xy = GOLDEN[f"{name}_xy"]
    vs, ud = sy.face_velocity_quads(w, xy)
    t = Transport(w, TransportConfig(cfl=w.cfl, integrator=3, diffusivity=0.02 if opt.get("diffusion") else 0.0),
                  vertices=xy)
    t.set_face_velocity(vs, ud)
    t.set_state(*sy.initial_state(w))
    if opt.get("diffusion"):
        t.set_thermal_bc((1, 2, 0, 1), (0.9, -0.02, 0.0, 0.4))
    return t


@pytest.mark.parametrize("name", qc.QUAD_CASES)
def test_quad_rhs_and_limiter_match_reference(cuda_lib, name):
    t = make_diffusion(name)
    r = t.rhs()
    for k in ["T", "phi", "rate"]:
        g = GOLDEN[f"{name}_rhs_{k}"]
        e = rel(r[k], g) if np.max(np.abs(g)) > 0 else np.max(np.abs(r[k]))
        assert e <= RTOL, (k, e)
    for k in ["rhsH", "rhsC"]:
        e = rel_inf(r[k], GOLDEN[f"{name}_rhs_{k}"])
        assert e <= RTOL, (k, e)
    tot = GOLDEN[f"{name}_rhs_totals"]
    assert abs(r["maxRate"] - tot[2]) <= RTOL * tot[2]
    assert abs(r["boundaryH"] - tot[0]) <= RTOL * max(1.0, abs(tot[0]))
    a, b = t.limiter()
    assert np.max(np.abs(a - GOLDEN[f"{name}_thetaH"])) <= RTOL
    assert np.max(np.abs(b - GOLDEN[f"{name}_thetaC"])) <= RTOL


@pytest.mark.parametrize("name", qc.QUAD_CASES)
def test_quad_steps_match_reference(cuda_lib, name):
    t = make_diffusion(name)
    _, reps = t.step(10)
    st = np.stack(t.get_state())
    ref = GOLDEN[f"{name}_rk3_10"]
    for k in range(4):
        g = ref[k]
        e = rel(st[k], g) if np.max(np.abs(g)) > 0 else np.max(np.abs(st[k]))
        assert e <= RTOL, (k, e)
    dts = np.array([x["dt"] for x in reps])
    assert np.max(np.abs(dts - GOLDEN[f"{name}_rk3_10_dt"]) / GOLDEN[f"{name}_rk3_10_dt"]) <= RTOL
    assert [x["retries"] for x in reps] == list(GOLDEN[f"{name}_rk3_10_retries"])


def test_rectangular_vertices_reproduce_the_uniform_path(cuda_lib):
    """The uniform mesh given as vertices runs the per-cell path and agrees
    with the uniform-table path to 1e-12."""
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.Workload(nx=20, ny=20)
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    a = Transport(w, TransportConfig(cfl=w.cfl, integrator=3))
    b = Transport(w, TransportConfig(cfl=w.cfl, integrator=3), vertices=sy.quad_vertices(w, sy.MESH_RECTANGULAR))
    for t in (a, b):
        t.set_face_velocity(vs, ud)
        t.set_state(H, C)
    ra, rb = a.rhs(), b.rhs()
    for k in ["T", "phi", "rate"]:
        assert rel(rb[k], ra[k]) <= RTOL, k
    for k in ["rhsH", "rhsC"]:
        assert rel_inf(rb[k], ra[k]) <= RTOL, k
    a.step(10)
    b.step(10)
    for x, y in zip(b.get_state(), a.get_state()):
        assert rel(x, y) <= 1e-11


def test_quad_product_features_match_oracle(cuda_lib):
    """Thermal diffusion, lithostatic pressure and the adiabatic source on a
    perturbed mesh, against the restated oracle (equal to the reference build
    bit for bit on these features)."""
    import dataclasses
    from oracle import pyoracle as po
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.Workload(nx=10, ny=12, seed=3)
    mat = dataclasses.replace(sy.material_s(), rho=100.0, alpha0=3e-5)
    o = po.TransportOracle(mat, w, integrator=3, mesh_family=1, perturbation=0.2, mesh_seed=5)
    xy = o.vertices()
    vs, ud = sy.face_velocity_quads(w, xy)
    cv = sy.cell_velocity_quads(w, xy)
    H, C = sy.initial_state(w)
    o.set_face_velocity(vs, ud)
    o.set_state(H, C)
    assert o.set_diffusion(0.01, (1, 1, 0, 0), (0.9, 0.2, 0.0, 0.0)) == 0
    assert o.set_pressure_model(1, 1.1) == 0
    assert o.set_cell_velocity(*cv) == 0
    t = Transport(w, TransportConfig(material=mat, cfl=w.cfl, integrator=3, diffusivity=0.01), vertices=xy)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    t.set_thermal_bc((1, 1, 0, 0), (0.9, 0.2, 0.0, 0.0))
    t.set_pressure_model(t.LITHOSTATIC, 1.1)
    t.set_cell_velocity(*cv)
    code, ro = o.rhs()
    assert code == 0
    rg = t.rhs()
    for k in ["T", "phi", "rate"]:
        assert rel(rg[k], ro[k]) <= RTOL, k
    assert rel_inf(rg["rhsH"], ro["rhsH"]) <= RTOL
    assert abs(rg["sourceH"] - ro["sourceH"]) <= RTOL * abs(ro["sourceH"]) and ro["sourceH"] != 0.0
    code, reps_o = o.step(5)
    assert code == 0
    _, reps_g = t.step(5)
    for x, y in zip(t.get_state(), o.get_state()):
        assert rel(x, y) <= RTOL
    assert [r["retries"] for r in reps_g] == [r["retries"] for r in reps_o]


def test_invalid_quad_meshes_are_rejected(cuda_lib):
    from mantlepar_b200._capi import MPError
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.Workload(nx=4, ny=4)
    xy = sy.quad_vertices(w, sy.MESH_RECTANGULAR).reshape(5, 5, 2).copy()
    xy[2, 2] = xy[3, 3] + [0.01, 0.01]          # fold one interior vertex past its neighbour
    with pytest.raises(MPError) as e:
        Transport(w, TransportConfig(), vertices=xy.reshape(-1))
    assert e.value.code == 62


def test_mixed_form_on_quads_equals_fp64(cuda_lib):
    """The mixed form evaluates the FP64 stage on a general quad mesh too:
    10 SSPRK3 steps equal the FP64 form bit for bit."""
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.Workload(nx=12, ny=10, seed=3)
    xy = sy.quad_vertices(w, sy.MESH_PERTURBED)
    out = []
    for precision in (0, 1):
        t = Transport(w, TransportConfig(cfl=w.cfl, integrator=3, precision=precision), vertices=xy)
        t.set_face_velocity(*sy.face_velocity_quads(w, xy))
        t.set_state(*sy.initial_state(w))
        _, reps = t.step(10)
        out.append((np.stack(t.get_state()), [r["dt"] for r in reps]))
        t.close()
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]


def test_quad_large_mesh_steps(cuda_lib):
    """1280x2560 perturbed-quadrilateral mesh: 3 SSPRK3 steps, every step
    within the balance bound, the state admissible."""
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.Workload(nx=1280, ny=2560)
    xy = sy.quad_vertices(w, sy.MESH_PERTURBED, 0.2, 11)
    t = Transport(w, TransportConfig(cfl=w.cfl, integrator=3), vertices=xy)
    t.set_face_velocity(*sy.face_velocity_quads(w, xy))
    t.set_state(*sy.initial_state(w))
    _, reps = t.step(3)
    assert all(abs(r["balanceH"]) < 1e-10 * abs(r["H_integral"]) for r in reps)
    H, C, T, phi = t.get_state()
    assert np.all(np.isfinite(H)) and H.min() >= 0 and C.min() >= 0 and C.max() <= 0.5


def test_gpu_tables_equal_host_builder(cuda_lib, tmp_path):
    """The GPU table builder (no FMA contraction) reproduces the host
    builder's per-cell candidate matrices, smoothness forms and geometry bit
    for bit, whole mesh, slab and boundary classes."""
    import subprocess
    from mantlepar_b200 import build as B
    exe = str(tmp_path / "quad_tables_check")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    obj = str(tmp_path / "qtk.o")
    subprocess.run([B.nvcc()] + B.ARCH + ["-O3", "-std=c++17", "--fmad=false", "-c",
                    os.path.join(B.CSRC, "quad_table_kernels.cu"), "-o", obj], check=True)
    subprocess.run([B.nvcc()] + B.ARCH + ["-O3", "-std=c++17", "-I", B.CSRC,
                    os.path.join(root, "tests", "cpp", "quad_tables_check.cu"), os.path.join(B.CSRC, "quad_tables.cpp"),
                    obj, "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:]
    assert "TOTAL DIFFERENT 0" in r.stdout


def test_perturbed_mesh_at_320x640_matches_the_reference_build(cuda_lib):
    """A 320x640 perturbed-quadrilateral mesh (perturbation 0.2, seed 11; 205k
    cells, each with its own stencil tables) against the reference's own
    classes (oracle/_ref; the restated oracle where it was not built):
    limiter factors, one stage and one SSPRK3 step, every quantity at 1e-12
    per cell (measured: at most 4.8e-13, theta and phi)."""
    from oracle import pyoracle as po
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.Workload(nx=320, ny=640)
    lib = po.reference() if po.reference_available() else po.restated()
    o = po.TransportOracle(sy.material_s(), w, lib=lib, integrator=3, threads=os.cpu_count() or 1,
                           mesh_family=1, perturbation=0.2, mesh_seed=11)
    xy = o.vertices()
    vs, ud = sy.face_velocity_quads(w, xy)
    H, C = sy.initial_state(w)
    o.set_face_velocity(vs, ud)
    o.set_state(H, C)
    t = Transport(w, TransportConfig(cfl=w.cfl, integrator=3), vertices=xy)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    code, oa, ob = o.limiter()
    assert code == 0
    ga, gb = t.limiter()
    assert rel(ga, oa) <= RTOL and rel(gb, ob) <= RTOL
    code, ro = o.rhs()
    assert code == 0
    rg = t.rhs()
    for k in ["T", "phi", "rate"]:
        assert rel(rg[k], ro[k]) <= RTOL, k
    for k in ["rhsH", "rhsC"]:
        assert rel_inf(rg[k], ro[k]) <= RTOL, k
    code, reps_o = o.step(1)
    assert code == 0
    _, reps_g = t.step(1)
    assert reps_g[0]["retries"] == reps_o[0]["retries"]
    assert abs(reps_g[0]["dt"] - reps_o[0]["dt"]) <= RTOL * reps_o[0]["dt"]
    for x, y in zip(t.get_state(), o.get_state()):
        assert rel(x, y) <= RTOL
    t.close()
    o.close()

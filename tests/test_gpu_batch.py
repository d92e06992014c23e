"""Batched transport: each instance equals its single-instance run bit for bit."""
import numpy as np
import pytest

from mantlepar_b200 import synthetic as sy

pytestmark = pytest.mark.gpu

WORKLOADS = [sy.Workload(nx=20, ny=20, seed=1), sy.Workload(nx=40, ny=60, seed=5, psi_amplitude=0.15),
             sy.Workload(nx=3, ny=5, seed=7), sy.Workload(nx=64, ny=32, seed=9, noise_H=0.1),
             sy.Workload(nx=2, ny=2, seed=11, psi_amplitude=0.05)]


def solo(w, cfg, steps):
    from mantlepar_b200.transport import Transport
    t = Transport(w, cfg)
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    _, reps = t.step(steps)
    return t.get_state(), reps


def batch_of(ws, cfg):
    from mantlepar_b200.batch import Batch
    b = Batch(ws, cfg)
    for i, w in enumerate(ws):
        vs, ud = sy.face_velocity(w)
        H, C = sy.initial_state(w)
        b.set_face_velocity(i, vs, ud)
        b.set_state(i, H, C)
    return b


@pytest.mark.parametrize("precision,integ", [(0, 3), (0, 2), (1, 3)])
def test_batch_equals_solo_bitwise(cuda_lib, precision, integ):
    from mantlepar_b200.transport import TransportConfig
    cfg = TransportConfig(cfl=0.4, integrator=integ, precision=precision)
    b = batch_of(WORKLOADS, cfg)
    reps = b.step(8)
    for i, w in enumerate(WORKLOADS):
        (H, C, T, phi), sreps = solo(w, cfg, 8)
        got = b.get_state(i)
        assert got["status"] == 0 and got["accepted"] == 8
        for a, x in ((got["H"], H), (got["C"], C), (got["T"], T), (got["phi"], phi)):
            assert np.array_equal(a, x)
        assert [r[i]["retries"] for r in reps] == [r["retries"] for r in sreps]
        assert [r[i]["dt"] for r in reps] == [r["dt"] for r in sreps]
        assert [r[i]["balanceH"] for r in reps] == [r["balanceH"] for r in sreps]


def test_failing_instance_is_isolated(cuda_lib):
    from mantlepar_b200.transport import TransportConfig
    cfg = TransportConfig(cfl=0.4, integrator=3)
    b = batch_of(WORKLOADS[:3], cfg)
    w = WORKLOADS[1]
    H, C = sy.initial_state(w)
    C = C.copy()
    C[17] = 0.9
    b.set_state(1, H, C)
    b.step(3)
    bad = b.get_state(1)
    assert bad["status"] == 63 and bad["accepted"] == 0
    assert np.array_equal(bad["C"], C)
    for i in (0, 2):
        (Hs, Cs, _, _), _ = solo(WORKLOADS[i], cfg, 3)
        got = b.get_state(i)
        assert got["status"] == 0 and np.array_equal(got["H"], Hs) and np.array_equal(got["C"], Cs)


def test_add_remove_and_autotune_keep_results(cuda_lib):
    from mantlepar_b200.transport import TransportConfig
    cfg = TransportConfig(cfl=0.4, integrator=3)
    b = batch_of(WORKLOADS[:2], cfg)
    tile, ms = b.autotune(reps=1)
    assert len(tile) == 3 and ms > 0
    b.step(2)
    b.remove(0)
    k = b.add(WORKLOADS[3])
    assert k == 0                       # the freed slot is reused
    vs, ud = sy.face_velocity(WORKLOADS[3])
    H, C = sy.initial_state(WORKLOADS[3])
    b.set_face_velocity(k, vs, ud)
    b.set_state(k, H, C)
    b.step(3)
    (H1, C1, _, _), _ = solo(WORKLOADS[1], cfg, 5)
    got = b.get_state(1)
    assert np.array_equal(got["H"], H1) and np.array_equal(got["C"], C1)
    (H3, C3, _, _), _ = solo(WORKLOADS[3], cfg, 3)
    got = b.get_state(k)
    assert np.array_equal(got["H"], H3) and np.array_equal(got["C"], C3)
    assert b.bytes_in_use() == sum(b.instance_bytes(w) for w in (WORKLOADS[1], WORKLOADS[3]))


@pytest.mark.parametrize("device_steps", [True, False])
def test_batch_adiabatic_source_equals_solo(cuda_lib, device_steps):
    """alpha0 != 0 with thermal diffusion: every instance takes its own
    cell-point velocities (src/couple/evolve.cpp:359-369); each equals its
    single-instance run bit for bit, source integral in the reports."""
    import dataclasses
    from mantlepar_b200.batch import Batch
    from mantlepar_b200.transport import Transport, TransportConfig
    mat = dataclasses.replace(sy.material_s(), alpha0=3e-5)
    cfg = TransportConfig(material=mat, cfl=0.4, integrator=3, diffusivity=1e-4)
    ws = WORKLOADS[:4]
    b = Batch(ws, cfg)
    b.set_device_steps(device_steps)
    b.set_thermal_bc((1, 1, 0, 0), (0.9, 0.2, 0.0, 0.0))
    for i, w in enumerate(ws):
        vs, ud = sy.face_velocity(w)
        H, C = sy.initial_state(w)
        b.set_face_velocity(i, vs, ud)
        b.set_state(i, H, C)
        b.set_cell_velocity(i, *sy.cell_velocity(w))
    reps = b.step(6)
    for i, w in enumerate(ws):
        t = Transport(w, cfg)
        t.set_thermal_bc((1, 1, 0, 0), (0.9, 0.2, 0.0, 0.0))
        t.set_cell_velocity(*sy.cell_velocity(w))
        t.set_face_velocity(*sy.face_velocity(w))
        t.set_state(*sy.initial_state(w))
        _, sreps = t.step(6)
        got = b.get_state(i)
        assert got["status"] == 0 and got["accepted"] == 6
        for a, x in zip((got["H"], got["C"], got["T"], got["phi"]), t.get_state()):
            assert np.array_equal(a, x)
        assert [r[i]["sourceH"] for r in reps] == [r["sourceH"] for r in sreps]
        assert [r[i]["balanceH"] for r in reps] == [r["balanceH"] for r in sreps]
        assert any(r["sourceH"] != 0.0 for r in sreps)
        t.close()
    b.close()


def test_batch_source_needs_cell_velocities(cuda_lib):
    import dataclasses
    from mantlepar_b200._capi import MPError
    from mantlepar_b200.transport import TransportConfig
    mat = dataclasses.replace(sy.material_s(), alpha0=3e-5)
    b = batch_of(WORKLOADS[:2], TransportConfig(material=mat, cfl=0.4, integrator=3))
    with pytest.raises(MPError) as err:
        b.step(1)
    assert err.value.code == 73


QUADS = [(sy.Workload(nx=20, ny=24, seed=5), sy.MESH_PERTURBED, 0.2),
         (sy.Workload(nx=16, ny=20, seed=6, psi_amplitude=0.15), sy.MESH_SINE_STRETCHED, 0.0),
         (sy.Workload(nx=7, ny=9, seed=8), sy.MESH_PERTURBED, 0.1),
         (sy.Workload(nx=2, ny=3, seed=12), sy.MESH_PERTURBED, 0.1)]


def solo_quads(w, xy, cfg, steps, kappa_bc=None):
    from mantlepar_b200.transport import Transport
    t = Transport(w, cfg, vertices=xy)
    if kappa_bc:
        t.set_thermal_bc(*kappa_bc)
    t.set_face_velocity(*sy.face_velocity_quads(w, xy))
    t.set_state(*sy.initial_state(w))
    _, reps = t.step(steps)
    out = t.get_state(), reps
    t.close()
    return out


@pytest.mark.parametrize("integ,device_steps,kappa", [(3, True, 0.0), (2, True, 0.0), (3, False, 0.0),
                                                      (3, True, 0.02)])
def test_batch_with_quad_instances_equals_solo_bitwise(cuda_lib, integ, device_steps, kappa):
    """General quad meshes (perturbed, sine-stretched) in one batch with
    uniform meshes: every instance equals its own single-mesh run bit for bit
    (states, dt, retries, balance), through the step graph and the host loop,
    with diffusion too."""
    from mantlepar_b200.batch import Batch
    from mantlepar_b200.transport import TransportConfig
    cfg = TransportConfig(cfl=0.4, integrator=integ, diffusivity=kappa)
    bc = None          # zero-flux walls: the diffusion runs on the interior edges
    uni = WORKLOADS[:2]
    b = Batch(uni, cfg)
    b.set_device_steps(device_steps)
    if bc:
        b.set_thermal_bc(*bc)
    for i, w in enumerate(uni):
        b.set_face_velocity(i, *sy.face_velocity(w))
        b.set_state(i, *sy.initial_state(w))
    slots = {}
    for k, (w, fam, pert) in enumerate(QUADS):
        xy = sy.quad_vertices(w, fam, pert, seed=21 + k)
        i = b.add_quads(w, xy)
        b.set_face_velocity(i, *sy.face_velocity_quads(w, xy))
        b.set_state(i, *sy.initial_state(w))
        slots[i] = (w, xy)
    reps = b.step(40)
    for i, (w, xy) in slots.items():
        (H, C, T, phi), sreps = solo_quads(w, xy, cfg, 40, bc)
        got = b.get_state(i)
        assert got["status"] == 0 and got["accepted"] == 40
        for a, x in ((got["H"], H), (got["C"], C), (got["T"], T), (got["phi"], phi)):
            assert np.array_equal(a, x)
        assert [r[i]["retries"] for r in reps] == [r["retries"] for r in sreps]
        assert [r[i]["dt"] for r in reps] == [r["dt"] for r in sreps]
        assert [r[i]["balanceH"] for r in reps] == [r["balanceH"] for r in sreps]
    if not bc:
        for i, w in enumerate(uni):
            (H, C, T, phi), _ = solo(w, cfg, 40)
            got = b.get_state(i)
            assert np.array_equal(got["H"], H) and np.array_equal(got["phi"], phi)
    b.close()


def test_batch_quad_instances_come_and_go(cuda_lib):
    """A folded quad mesh is refused (MP_ERR_ARG_WRONG, no instance); quad
    instances removed and added again between steps leave the others' results
    equal to their solo runs, and re-use the captured step graph."""
    from mantlepar_b200._capi import MPError
    from mantlepar_b200.batch import Batch
    from mantlepar_b200.transport import TransportConfig
    cfg = TransportConfig(cfl=0.4, integrator=3)
    w0, fam0, p0 = QUADS[0]
    xy0 = sy.quad_vertices(w0, fam0, p0, seed=21)
    b = Batch([WORKLOADS[0]], cfg)
    b.set_face_velocity(0, *sy.face_velocity(WORKLOADS[0]))
    b.set_state(0, *sy.initial_state(WORKLOADS[0]))
    wb = sy.Workload(nx=4, ny=4)
    bad = sy.quad_vertices(wb, sy.MESH_RECTANGULAR).reshape(5, 5, 2).copy()
    bad[2, 2] = bad[3, 3] + [0.01, 0.01]
    with pytest.raises(MPError) as err:
        b.add_quads(wb, bad.reshape(-1))
    assert err.value.code == 62
    q = b.add_quads(w0, xy0)
    b.set_face_velocity(q, *sy.face_velocity_quads(w0, xy0))
    b.set_state(q, *sy.initial_state(w0))
    b.step(10)
    captures = b.graph_captures()
    b.remove(q)
    q2 = b.add_quads(w0, xy0)
    b.set_face_velocity(q2, *sy.face_velocity_quads(w0, xy0))
    b.set_state(q2, *sy.initial_state(w0))
    b.step(10)
    assert b.graph_captures() == captures
    (H, C, T, phi), _ = solo_quads(w0, xy0, cfg, 10)
    got = b.get_state(q2)
    assert got["status"] == 0 and np.array_equal(got["H"], H) and np.array_equal(got["phi"], phi)
    (H, C, T, phi), _ = solo(WORKLOADS[0], cfg, 20)
    got = b.get_state(0)
    assert np.array_equal(got["H"], H) and np.array_equal(got["phi"], phi)
    b.close()


def test_batch_quad_instances_with_adiabatic_source_equal_solo(cuda_lib):
    """alpha0 != 0 on general quad meshes in a batch (cell-point velocities
    at each quad cell's own quadrature points, evolve.cpp:359-369) with
    thermal diffusion: each equals its single-mesh run bit for bit, the source
    integral in the reports."""
    import dataclasses
    from mantlepar_b200.batch import Batch
    from mantlepar_b200.transport import Transport, TransportConfig
    mat = dataclasses.replace(sy.material_s(), alpha0=3e-5)
    cfg = TransportConfig(material=mat, cfl=0.4, integrator=3, diffusivity=1e-4)
    b = Batch([], cfg)
    slots = {}
    for k, (w, fam, pert) in enumerate(QUADS[:2]):
        xy = sy.quad_vertices(w, fam, pert, seed=31 + k)
        i = b.add_quads(w, xy)
        b.set_face_velocity(i, *sy.face_velocity_quads(w, xy))
        b.set_state(i, *sy.initial_state(w))
        b.set_cell_velocity(i, *sy.cell_velocity_quads(w, xy))
        slots[i] = (w, xy)
    reps = b.step(6)
    for i, (w, xy) in slots.items():
        t = Transport(w, cfg, vertices=xy)
        t.set_cell_velocity(*sy.cell_velocity_quads(w, xy))
        t.set_face_velocity(*sy.face_velocity_quads(w, xy))
        t.set_state(*sy.initial_state(w))
        _, sreps = t.step(6)
        got = b.get_state(i)
        assert got["status"] == 0 and got["accepted"] == 6
        for a, x in zip((got["H"], got["C"], got["T"], got["phi"]), t.get_state()):
            assert np.array_equal(a, x)
        assert [r[i]["sourceH"] for r in reps] == [r["sourceH"] for r in sreps]
        assert any(r["sourceH"] != 0.0 for r in sreps)
        t.close()
    b.close()

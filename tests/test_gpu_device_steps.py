"""Device-resident stepping: the CUDA-graph step loop (step controller on the
device, one host wait per 64 steps) against the host-driven loop (one
device->host read per stage), for one instance and for a batch.

Both loops run the same kernels; the controller replays the reference's
step rule (src/couple/evolve.cpp:449-507) with explicitly rounded FP64
operations, so states, reports and errors must agree bit for bit -- over
CFL retries, end times, the fixed control, failures and the product
features."""
import numpy as np
import pytest

from mantlepar_b200 import synthetic as sy

pytestmark = pytest.mark.gpu


def make(w, cfg, device_steps):
    from mantlepar_b200.transport import Transport
    t = Transport(w, cfg)
    t.set_device_steps(device_steps)
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    return t


def run_pair(w, cfg, steps, setup=None):
    out = []
    for dev in (True, False):
        t = make(w, cfg, dev)
        if setup:
            setup(t)
        code, reps = t.step(steps, raise_on_error=False)
        msg = t._lib.mp_last_error_string()
        out.append(dict(code=code, reps=reps, state=t.get_state(), time=t.get_time(), syncs=t.host_syncs(),
                        msg=msg if code else b""))
        t.close()
    return out


def assert_same(a, b):
    assert a["code"] == b["code"]
    assert a["msg"] == b["msg"]
    assert a["reps"] == b["reps"]
    assert a["time"] == b["time"]
    for x, y in zip(a["state"], b["state"]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("integ,precision", [(3, 0), (2, 0), (3, 1)])
def test_single_instance_graph_equals_host_loop(cuda_lib, integ, precision):
    from mantlepar_b200.transport import TransportConfig
    w = sy.plain_small()
    g, h = run_pair(w, TransportConfig(cfl=w.cfl, integrator=integ, precision=precision), 200)
    assert g["code"] == 0
    assert sum(r["retries"] for r in g["reps"]) > 0          # the run exercises CFL retries
    assert_same(g, h)
    # one wait for L(U^0) and one per 64 steps, against one per stage
    assert g["syncs"] <= 1 + 4 and h["syncs"] >= (4 if integ == 3 else 3) * 200


def test_single_instance_graph_small_and_noisy_meshes(cuda_lib):
    from mantlepar_b200.transport import TransportConfig
    for w in (sy.Workload(nx=7, ny=4, seed=9, noise_H=0.1), sy.Workload(nx=2, ny=2), sy.Workload(nx=3, ny=5, seed=7)):
        g, h = run_pair(w, TransportConfig(cfl=w.cfl, integrator=3), 70)
        assert_same(g, h)


def test_single_instance_end_time_and_fixed_control(cuda_lib):
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.plain_small()
    cfg = TransportConfig(cfl=w.cfl, integrator=3)
    # The end time falls inside the run: the last step lands on it, the
    # remaining reports carry dt = 0 and the end time.
    g, h = run_pair(w, cfg, 40, lambda t: t.set_time_control(Transport.CFL, 2.5e-3))
    assert g["code"] == 0 and g["time"][0] == 2.5e-3 and g["reps"][-1]["dt"] == 0.0
    assert_same(g, h)
    # Fixed control with a step below the CFL bound runs; above it, fails.
    cfg_ok = TransportConfig(cfl=w.cfl, integrator=3, dt_initial=2e-5)
    g, h = run_pair(w, cfg_ok, 20, lambda t: t.set_time_control(Transport.FIXED))
    assert g["code"] == 0
    assert_same(g, h)
    cfg_bad = TransportConfig(cfl=w.cfl, integrator=3, dt_initial=1.0)
    g, h = run_pair(w, cfg_bad, 5, lambda t: t.set_time_control(Transport.FIXED))
    assert g["code"] == 63 and b"Fixed time step exceeds" in g["msg"]
    assert_same(g, h)


def test_single_instance_failures_match(cuda_lib):
    from mantlepar_b200.transport import TransportConfig
    w = sy.plain_small()
    # dt_min above every admissible step: the retry rule gives up at once.
    g, h = run_pair(w, TransportConfig(cfl=w.cfl, integrator=3, dt_min=10.0), 5)
    assert g["code"] == 91
    assert_same(g, h)
    # A state that leaves [0, Xe] after a few steps through an inflow of
    # composition Xe: the run either fails or retries identically.
    cfg = TransportConfig(cfl=w.cfl, integrator=2, inflow_C=0.5)
    g, h = run_pair(w, cfg, 60)
    assert_same(g, h)


def test_single_instance_product_features(cuda_lib):
    import dataclasses
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.Workload(nx=24, ny=32, seed=4)
    mat = dataclasses.replace(sy.material_s(), rho=100.0, alpha0=3e-5)
    cfg = TransportConfig(material=mat, cfl=w.cfl, integrator=3, diffusivity=1e-4)

    def setup(t):
        t.set_thermal_bc((1, 1, 0, 0), (0.9, 0.2, 0.0, 0.0))
        t.set_pressure_model(Transport.LITHOSTATIC, 1.1)
        t.set_cell_velocity(*sy.cell_velocity(w))

    g, h = run_pair(w, cfg, 30, setup)
    assert g["code"] == 0
    assert_same(g, h)


def test_graph_follows_setter_changes(cuda_lib):
    """A setter between runs (thermal walls, new state) is seen by the next
    graph run exactly as by the host loop."""
    from mantlepar_b200.transport import TransportConfig
    w = sy.Workload(nx=16, ny=20, seed=6)
    cfg = TransportConfig(cfl=w.cfl, integrator=3, diffusivity=1e-4)
    res = []
    for dev in (True, False):
        t = make(w, cfg, dev)
        _, r1 = t.step(10)
        t.set_thermal_bc((1, 1, 0, 0), (0.9, 0.2, 0.0, 0.0))
        _, r2 = t.step(10)
        H, C = sy.initial_state(w)
        t.set_state(H, C)
        _, r3 = t.step(5)
        res.append((r1, r2, r3, t.get_state()))
        t.close()
    assert res[0][:3] == res[1][:3]
    for x, y in zip(res[0][3], res[1][3]):
        assert np.array_equal(x, y)


WORKLOADS = [sy.Workload(nx=20, ny=20, seed=1), sy.Workload(nx=40, ny=60, seed=5, psi_amplitude=0.15),
             sy.Workload(nx=3, ny=5, seed=7), sy.Workload(nx=64, ny=32, seed=9, noise_H=0.1),
             sy.Workload(nx=2, ny=2, seed=11, psi_amplitude=0.05)]


def batch_run(cfg, device_steps, steps, ends=None, bad=None):
    from mantlepar_b200.batch import Batch
    b = Batch(WORKLOADS, cfg)
    b.set_device_steps(device_steps)
    for i, w in enumerate(WORKLOADS):
        vs, ud = sy.face_velocity(w)
        H, C = sy.initial_state(w)
        if bad == i:
            C = C.copy()
            C[3] = 0.9
        b.set_face_velocity(i, vs, ud)
        b.set_state(i, H, C)
    for i, e in (ends or {}).items():
        b._lib.mp_batch_set_end_time(b._h, i, float(e))
    reps = b.step(steps)
    states = [b.get_state(i) for i in range(len(WORKLOADS))]
    syncs = b.host_syncs()
    b.close()
    return reps, states, syncs


@pytest.mark.parametrize("integ,precision", [(3, 0), (2, 0), (3, 1)])
def test_batch_graph_equals_host_loop(cuda_lib, integ, precision):
    from mantlepar_b200.transport import TransportConfig
    cfg = TransportConfig(cfl=0.4, integrator=integ, precision=precision)
    ends = {2: 4e-3}                      # one instance stops at its end time
    g = batch_run(cfg, True, 70, ends=ends, bad=4)
    h = batch_run(cfg, False, 70, ends=ends, bad=4)
    assert g[0] == h[0]
    for a, b in zip(g[1], h[1]):
        assert a["status"] == b["status"] and a["accepted"] == b["accepted"] and a["time"] == b["time"]
        for k in ("H", "C", "T", "phi"):
            assert np.array_equal(a[k], b[k]), k
    assert g[1][4]["status"] == 63 and g[1][2]["time"] == 4e-3
    assert sum(r[0]["retries"] for r in g[0]) > 0
    assert g[2] <= 2 + 2 and h[2] >= 3 * 70


def test_batch_graph_survives_instance_changes(cuda_lib):
    """Instances leaving and joining rewrite the batch's device records in
    place: the step graph is captured once, and the results equal the
    host-driven loop's for the same sequence of changes."""
    from mantlepar_b200.batch import Batch
    from mantlepar_b200.transport import TransportConfig
    cfg = TransportConfig(cfl=0.4, integrator=3)
    out = []
    for dev in (True, False):
        b = Batch(WORKLOADS[:3], cfg)
        b.set_device_steps(dev)
        for i, w in enumerate(WORKLOADS[:3]):
            b.set_face_velocity(i, *sy.face_velocity(w))
            b.set_state(i, *sy.initial_state(w))
        r1 = b.step(5)
        b.remove(1)
        k = b.add(WORKLOADS[3])
        b.set_face_velocity(k, *sy.face_velocity(WORKLOADS[3]))
        b.set_state(k, *sy.initial_state(WORKLOADS[3]))
        r2 = b.step(5)
        b.remove(0)
        r3 = b.step(3)
        states = [b.get_state(i) for i in (1, 2)]
        out.append((r1, r2, r3, states, b.graph_captures()))
        b.close()
    assert out[0][:3] == out[1][:3]
    for a, c in zip(out[0][3], out[1][3]):
        for key in ("H", "C", "T", "phi"):
            assert np.array_equal(a[key], c[key])
    assert out[0][4] == 1 and out[1][4] == 0


@pytest.mark.parametrize("family,integ,kappa", [(sy.MESH_PERTURBED, 3, 0.0), (sy.MESH_PERTURBED, 2, 0.0),
                                                (sy.MESH_SINE_STRETCHED, 3, 0.0), (sy.MESH_PERTURBED, 3, 0.02)])
def test_quad_mesh_graph_equals_host_loop(cuda_lib, family, integ, kappa):
    """General quad meshes (per-cell tables) step in the same graph: states,
    reports and retries equal the host-driven loop bit for bit, with one host
    wait per 64 steps; with diffusion too."""
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.Workload(nx=20, ny=24, seed=5)
    xy = sy.quad_vertices(w, family, 0.2 if family == sy.MESH_PERTURBED else 0.0, seed=11)
    cfg = TransportConfig(cfl=w.cfl, integrator=integ, diffusivity=kappa)
    out = []
    for dev in (True, False):
        t = Transport(w, cfg, vertices=xy)
        t.set_device_steps(dev)
        t.set_face_velocity(*sy.face_velocity_quads(w, xy))
        t.set_state(*sy.initial_state(w))
        code, reps = t.step(150, raise_on_error=False)
        out.append(dict(code=code, reps=reps, state=t.get_state(), time=t.get_time(), syncs=t.host_syncs(),
                        msg=t._lib.mp_last_error_string() if code else b""))
        t.close()
    g, h = out
    assert g["code"] == 0
    if kappa == 0.0:
        assert sum(r["retries"] for r in g["reps"]) > 0      # the run exercises CFL retries
    assert_same(g, h)
    assert g["syncs"] <= 1 + 3 and h["syncs"] >= (3 if integ == 3 else 2) * 150

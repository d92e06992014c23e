"""Serving: continuous batching with memory admission; every served result is
bitwise the result of the same solve run alone."""
import ctypes as C

import numpy as np
import pytest

from mantlepar_b200 import synthetic as sy

pytestmark = pytest.mark.gpu


def alone(w, tf, cfg):
    from mantlepar_b200.batch import Batch
    b = Batch([w], cfg)
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    b.set_face_velocity(0, vs, ud)
    b.set_state(0, H, C)
    b._lib.mp_batch_set_end_time(b._h, 0, tf)
    for _ in range(10000):
        if b._lib.mp_batch_finished(b._h, 0):
            break
        b.step(1)
    return b.get_state(0)


@pytest.mark.parametrize("order", [0, 1], ids=["fifo", "smallest_work"])
def test_served_results_equal_solo_runs(cuda_lib, order):
    from mantlepar_b200.batch import Batch
    from mantlepar_b200.serve import Server
    from mantlepar_b200.transport import TransportConfig
    cfg = TransportConfig(cfl=0.4, integrator=3)
    reqs = [(sy.Workload(nx=20, ny=20, seed=21), 0.02), (sy.Workload(nx=40, ny=80, seed=22), 0.004),
            (sy.Workload(nx=60, ny=60, seed=23), 0.003), (sy.Workload(nx=20, ny=40, seed=24), 0.03),
            (sy.Workload(nx=80, ny=80, seed=25), 0.002), (sy.Workload(nx=40, ny=40, seed=26), 0.01)]
    # A budget for about two of the larger requests at once forces queueing.
    budget = 2 * Batch.instance_bytes(sy.Workload(nx=80, ny=80)) + Batch.instance_bytes(sy.Workload(nx=20, ny=20))
    srv = Server(cfg, memory_budget=budget)
    # A resident target below the total forces the order to matter.
    srv.set_policy(order, 6000)
    ids = [srv.submit(w, tf) for w, tf in reqs]
    got = [srv.wait(i, timeout=120.0) for i in ids]
    st = srv.stats()
    srv.close()
    assert st["cell_updates"] > 0 and st["steps"] > 0
    assert any(g["queue_s"] > 0 for g in got)
    if order == Server.SMALLEST_WORK:
        work = [w.cells * tf * max(w.nx, w.ny) for w, tf in reqs]
        assert got[int(np.argmin(work))]["latency_s"] <= got[int(np.argmax(work))]["latency_s"]
    for (w, tf), g in zip(reqs, got):
        assert g["status"] == 0 and g["time"] == tf
        ref = alone(w, tf, cfg)
        assert g["accepted"] == ref["accepted"]
        for k in ("H", "C", "T", "phi"):
            assert np.array_equal(g[k], ref[k]), k


def test_oversized_request_is_refused(cuda_lib):
    from mantlepar_b200._capi import MPError
    from mantlepar_b200.serve import Server
    srv = Server(memory_budget=1 << 20)
    with pytest.raises(MPError) as err:
        srv.submit(sy.Workload(nx=200, ny=200), 0.01)
    assert err.value.code == 111
    with pytest.raises(MPError):
        srv.set_policy(7, 0)
    with pytest.raises(MPError):
        srv.set_policy(0, -1)
    srv.close()


def test_bounded_stream_reports_completed_and_censored(cuda_lib):
    """run_stream with a wall bound: a short stream of small solves finishes
    within it; with a bound shorter than the work, the unfinished requests
    are reported as censored and the server still shuts down cleanly."""
    from mantlepar_b200.serve import Server, poisson_requests, run_stream
    from mantlepar_b200.transport import TransportConfig
    reqs = poisson_requests(6, rate=50.0, seed=7, max_nx=60)
    srv = Server(TransportConfig(cfl=0.4, integrator=3, precision=1), memory_budget=1 << 30)
    out = run_stream(srv, reqs, wall_limit=120.0)
    srv.close()
    assert out["completed"] == 6 and out["censored"] == 0 and out["all_ok"]
    assert out["p50_ms"] <= out["p99_ms"] and out["service_p50_ms"] > 0
    big = poisson_requests(4, rate=50.0, seed=8, max_nx=1280)
    srv = Server(TransportConfig(cfl=0.4, integrator=3, precision=1), memory_budget=8 << 30)
    out = run_stream(srv, big, wall_limit=1.0)
    srv.close()
    assert out["completed"] + out["censored"] == 4 and out["censored"] >= 1


def alone_quads(w, xy, tf, cfg):
    """The same quad-mesh solve run alone, one step per call as the server
    steps it."""
    from mantlepar_b200.transport import Transport
    t = Transport(w, cfg, vertices=xy)
    t.set_face_velocity(*sy.face_velocity_quads(w, xy))
    t.set_state(*sy.initial_state(w))
    t.set_time_control(0, tf)
    for _ in range(10000):
        if t.get_time()[0] >= tf:
            break
        t.step(1)
    H, C, T, phi = t.get_state()
    time, acc = t.get_time()
    t.close()
    return dict(H=H, C=C, T=T, phi=phi, time=time, accepted=acc)


def test_served_quad_mesh_requests_equal_solo_runs(cuda_lib):
    """Perturbed-quadrilateral and sine-stretched requests (the reference's
    mesh families) served beside uniform ones under a budget that queues
    them: each quad result is bitwise the solo quad transport's, each uniform
    result the solo batch's, and a folded quad mesh ends only its own request
    with MP_ERR_ARG_WRONG."""
    from mantlepar_b200.serve import Server
    from mantlepar_b200.transport import TransportConfig
    from mantlepar_b200 import _capi
    cfg = TransportConfig(cfl=0.4, integrator=3)
    quads = [(sy.Workload(nx=20, ny=20, seed=31), sy.MESH_PERTURBED, 0.01),
             (sy.Workload(nx=24, ny=16, seed=32), sy.MESH_SINE_STRETCHED, 0.005),
             (sy.Workload(nx=16, ny=32, seed=33), sy.MESH_PERTURBED, 0.008)]
    uniform = [(sy.Workload(nx=20, ny=20, seed=34), 0.02), (sy.Workload(nx=40, ny=40, seed=35), 0.005)]
    big = max(_capi.lib().mp_transport_instance_bytes(C.byref(_capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)), 1)
              for w, _, _ in quads)
    srv = Server(cfg, memory_budget=2 * big)
    ids = []
    for k, (w, fam, tf) in enumerate(quads):
        xy = sy.quad_vertices(w, fam, 0.2 if fam == sy.MESH_PERTURBED else 0.0, seed=11 + k)
        ids.append(("q", w, xy, tf, srv.submit(w, tf, vertices=xy)))
        uw, utf = uniform[k % len(uniform)]
        if k < len(uniform):
            ids.append(("u", uw, None, utf, srv.submit(uw, utf)))
    wb = sy.Workload(nx=4, ny=4)
    bad = sy.quad_vertices(wb, sy.MESH_RECTANGULAR).reshape(5, 5, 2).copy()
    bad[2, 2] = bad[3, 3] + [0.01, 0.01]
    bad_id = srv.submit(wb, 0.01, vertices=bad.reshape(-1), vs=np.zeros(40 * 5), ud=np.zeros(40 * 5))
    got = {rid: srv.wait(rid, timeout=300.0) for *_, rid in ids}
    bad_res = srv.wait(bad_id, timeout=60.0)
    st = srv.stats()
    srv.close()
    assert bad_res["status"] == 62
    assert st["cell_updates"] > 0
    for kind, w, xy, tf, rid in ids:
        g = got[rid]
        assert g["status"] == 0 and g["time"] == tf, (kind, g["status"], g["time"])
        ref = alone_quads(w, xy, tf, cfg) if kind == "q" else alone(w, tf, cfg)
        assert g["accepted"] == ref["accepted"]
        for k in ("H", "C", "T", "phi"):
            assert np.array_equal(g[k], ref[k]), (kind, k)


def test_transport_instance_bytes_covers_the_allocation(cuda_lib):
    """The serving budget of a request (mp_transport_instance_bytes) covers
    what creating its transport takes from the device, uniform and quad
    mesh, and is not far above it (the quad estimate adds the builder's
    transient copy of the vertices). The first quad-mesh transport of a
    process also raises the runtime's per-thread stack reservation for the
    table builder (2.7 KB a thread), once for the process: a small quad
    transport is made first, so that the measurement sees one request."""
    import torch
    from mantlepar_b200 import _capi
    from mantlepar_b200.transport import Transport, TransportConfig
    lib = _capi.lib()
    w = sy.Workload(nx=512, ny=1024)
    mesh = _capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)
    w0 = sy.Workload(nx=8, ny=8)
    Transport(w0, TransportConfig(cfl=0.4, integrator=3), vertices=sy.quad_vertices(w0, sy.MESH_PERTURBED)).close()
    for quads in (0, 1):
        xy = sy.quad_vertices(w, sy.MESH_PERTURBED) if quads else None
        est = lib.mp_transport_instance_bytes(C.byref(mesh), quads)
        steady = est - ((2 * (w.nx + 1) * (w.ny + 1) * 8 + 4 + (2 << 20) - 1) // (2 << 20) * (2 << 20) if quads else 0)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        t = Transport(w, TransportConfig(cfl=0.4, integrator=3), vertices=xy)
        torch.cuda.synchronize()
        used = free0 - torch.cuda.mem_get_info()[0]
        t.close()
        print(f"quads={quads}: estimate {est / 2**20:.1f} MiB, taken {used / 2**20:.1f} MiB")
        assert used <= est, (quads, used, est)
        assert used >= 0.8 * steady, (quads, used, steady)

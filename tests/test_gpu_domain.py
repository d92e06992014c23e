"""Row-slab decomposition on one GPU: the slabs of one mesh, run as host
threads with halo copies and combined totals (ThreadExchange), reproduce the
single-domain run cell for cell -- the same dt and retry sequence and bitwise
equal H, C, T, phi."""
import numpy as np
import pytest
import torch

from mantlepar_b200 import synthetic as sy

pytestmark = pytest.mark.gpu


def single(w, cfg, steps):
    from mantlepar_b200.transport import Transport
    t = Transport(w, cfg)
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    _, reps = t.step(steps)
    return np.stack(t.get_state()), reps


def decomposed(w, cfg, steps, parts):
    from mantlepar_b200.domain import Slab, ThreadExchange, partition
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    slabs = [Slab(w, r, cfg, stream=torch.cuda.Stream()) for r in partition(w.ny, parts)]
    for s in slabs:
        s.set_face_velocity(vs, ud)
        s.set_state(H, C)
    ex = ThreadExchange(slabs)
    out = ex.step(steps)
    state = np.concatenate([np.stack(s.get_state()) for s in slabs], axis=1)
    return state, out


@pytest.mark.parametrize("integ,parts", [(3, 2), (2, 3), (3, 4)])
def test_slabs_reproduce_single_domain(cuda_lib, integ, parts):
    from mantlepar_b200.transport import TransportConfig
    w = sy.Workload(nx=24, ny=30, seed=5, noise_H=0.1)
    cfg = TransportConfig(cfl=0.4, integrator=integ)
    ref, reps = single(w, cfg, 12)
    got, outs = decomposed(w, cfg, 12, parts)
    for code, r in outs:
        assert code == 0
        assert [x["dt"] for x in r] == [x["dt"] for x in reps]
        assert [x["retries"] for x in r] == [x["retries"] for x in reps]
    assert sum(x["retries"] for x in reps) > 0          # the retry path is exercised
    for k, name in enumerate(["H", "C", "T", "phi"]):
        assert np.array_equal(got[k], ref[k]), name


def test_slabs_mixed_precision(cuda_lib):
    from mantlepar_b200.transport import TransportConfig
    w = sy.Workload(nx=32, ny=40, seed=2)
    cfg = TransportConfig(cfl=0.4, integrator=3, precision=1)
    ref, _ = single(w, cfg, 6)
    got, _ = decomposed(w, cfg, 6, 3)
    assert np.array_equal(got, ref)


def test_dist_exchange_hooks_with_one_nccl_rank(cuda_lib):
    """DistExchange wired into a slab's hooks over a one-rank NCCL group: the
    callbacks, device views and collectives run, and the result equals the
    single-domain run (with one rank the slab is the whole mesh)."""
    import os
    import socket
    import torch.distributed as dist
    from mantlepar_b200.domain import DistExchange, Slab, partition
    from mantlepar_b200.transport import TransportConfig
    w = sy.Workload(nx=20, ny=24, seed=3)
    cfg = TransportConfig(cfl=0.4, integrator=3)
    ref, reps = single(w, cfg, 5)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    store = dist.TCPStore("127.0.0.1", port, 1, True)
    dist.init_process_group("nccl", store=store, rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        rows = partition(w.ny, 1)
        slab = Slab(w, rows[0], cfg)
        vs, ud = sy.face_velocity(w)
        H, C = sy.initial_state(w)
        slab.set_face_velocity(vs, ud)
        slab.set_state(H, C)
        DistExchange(0, 1, rows, w.nx, device=torch.device("cuda", 0)).attach(slab)
        code, got_reps = slab.step(5)
        assert code == 0
        assert [x["dt"] for x in got_reps] == [x["dt"] for x in reps]
        assert np.array_equal(np.stack(slab.get_state()), ref)
        slab.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("parts", [2, 3])
def test_quad_slabs_reproduce_single_domain(cuda_lib, parts):
    """Row slabs of a perturbed-quadrilateral mesh (each slab's cell tables
    built from the whole mesh) reproduce the single quad run bit for bit,
    with thermal diffusion on."""
    from mantlepar_b200.domain import Slab, ThreadExchange, partition
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.Workload(nx=20, ny=26, seed=8, noise_H=0.1)
    xy = sy.quad_vertices(w, sy.MESH_PERTURBED, 0.2, 7)
    vs, ud = sy.face_velocity_quads(w, xy)
    H, C = sy.initial_state(w)
    cfg = TransportConfig(cfl=0.4, integrator=3, diffusivity=5e-3)
    bc = ((1, 1, 0, 2), (0.6, 0.2, 0.0, 0.01))
    t = Transport(w, cfg, vertices=xy)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    t.set_thermal_bc(*bc)
    _, reps = t.step(10)
    ref = np.stack(t.get_state())
    slabs = [Slab(w, r, cfg, stream=torch.cuda.Stream(), vertices=xy) for r in partition(w.ny, parts)]
    for s in slabs:
        s.set_face_velocity(vs, ud)
        s.set_state(H, C)
        s.set_thermal_bc(*bc)
    outs = ThreadExchange(slabs).step(10)
    got = np.concatenate([np.stack(s.get_state()) for s in slabs], axis=1)
    for code, r in outs:
        assert code == 0
        assert [x["dt"] for x in r] == [x["dt"] for x in reps]
    for k, name in enumerate(["H", "C", "T", "phi"]):
        assert np.array_equal(got[k], ref[k]), name

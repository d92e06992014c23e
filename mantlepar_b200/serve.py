"""Serving: a request loop for transport solves of different sizes.

`Server` wraps mp_serve_* (C++ loop thread, memory admission, continuous
batching). `poisson_requests` draws the served workload: Poisson arrivals
(mean 200 req/s), nx in {20..1280 step 20}, ny = nx * U{1,2}, final time
U[0.01, 0.1], initial H/C as the 20x20 workload's construction.
`run_stream` submits each request at its arrival time from a client thread
and returns per-request latencies and the aggregate throughput.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import threading
import time

import numpy as np

from . import _capi
from .synthetic import Workload, face_velocity, face_velocity_quads, initial_state
from .transport import TransportConfig


@dataclasses.dataclass
class Request:
    arrival: float
    workload: Workload
    t_final: float


def poisson_requests(n: int, rate: float = 200.0, seed: int = 4, max_nx: int = 1280) -> list[Request]:
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        nx = int(rng.integers(1, max_nx // 20 + 1)) * 20
        ny = nx * int(rng.integers(1, 3))
        tf = float(rng.uniform(0.01, 0.1))
        out.append(Request(t, Workload(nx=nx, ny=ny, seed=100 + k), tf))
    return out


class Server:
    def __init__(self, config: TransportConfig | None = None, memory_budget: int = 16 << 30):
        self._lib = _capi.lib()
        self.config = config or TransportConfig()
        opts = self.config.to_c()
        h = C.c_void_p()
        _capi.check(self._lib.mp_serve_create(C.byref(opts), C.c_size_t(memory_budget), C.byref(h)))
        self._h = h
        self._cells = {}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mp_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, w: Workload, t_final: float, H=None, Cc=None, vs=None, ud=None, vertices=None) -> int:
        """Queue one solve. vertices ((nx+1)*(ny+1) (x, y) pairs) makes it a
        general-quad-mesh request (mp_serve_submit_quads); its face velocities
        then belong to that mesh's edges."""
        if H is None:
            H, Cc = initial_state(w)
        if vs is None:
            vs, ud = face_velocity(w) if vertices is None else face_velocity_quads(w, vertices)
        m = _capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (H, Cc, vs, ud)]
        rid = C.c_longlong(0)
        if vertices is None:
            _capi.check(self._lib.mp_serve_submit(self._h, C.byref(m), *[a.ctypes.data for a in arrs],
                                                  float(t_final), C.byref(rid)))
        else:
            xy = np.ascontiguousarray(vertices, dtype=np.float64)
            if xy.size != 2 * (w.nx + 1) * (w.ny + 1):
                raise ValueError("vertices must hold (nx+1)*(ny+1) (x, y) pairs")
            _capi.check(self._lib.mp_serve_submit_quads(self._h, C.byref(m), xy.ctypes.data,
                                                        *[a.ctypes.data for a in arrs], float(t_final), C.byref(rid)))
        self._cells[rid.value] = w.cells
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0):
        n = self._cells.pop(rid)
        H, Cc, T, phi = (np.zeros(n) for _ in range(4))
        info = _capi.RequestInfo()
        _capi.check(self._lib.mp_serve_wait(self._h, C.c_longlong(rid), float(timeout), H.ctypes.data,
                                            Cc.ctypes.data, T.ctypes.data, phi.ctypes.data, C.byref(info)))
        return dict(H=H, C=Cc, T=T, phi=phi, **{k: getattr(info, k) for k, _ in _capi.RequestInfo._fields_})

    FIFO, SMALLEST_WORK = 0, 1

    def set_policy(self, order: int, resident_cells_target: float):
        _capi.check(self._lib.mp_serve_set_policy(self._h, int(order), float(resident_cells_target)))

    def stats(self):
        cu, busy, steps, res, q = C.c_double(0), C.c_double(0), C.c_longlong(0), C.c_int(0), C.c_int(0)
        _capi.check(self._lib.mp_serve_stats(self._h, C.byref(cu), C.byref(busy), C.byref(steps), C.byref(res), C.byref(q)))
        return dict(cell_updates=cu.value, busy_s=busy.value, steps=steps.value, resident=res.value, queued=q.value)


def prepare_inputs(requests: list[Request]):
    """Inputs of every request, built before a stream starts: the cell
    averages per request, the face velocities once per distinct mesh (they
    depend on the mesh and the flow amplitude only)."""
    flows = {}
    inputs = []
    for r in requests:
        w = r.workload
        key = (w.nx, w.ny, w.x0, w.x1, w.y0, w.y1, w.psi_amplitude, w.darcy)
        if key not in flows:
            flows[key] = face_velocity(w)
        inputs.append((initial_state(w), flows[key]))
    return inputs


def input_bytes(r: Request) -> int:
    """Host bytes of one request's inputs (H, C and the two face-velocity arrays)."""
    return 8 * (2 * r.workload.cells + 10 * r.workload.edges)


def run_stream(server: Server, requests: list[Request], wall_limit: float | None = None) -> dict:
    """Submit each request at its arrival time from a client thread (inputs
    are built before the clock starts); wait for the results.

    wall_limit: stop waiting that many seconds after the first arrival;
    requests not finished by then are reported as censored (their latency
    is at least the time they waited). Latencies in ms; queue = submit to
    admission, service = admission to result."""
    inputs = prepare_inputs(requests)
    ids = [None] * len(requests)
    submit_at = [None] * len(requests)
    t0 = time.perf_counter()

    def client():
        for k, r in enumerate(requests):
            delay = r.arrival - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            if wall_limit is not None and time.perf_counter() - t0 > wall_limit:
                return
            (H, Cc), (vs, ud) = inputs[k]
            ids[k] = server.submit(r.workload, r.t_final, H, Cc, vs, ud)
            submit_at[k] = time.perf_counter() - t0

    th = threading.Thread(target=client)
    th.start()
    th.join()
    results, censored = [], []
    for k, rid in enumerate(ids):
        if rid is None:
            censored.append(0.0)
            continue
        left = -1.0 if wall_limit is None else max(0.0, wall_limit - (time.perf_counter() - t0))
        try:
            results.append(server.wait(rid, timeout=left))
        except _capi.MPError as e:
            if e.code != 110:
                raise
            censored.append((time.perf_counter() - t0 - submit_at[k]) * 1e3)
    wall = time.perf_counter() - t0
    stats = server.stats()
    pct = lambda a, q: float(np.percentile(a, q)) if len(a) else None
    lat = np.array([r["latency_s"] for r in results]) * 1e3
    queue = np.array([r["queue_s"] for r in results]) * 1e3
    service = lat - queue
    submitted = [x for x in submit_at if x is not None]
    return dict(requests=len(requests), completed=len(results), censored=len(censored),
                submit_span_s=float(max(submitted)) if submitted else None,
                censored_min_latency_ms=float(min(censored)) if censored else None, wall_s=wall,
                p50_ms=pct(lat, 50), p99_ms=pct(lat, 99), mean_ms=float(lat.mean()) if len(lat) else None,
                queue_p50_ms=pct(queue, 50), queue_p99_ms=pct(queue, 99),
                service_p50_ms=pct(service, 50), service_p99_ms=pct(service, 99),
                cell_updates=stats["cell_updates"], value=stats["cell_updates"] / wall,
                gpu_busy_value=stats["cell_updates"] / max(stats["busy_s"], 1e-12),
                all_ok=all(r["status"] == 0 for r in results), results=results)


def request_work(r: Request) -> float:
    """Cell-updates of a request on this construction: about 24 nx t_final
    accepted steps (CFL 0.4 at a stage rate of about 9.5 nx) of nx*ny cells."""
    return 24.0 * r.workload.nx * r.t_final * r.workload.cells

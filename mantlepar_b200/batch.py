"""Batched transport: many independent uneven meshes advanced together.

Thin wrapper of the mp_batch_* C ABI. Every instance keeps the reference's
per-mesh semantics (own dt, retries, balance check, rollback); results are
bitwise those of a single-instance run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi
from .synthetic import Workload
from .transport import REPORT_FIELDS, TransportConfig, _host, _ptr


def mesh_of(w: Workload) -> _capi.MeshDesc:
    return _capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)


class Batch:
    def __init__(self, workloads: list[Workload], config: TransportConfig | None = None, stream=None):
        self._lib = _capi.lib()
        self.config = config or TransportConfig()
        meshes = (_capi.MeshDesc * max(1, len(workloads)))(*[mesh_of(w) for w in workloads])
        opts = self.config.to_c()
        h = C.c_void_p()
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        _capi.check(self._lib.mp_batch_create(meshes, len(workloads), C.byref(opts), s, C.byref(h)))
        self._h = h
        self.cells = {i: w.cells for i, w in enumerate(workloads)}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def slots(self) -> int:
        return self._lib.mp_batch_slots(self._h)

    def bytes_in_use(self) -> int:
        return int(self._lib.mp_batch_bytes_in_use(self._h))

    @staticmethod
    def instance_bytes(w: Workload) -> int:
        m = mesh_of(w)
        return int(_capi.lib().mp_batch_instance_bytes(C.byref(m)))

    def add(self, w: Workload) -> int:
        m = mesh_of(w)
        slot = C.c_int(-1)
        _capi.check(self._lib.mp_batch_add(self._h, C.byref(m), C.byref(slot)))
        self.cells[slot.value] = w.cells
        return slot.value

    def add_quads(self, w: Workload, vertices) -> int:
        """An instance on a general quad mesh: vertices holds the
        (nx+1)*(ny+1) (x, y) pairs (mp_batch_add_quads)."""
        m = mesh_of(w)
        xy = np.ascontiguousarray(vertices, dtype=np.float64)
        if xy.size != 2 * (w.nx + 1) * (w.ny + 1):
            raise ValueError("vertices must hold (nx+1)*(ny+1) (x, y) pairs")
        slot = C.c_int(-1)
        _capi.check(self._lib.mp_batch_add_quads(self._h, C.byref(m), xy.ctypes.data, C.byref(slot)))
        self.cells[slot.value] = w.cells
        return slot.value

    def remove(self, i: int):
        _capi.check(self._lib.mp_batch_remove(self._h, int(i)))
        self.cells.pop(i, None)

    def set_face_velocity(self, i: int, vs_n, ud_n):
        vs, ud = _host(vs_n), _host(ud_n)
        _capi.check(self._lib.mp_batch_set_face_velocity(self._h, int(i), _ptr(vs), _ptr(ud)))

    def set_state(self, i: int, H, Cc, time: float = 0.0):
        Hh, Ch = _host(H), _host(Cc)
        _capi.check(self._lib.mp_batch_set_state(self._h, int(i), _ptr(Hh), _ptr(Ch), float(time)))

    def get_state(self, i: int):
        n = self.cells[i]
        H, Cc, T, phi = (np.zeros(n) for _ in range(4))
        t, acc, st = C.c_double(0), C.c_int(0), C.c_int(0)
        _capi.check(self._lib.mp_batch_get_state(self._h, int(i), _ptr(H), _ptr(Cc), _ptr(T), _ptr(phi),
                                                 C.byref(t), C.byref(acc), C.byref(st)))
        return dict(H=H, C=Cc, T=T, phi=phi, time=t.value, accepted=acc.value, status=st.value)

    def info(self, i: int):
        t, acc, st = C.c_double(0), C.c_int(0), C.c_int(0)
        _capi.check(self._lib.mp_batch_get_state(self._h, int(i), None, None, None, None,
                                                 C.byref(t), C.byref(acc), C.byref(st)))
        return dict(time=t.value, accepted=acc.value, status=st.value)

    def set_thermal_bc(self, types=(0, 0, 0, 0), values=(0.0, 0.0, 0.0, 0.0)):
        ti = (C.c_int * 4)(*[int(x) for x in types])
        tv = (C.c_double * 4)(*[float(x) for x in values])
        _capi.check(self._lib.mp_batch_set_thermal_bc(self._h, ti, tv))

    def step(self, nsteps: int = 1):
        slots = self.slots
        reps = (_capi.StepReport * max(1, nsteps * slots))()
        _capi.check(self._lib.mp_batch_step(self._h, int(nsteps), reps))
        return [[{k: getattr(reps[s * slots + i], k) for k in REPORT_FIELDS} for i in range(slots)]
                for s in range(nsteps)]

    def set_cell_velocity(self, i: int, vs_y, ud_y):
        """Vertical solid / Darcy velocity at instance i's cell quadrature
        points [cell*25 + b*5 + a] (adiabatic source, alpha0 != 0)."""
        a, b = _host(vs_y), _host(ud_y)
        _capi.check(self._lib.mp_batch_set_cell_velocity(self._h, int(i), _ptr(a), _ptr(b)))

    def set_device_steps(self, enable: bool = True):
        """step() as CUDA graphs with every instance's step decisions on the
        device (default) or as the host-driven loop."""
        _capi.check(self._lib.mp_batch_set_device_steps(self._h, int(enable)))

    def host_syncs(self) -> int:
        """Host waits for device results made by step() so far."""
        n = C.c_ulonglong(0)
        _capi.check(self._lib.mp_batch_run_stats(self._h, C.byref(n), None))
        return n.value

    def graph_captures(self) -> int:
        """Times the step graph was captured so far."""
        n = C.c_ulonglong(0)
        _capi.check(self._lib.mp_batch_run_stats(self._h, None, C.byref(n)))
        return n.value

    def autotune(self, reps: int = 2):
        tile = (C.c_int * 3)()
        best = C.c_double(0)
        _capi.check(self._lib.mp_batch_autotune(self._h, int(reps), tile, C.byref(best)))
        return tuple(tile), best.value

    def profile(self, enable: bool):
        _capi.check(self._lib.mp_batch_profile(self._h, int(enable)))

    def kernel_times(self):
        ms = (C.c_double * 6)()
        n = (C.c_ulonglong * 6)()
        _capi.check(self._lib.mp_batch_kernel_times(self._h, ms, n))
        return list(ms), list(n)

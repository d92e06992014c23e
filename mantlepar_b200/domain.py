"""Row-slab domain decomposition of one large transport instance.

The mesh is cut into row slabs (the reference partitions its cell DMDA the
same way, src/couple/state_reconstruction.cpp:40-58); each slab is a
`mp_transport_create_slab` instance holding its owned rows plus up to two
halo rows each side. Before every stage the halo hook copies the neighbours'
owned rows of the stage input into the halo rows (2 x nx x 2 fields doubles
per neighbour); after every reduction the combine hook reduces the stage
totals across slabs (max / min / sum, status: min) so that every slab takes
the same dt, retry and admissibility decisions. A decomposed run gives the
single-domain run's H, C, T and phi cell for cell.

Two exchanges implement the hooks:

* `DistExchange` -- one slab per process over `torch.distributed`: point to
  point sends of halo rows and all-reduces of the totals (NCCL on GPUs; the
  same code runs on gloo with CPU tensors);
* `ThreadExchange` -- all slabs of one process on one GPU, one host thread
  each; halo rows are device-to-device copies and the totals are combined
  in slab order under a host barrier (no kernel waits for another).

Every slab owns at least two rows, so halo rows come from the neighbouring
slabs only.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np
import torch

from . import _capi
from .synthetic import Workload
from .transport import REPORT_FIELDS, TransportConfig, _host, _ptr

NONE_KEY = (1 << 63) - 1          # "no failure" status key as int64
MAX_FIELDS = (0, 1, 8, 9)         # maxRate, divergence, Cmax, nonfinite
MIN_FIELDS = (6, 7)               # Hmin, Cmin
SUM_FIELDS = (2, 3, 4, 5, 10)     # boundaryH, boundaryC, H_integral, C_integral, sourceH
NFIELDS = 11


def partition(ny: int, parts: int) -> list[tuple[int, int]]:
    """Balanced row ranges [begin, end), each of at least two rows."""
    if parts < 1 or ny < 2 * parts:
        raise ValueError(f"{ny} rows cannot form {parts} slabs of at least two rows")
    base, extra = divmod(ny, parts)
    out, j = [], 0
    for k in range(parts):
        n = base + (1 if k < extra else 0)
        out.append((j, j + n))
        j += n
    return out


def combine_totals(parts: list[np.ndarray], statuses: list[int]) -> tuple[np.ndarray, int]:
    """Totals and status of all slabs in slab order (the reduction every slab applies)."""
    out = np.array(parts[0], dtype=np.float64)
    for p in parts[1:]:
        for k in MAX_FIELDS:
            out[k] = max(out[k], p[k])
        for k in MIN_FIELDS:
            out[k] = min(out[k], p[k])
        for k in SUM_FIELDS:
            out[k] = out[k] + p[k]
    return out, min(statuses)


class _DeviceArray:
    """A raw device buffer seen as a torch tensor (no copy)."""

    def __init__(self, ptr: int, n: int, device: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3}
        self.device = device


def device_view(ptr: int, n: int, device: int) -> torch.Tensor:
    return torch.as_tensor(_DeviceArray(ptr, n, device), device=f"cuda:{device}")


class Slab:
    """One row slab of a global mesh on the current GPU."""

    def __init__(self, w: Workload, rows: tuple[int, int], config: TransportConfig | None = None, stream=None,
                 vertices=None):
        """vertices: the whole mesh's (nx+1)*(ny+1) (x, y) pairs for a general
        quad mesh (mp_transport_create_quads_slab); None for the uniform mesh."""
        self._lib = _capi.lib()
        self.w = w
        self.rows = rows
        self.config = config or TransportConfig(cfl=w.cfl, integrator=w.integrator)
        mesh = _capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)
        opts = self.config.to_c()
        h = C.c_void_p()
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        if vertices is None:
            _capi.check(self._lib.mp_transport_create_slab(C.byref(mesh), int(rows[0]), int(rows[1]), C.byref(opts),
                                                            self.stream.cuda_stream, C.byref(h)))
        else:
            xy = np.ascontiguousarray(vertices, dtype=np.float64)
            _capi.check(self._lib.mp_transport_create_quads_slab(C.byref(mesh), xy.ctypes.data, int(rows[0]),
                                                                  int(rows[1]), C.byref(opts), self.stream.cuda_stream,
                                                                  C.byref(h)))
        self._h = h
        lr, r0, o0, o1 = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _capi.check(self._lib.mp_transport_slab_layout(h, C.byref(lr), C.byref(r0), C.byref(o0), C.byref(o1)))
        self.local_rows, self.row0, self.own0, self.own1 = lr.value, r0.value, o0.value, o1.value
        self._hooks = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mp_transport_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- data in the global numbering, sliced to this slab
    def local_edges(self, a: np.ndarray) -> np.ndarray:
        """Rows of a global [edge, 5] array that belong to the local mesh."""
        nx, ny = self.w.nx, self.w.ny
        nI = nx * (ny + 1)
        a = np.asarray(a).reshape(-1, 5)
        h = a[self.row0 * nx:(self.row0 + self.local_rows + 1) * nx]
        v = a[nI + self.row0 * (nx + 1):nI + (self.row0 + self.local_rows) * (nx + 1)]
        return np.ascontiguousarray(np.concatenate([h, v]))

    def owned(self, a: np.ndarray) -> np.ndarray:
        nx = self.w.nx
        return np.ascontiguousarray(np.asarray(a)[self.rows[0] * nx:self.rows[1] * nx])

    def set_face_velocity(self, vs_global, ud_global):
        vs, ud = self.local_edges(vs_global), self.local_edges(ud_global)
        _capi.check(self._lib.mp_transport_set_face_velocity(self._h, _ptr(vs), _ptr(ud)))

    def set_state(self, H_global, C_global, time: float = 0.0):
        H, Cc = _host(self.owned(H_global)), _host(self.owned(C_global))
        _capi.check(self._lib.mp_transport_set_state(self._h, _ptr(H), _ptr(Cc), float(time)))

    def get_state(self):
        n = (self.rows[1] - self.rows[0]) * self.w.nx
        H, Cc, T, phi = (np.zeros(n) for _ in range(4))
        _capi.check(self._lib.mp_transport_get_state(self._h, _ptr(H), _ptr(Cc), _ptr(T), _ptr(phi)))
        return H, Cc, T, phi

    def set_pressure_model(self, model: int, value: float):
        _capi.check(self._lib.mp_transport_set_pressure_model(self._h, int(model), float(value)))

    def set_cell_velocity(self, vs_y_global, ud_y_global):
        """Cell-point vertical velocities of the global mesh, sliced to the local cells."""
        nx, q = self.w.nx, 25
        lo, hi = self.row0 * nx * q, (self.row0 + self.local_rows) * nx * q
        a = np.ascontiguousarray(np.asarray(vs_y_global)[lo:hi])
        b = np.ascontiguousarray(np.asarray(ud_y_global)[lo:hi])
        _capi.check(self._lib.mp_transport_set_cell_velocity(self._h, _ptr(a), _ptr(b)))

    def set_thermal_bc(self, types=(0, 0, 0, 0), values=(0.0, 0.0, 0.0, 0.0)):
        """Thermal conditions per wall (bottom, top, left, right) of the GLOBAL mesh."""
        ti = (C.c_int * 4)(*[int(x) for x in types])
        tv = (C.c_double * 4)(*[float(x) for x in values])
        _capi.check(self._lib.mp_transport_set_thermal_bc(self._h, ti, tv))

    def set_hooks(self, halo, combine):
        """halo(H_ptr, C_ptr) -> int, combine(totals: ndarray[10] view, status: list[int]) -> int."""
        def _halo(user, H, Cc):
            try:
                return int(halo(int(H), int(Cc)))
            except Exception:
                return 112   # MP_ERR_CUDA

        def _combine(user, tot, status):
            try:
                arr = np.ctypeslib.as_array(C.cast(tot, C.POINTER(C.c_double)), shape=(NFIELDS,))
                st = [int(status[0])]
                rc = int(combine(arr, st))
                status[0] = st[0]
                return rc
            except Exception:
                return 112

        HALO = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)
        COMB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_ulonglong))
        self._hooks = (HALO(_halo), COMB(_combine))      # kept alive with the slab
        fp = [C.cast(f, C.c_void_p).value for f in self._hooks]
        _capi.check(self._lib.mp_transport_set_hooks(self._h, fp[0], fp[1], None))

    def step(self, nsteps: int):
        reps = (_capi.StepReport * max(1, nsteps))()
        code = self._lib.mp_transport_step(self._h, int(nsteps), reps)
        return code, [{k: getattr(r, k) for k in REPORT_FIELDS} for r in reps[:nsteps]]

    # halo geometry in local rows: (local destination row, global source row)
    def halo_rows(self):
        out = []
        for r in range(0, self.own0):
            out.append((r, self.row0 + r))
        for r in range(self.own1, self.local_rows):
            out.append((r, self.row0 + r))
        return out


def _status_in(st: int) -> int:
    return NONE_KEY if st == (1 << 64) - 1 else st


def _status_out(st: int) -> int:
    return (1 << 64) - 1 if st == NONE_KEY else st


class ThreadExchange:
    """All slabs of one mesh in this process and on one GPU, one thread each."""

    def __init__(self, slabs: list[Slab]):
        self.slabs = slabs
        self.n = len(slabs)
        # A slab that stops answering breaks the barrier: its peers' hooks
        # then fail with an error instead of waiting for ever.
        self.barrier = threading.Barrier(self.n, timeout=120.0)
        self.inputs: list[tuple[int, int] | None] = [None] * self.n
        self.parts: list[np.ndarray | None] = [None] * self.n
        self.status: list[int] = [0] * self.n
        self.result: tuple[np.ndarray, int] | None = None
        self.owner = {}
        for k, s in enumerate(slabs):
            for g in range(s.rows[0], s.rows[1]):
                self.owner[g] = k
        for k, s in enumerate(slabs):
            s.set_hooks(lambda H, Cc, k=k: self._halo(k, H, Cc),
                        lambda tot, st, k=k: self._combine(k, tot, st))

    def _halo(self, k: int, H: int, Cc: int) -> int:
        s = self.slabs[k]
        nx = s.w.nx
        dev = torch.cuda.current_device()
        self.inputs[k] = (H, Cc)
        self.barrier.wait()
        with torch.cuda.stream(s.stream):
            for dst_row, g in s.halo_rows():
                m = self.owner[g]
                src = self.slabs[m]
                sH, sC = self.inputs[m]
                src_row = g - src.row0
                for dptr, sptr in ((H, sH), (Cc, sC)):
                    d = device_view(dptr + 8 * dst_row * nx, nx, dev)
                    d.copy_(device_view(sptr + 8 * src_row * nx, nx, dev))
        s.stream.synchronize()
        self.barrier.wait()
        return 0

    def _combine(self, k: int, tot: np.ndarray, st: list) -> int:
        self.parts[k] = np.array(tot)
        self.status[k] = _status_in(st[0])
        if self.barrier.wait() == 0:
            self.result = combine_totals(self.parts, self.status)
        self.barrier.wait()
        tot[:] = self.result[0]
        st[0] = _status_out(self.result[1])
        self.barrier.wait()
        return 0

    def step(self, nsteps: int):
        out = [None] * self.n

        def run(k):
            with torch.cuda.stream(self.slabs[k].stream):
                out[k] = self.slabs[k].step(nsteps)

        threads = [threading.Thread(target=run, args=(k,)) for k in range(self.n)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        return out


class DistExchange:
    """One slab per process over torch.distributed (NCCL on GPUs, gloo on CPU)."""

    def __init__(self, rank: int, world: int, rows: list[tuple[int, int]], nx: int, group=None, device=None):
        import torch.distributed as dist
        self.dist = dist
        self.rank, self.world, self.rows, self.nx = rank, world, rows, nx
        self.group = group
        self.device = device if device is not None else torch.device("cpu")

    def exchange(self, H: torch.Tensor, Cc: torch.Tensor, row0: int, own0: int, own1: int, local_rows: int):
        """Fill the halo rows of local arrays H, Cc ([local_rows * nx]) from the
        neighbours' owned rows; send this slab's boundary rows to them."""
        dist, nx, ops = self.dist, self.nx, []
        recv_lo = own0 if self.rank > 0 else 0
        recv_hi = local_rows - own1 if self.rank < self.world - 1 else 0
        bufs = []
        for f in (H, Cc):
            if self.rank > 0 and recv_lo:
                send = f[own0 * nx:(own0 + recv_lo) * nx].contiguous()
                recv = torch.empty(recv_lo * nx, dtype=f.dtype, device=f.device)
                ops += [dist.P2POp(dist.isend, send, self.rank - 1, self.group),
                        dist.P2POp(dist.irecv, recv, self.rank - 1, self.group)]
                bufs.append((f, 0, recv))
            if self.rank < self.world - 1 and recv_hi:
                send = f[(own1 - recv_hi) * nx:own1 * nx].contiguous()
                recv = torch.empty(recv_hi * nx, dtype=f.dtype, device=f.device)
                ops += [dist.P2POp(dist.isend, send, self.rank + 1, self.group),
                        dist.P2POp(dist.irecv, recv, self.rank + 1, self.group)]
                bufs.append((f, own1, recv))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for f, row, recv in bufs:
            f[row * nx:row * nx + recv.numel()].copy_(recv)

    def combine(self, tot: np.ndarray, st: list) -> int:
        """One all-gather of every slab's totals (bit-cast to int64) and status;
        each rank then combines them in slab order, as ThreadExchange does, so
        the sums are deterministic."""
        dist = self.dist
        mine = np.empty(NFIELDS + 1, dtype=np.int64)
        mine[:NFIELDS] = np.asarray(tot, dtype=np.float64).view(np.int64)
        mine[NFIELDS] = _status_in(st[0])
        t = torch.from_numpy(mine).to(self.device)
        out = torch.empty(self.world * (NFIELDS + 1), dtype=torch.int64, device=self.device)
        dist.all_gather_into_tensor(out, t, group=self.group)
        rows = out.cpu().numpy().reshape(self.world, NFIELDS + 1)
        parts = [r[:NFIELDS].view(np.float64) for r in rows]
        res, key = combine_totals(parts, [int(r[NFIELDS]) for r in rows])
        tot[:] = res
        st[0] = _status_out(key)
        return 0

    def attach(self, slab: Slab):
        """Use this exchange as the slab's hooks (device buffers viewed in place)."""
        dev = torch.cuda.current_device()
        n = slab.local_rows * slab.w.nx

        def halo(H, Cc):
            torch.cuda.current_stream().wait_stream(slab.stream)
            self.exchange(device_view(H, n, dev), device_view(Cc, n, dev), slab.row0, slab.own0, slab.own1,
                          slab.local_rows)
            torch.cuda.current_stream().synchronize()
            return 0

        slab.set_hooks(halo, self.combine)
